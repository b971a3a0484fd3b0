// trtc_misc.cuh -- the reference's remaining algorithms as NVRTC-instantiated kernels over
// any views and user functors: element-wise transforms (fill, sequence, tabulate,
// transform*, replace*, for_each, adjacent_difference, gather*, scatter*, swap), counts,
// first-index searches (find*, mismatch, is_sorted_until, partition_point and the boolean
// forms built on them), the index-reduction tree of max/min element, and merges.
// Grid-stride loops; each search CTA skips work once an earlier index has been found.
#pragma once
#include "trtc_builtins.cuh"

namespace trtc {

#define TRTC_GRID_LOOP(i, n) \
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

template <class V> using value_of = typename remove_cvref<typename V::value_t>::type;

// ---------------------------------------------------------------- element-wise
template <class V, class T>
__global__ void fill_kernel(V vec, T value, size_t n) {
    TRTC_GRID_LOOP(i, n) vec[i] = (value_of<V>)value;
}

// vec[i] = init + i * step in the element type (sequence.cpp:24-33)
template <class V, class TI, class TS>
__global__ void sequence_kernel(V vec, TI init, TS step, size_t n) {
    typedef value_of<V> E;
    TRTC_GRID_LOOP(i, n) vec[i] = (E)init + (E)i * (E)step;
}

// vec[i] = op(vec[i]): the reference's Tabulate applies op to the element in place
// (tabulate.cpp:5-7), which is what its programs depend on
template <class V, class Op>
__global__ void tabulate_kernel(V vec, Op op, size_t n) {
    TRTC_GRID_LOOP(i, n) vec[i] = (value_of<V>)op(vec[i]);
}

template <class V, class F>
__global__ void for_each_kernel(V vec, F f, size_t n) {
    TRTC_GRID_LOOP(i, n) f(vec[i]);
}

// out[i] = op(in[i]) where the selector holds (MODE 0: always, 1: pred(in[i]), 2: pred(st[i]))
template <int MODE, class In, class St, class Out, class Op, class Pred>
__global__ void transform_kernel(In in, St st, Out out, Op op, Pred pred, size_t n) {
    TRTC_GRID_LOOP(i, n) {
        if constexpr (MODE == 1) { if (!pred(in[i])) continue; }
        if constexpr (MODE == 2) { if (!pred(st[i])) continue; }
        out[i] = (value_of<Out>)op(in[i]);
    }
}

// out[i] = op(in1[i], in2[i]) (STENCIL: where pred(st[i]))
template <bool STENCIL, class In1, class In2, class St, class Out, class Op, class Pred>
__global__ void transform_binary_kernel(In1 in1, In2 in2, St st, Out out, Op op, Pred pred, size_t n) {
    TRTC_GRID_LOOP(i, n) {
        if constexpr (STENCIL) { if (!pred(st[i])) continue; }
        out[i] = (value_of<Out>)op(in1[i], in2[i]);
    }
}

// out[i] = selected ? new_value : in[i]; selected = in[i] == old_value (PRED false) or pred(in[i])
template <bool PRED, class In, class Out, class T, class P, class T2>
__global__ void replace_kernel(In in, Out out, T old_value, P pred, T2 new_value, size_t n) {
    TRTC_GRID_LOOP(i, n) {
        const value_of<In> v = in[i];
        bool sel;
        if constexpr (PRED) sel = (bool)pred(v);
        else sel = v == (value_of<In>)old_value;
        out[i] = sel ? (value_of<Out>)new_value : (value_of<Out>)v;
    }
}

// out[0] = in[0], out[i] = op(in[i], in[i-1]) (adjacent_difference.cpp:15-27); `in` never aliases `out`
template <class In, class Out, class Op>
__global__ void adjacent_difference_kernel(In in, Out out, Op op, size_t n) {
    TRTC_GRID_LOOP(i, n) {
        value_of<In> v = in[i];
        if (i > 0) v = (value_of<In>)op(v, in[i - 1]);
        out[i] = (value_of<Out>)v;
    }
}

// out[i] = in[map[i]] where the selector holds (SEL 0: always, 1: st[i] is true, 2: pred(st[i]))
template <int SEL, class Map, class St, class In, class Out, class Pred>
__global__ void gather_kernel(Map map, St st, In in, Out out, Pred pred, size_t n) {
    TRTC_GRID_LOOP(i, n) {
        if constexpr (SEL == 1) { if (!st[i]) continue; }
        if constexpr (SEL == 2) { if (!pred(st[i])) continue; }
        out[i] = (value_of<Out>)in[map[i]];
    }
}

// out[map[i]] = in[i] where the selector holds (SEL as for gather)
template <int SEL, class In, class Map, class St, class Out, class Pred>
__global__ void scatter_kernel(In in, Map map, St st, Out out, Pred pred, size_t n) {
    TRTC_GRID_LOOP(i, n) {
        if constexpr (SEL == 1) { if (!st[i]) continue; }
        if constexpr (SEL == 2) { if (!pred(st[i])) continue; }
        out[map[i]] = (value_of<Out>)in[i];
    }
}

template <class V1, class V2>
__global__ void swap_kernel(V1 a, V2 b, size_t n) {
    TRTC_GRID_LOOP(i, n) {
        const value_of<V1> t = a[i];
        a[i] = (value_of<V1>)b[i];
        b[i] = (value_of<V2>)t;
    }
}

// ---------------------------------------------------------------- counts
// MODE 0: v[i] == value, 1: pred(v[i]); per-CTA totals added to *count
template <int MODE, class V, class T, class Pred>
__global__ void __launch_bounds__(256) count_kernel(V vec, T value, Pred pred, size_t n, unsigned long long* count) {
    __shared__ unsigned long long s_w[8];
    unsigned long long c = 0;
    TRTC_GRID_LOOP(i, n) {
        if constexpr (MODE == 0) c += (vec[i] == (value_of<V>)value) ? 1 : 0;
        else c += (bool)pred(vec[i]) ? 1 : 0;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
    if ((threadIdx.x & 31u) == 0) s_w[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s_w[w];
        if (t) atomicAdd(count, t);
    }
}

// ---------------------------------------------------------------- first index with a property
enum FindMode : int {
    FIND_VALUE = 0,       // v[i] == value (find.cpp:6, no conversion of value)
    FIND_IF = 1,          // pred(v[i])
    FIND_IF_NOT = 2,      // !pred(v[i])
    FIND_MISMATCH = 3,    // !pred(v[i], w[i]) (mismatch.cpp, equal.cpp with a predicate)
    FIND_NE = 4,          // v[i] != w[i] (mismatch.cpp default)
    FIND_NE_CAST = 5,     // v[i] != (value_t of v)w[i] (equal.cpp default)
    FIND_UNSORTED = 6,    // comp(v[i], v[i-1]), i >= 1 (sort.cpp is_sorted / is_sorted_until)
    FIND_PART_BREAK = 7,  // !pred(v[i-1]) && pred(v[i]), i >= 1 (partition.cpp is_partitioned)
};

// *res = min(*res, first index in [begin, n) with the property); *res starts at n
template <int MODE, class V, class W, class T, class Pred>
__global__ void __launch_bounds__(256) find_first_kernel(V v, W w, T value, Pred pred, size_t begin, size_t n,
                                                         unsigned long long* res) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t base = begin + (size_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        // an index at or below this CTA's next chunk was already found: stop
        if (*(volatile unsigned long long*)res <= base) return;
        const size_t i = base + threadIdx.x;
        bool hit = false;
        if (i < n) {
            if constexpr (MODE == FIND_VALUE) hit = v[i] == value;
            else if constexpr (MODE == FIND_IF) hit = (bool)pred(v[i]);
            else if constexpr (MODE == FIND_IF_NOT) hit = !(bool)pred(v[i]);
            else if constexpr (MODE == FIND_MISMATCH) hit = !(bool)pred(v[i], w[i]);
            else if constexpr (MODE == FIND_NE) hit = v[i] != w[i];
            else if constexpr (MODE == FIND_NE_CAST) hit = v[i] != (value_of<V>)w[i];
            else if constexpr (MODE == FIND_UNSORTED) hit = i > 0 && (bool)pred(v[i], v[i - 1]);
            else hit = i > 0 && !(bool)pred(v[i - 1]) && (bool)pred(v[i]);
        }
        if (hit) atomicMin(res, (unsigned long long)i);
    }
}

// ---------------------------------------------------------------- index-reduction tree
// The reference's element-index reduction (extrema.cpp over internal/general_reduce.cpp:55-95):
// blocks of 256 consecutive slots, inside a block s = 128..1 with
// "if (tid < s && i + s < m) h[tid] = op(h[tid], h[tid+s])"; later rounds repeat the tree on
// the block results.  MAX: op(i1, i2) = comp(v[i1], v[i2]) ? i2 : i1; min: comp(v[i2], v[i1]) ? i2 : i1.
template <bool MAX, bool FIRST, class V, class Comp>
__global__ void __launch_bounds__(256) index_tree_kernel(V v, Comp comp, const unsigned long long* in, size_t m,
                                                         unsigned long long* out) {
    __shared__ unsigned long long h[256];
    const size_t nb = (m + 255) / 256;
    for (size_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const size_t base = b * 256;
        const uint32_t L = (uint32_t)((m - base) < 256 ? (m - base) : 256);
        const uint32_t t = threadIdx.x;
        if (t < L) h[t] = FIRST ? (unsigned long long)(base + t) : in[base + t];
        __syncthreads();
        for (uint32_t s = 128; s > 0; s >>= 1) {
            if (t < s && t + s < L) {
                const unsigned long long i1 = h[t], i2 = h[t + s];
                bool take2;
                if constexpr (MAX) take2 = (bool)comp(v[i1], v[i2]);
                else take2 = (bool)comp(v[i2], v[i1]);
                h[t] = take2 ? i2 : i1;
            }
            __syncthreads();
        }
        if (t == 0) out[b] = h[0];
        __syncthreads();
    }
}

// ---------------------------------------------------------------- merge
// Rank merge (merge.cpp:5-20): a[i] lands at i + #(b < a[i]) (lower bound in b), b[j] at
// j + #(a <= b[j]) (upper bound in a), so a's elements come first among equals.  One thread
// per index of the longer input places a[idx] and b[idx].  VALS: values follow their keys.
template <bool VALS, class A, class B, class Out, class VA, class VB, class VOut, class Comp>
__global__ void merge_kernel(A a, B b, Out out, VA va, VB vb, VOut vout, Comp comp, size_t na, size_t nb) {
    const size_t n = na > nb ? na : nb;
    TRTC_GRID_LOOP(k, n) {
        if (k < na) {
            const value_of<A> x = a[k];
            size_t lo = 0, hi = nb;
            while (lo < hi) {
                const size_t mid = lo + ((hi - lo) >> 1);
                if ((bool)comp(b[mid], x)) lo = mid + 1;
                else hi = mid;
            }
            out[k + lo] = (value_of<Out>)x;
            if constexpr (VALS) vout[k + lo] = (value_of<VOut>)va[k];
        }
        if (k < nb) {
            const value_of<B> y = b[k];
            size_t lo = 0, hi = na;
            while (lo < hi) {
                const size_t mid = lo + ((hi - lo) >> 1);
                if ((bool)comp(y, a[mid])) hi = mid;
                else lo = mid + 1;
            }
            out[k + lo] = (value_of<Out>)y;
            if constexpr (VALS) vout[k + lo] = (value_of<VOut>)vb[k];
        }
    }
}

// a * b under the operands' own arithmetic conversions: the default inner-product term
// (inner_product.cpp:7 multiplies vec1[i] * vec2[i] directly)
struct ProductOf {
    template <class A, class B>
    __device__ auto operator()(const A& a, const B& b) const { return a * b; }
};

// element i = op(a[i], b[i]) in type T: the terms of an inner product
template <class T, class A, class B, class Op>
struct BinaryTransformView {
    typedef T value_t;
    typedef T ref_t;
    A _a;
    B _b;
    Op _op;
    __device__ size_t size() const { return _a.size(); }
    __device__ T operator[](size_t i) { return (T)_op(_a[i], _b[i]); }
};

#undef TRTC_GRID_LOOP

}  // namespace trtc
