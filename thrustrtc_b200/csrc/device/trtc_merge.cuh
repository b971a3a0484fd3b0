// trtc_merge.cuh -- stable comparison sort for user comparators, and generic view copies.
//
// The reference sorts with a user Functor comparator (or non-radix key types) through a
// merge sort (internal/merge_sort.cpp:7-280): 512-element block sorts in shared memory,
// then pairwise merges of sorted runs where every element finds its output position by a
// binary search in the partner run.  The same stable scheme is restated here with the
// comparator as a template slot, instantiated by NVRTC with the user's Functor struct:
//   * block sort: an element's rank inside its block is the number of block elements that
//     must precede it (strictly smaller ones, and equal ones with a smaller index);
//   * merge level: an element of the left run lands at its index in the run plus the number
//     of right-run elements strictly smaller (lower bound); an element of the right run at
//     its index plus the number of left-run elements not greater (upper bound).  Ties keep
//     left before right, which keeps the sort stable.
#pragma once
#include "trtc_prelude.cuh"
#include "trtc_builtins.cuh"

namespace trtc {

template <class KV, class VV, class Comp, bool HAS_VALS, int BLOCK>
__global__ void __launch_bounds__(BLOCK) merge_block_sort_kernel(KV keys, VV vals, Comp comp, size_t n,
                                                                 typename remove_cvref<typename KV::value_t>::type* out_k,
                                                                 void* out_v_raw) {
    typedef typename remove_cvref<typename KV::value_t>::type K;
    typedef typename remove_cvref<decltype(vals[0])>::type V;
    constexpr int T = BLOCK * 2;
    __shared__ K s_k[T];
    V* out_v = reinterpret_cast<V*>(out_v_raw);
    const size_t base = (size_t)blockIdx.x * T;
    const int cnt = (int)((n - base) < (size_t)T ? (n - base) : (size_t)T);
    for (int i = threadIdx.x; i < cnt; i += BLOCK) s_k[i] = keys[base + i];
    __syncthreads();
    for (int i = threadIdx.x; i < cnt; i += BLOCK) {
        const K ki = s_k[i];
        int rank = 0;
        for (int j = 0; j < i; j++) rank += comp(ki, s_k[j]) ? 0 : 1;
        for (int j = i + 1; j < cnt; j++) rank += comp(s_k[j], ki) ? 1 : 0;
        out_k[base + rank] = ki;
        if constexpr (HAS_VALS) out_v[base + rank] = vals[base + i];
    }
}

template <class K, class V, class Comp, bool HAS_VALS>
__global__ void merge_level_kernel(const K* __restrict__ in_k, const V* __restrict__ in_v, K* __restrict__ out_k,
                                   V* __restrict__ out_v, size_t n, size_t width, Comp comp) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t a0 = (i / (2 * width)) * (2 * width);
        const size_t mid = a0 + width < n ? a0 + width : n;
        const size_t end = a0 + 2 * width < n ? a0 + 2 * width : n;
        const K ki = in_k[i];
        size_t pos;
        if (i < mid) {
            size_t lo = mid, hi = end;  // first right element not smaller than ki
            while (lo < hi) {
                const size_t m = lo + ((hi - lo) >> 1);
                if (comp(in_k[m], ki)) lo = m + 1; else hi = m;
            }
            pos = (i - a0) + (lo - mid);
        } else {
            size_t lo = a0, hi = mid;  // first left element greater than ki
            while (lo < hi) {
                const size_t m = lo + ((hi - lo) >> 1);
                if (comp(ki, in_k[m])) hi = m; else lo = m + 1;
            }
            pos = (i - mid) + (lo - a0);
        }
        out_k[a0 + pos] = ki;
        if constexpr (HAS_VALS) out_v[a0 + pos] = in_v[i];
    }
}

// out[out_off + i] = (out element type) in[in_off + i] for i < count, where count is n, or
// n - *tail_base when tail_base is given (partition tails whose length is known on device).
template <class InV, class OutV>
__global__ void copy_view_kernel(InV in, OutV out, size_t n, size_t in_off, size_t out_off,
                                 const unsigned long long* tail_base) {
    typedef typename remove_cvref<typename OutV::value_t>::type O;
    size_t count = n;
    size_t ooff = out_off;
    if (tail_base) {
        count = n - (size_t)*tail_base;
        ooff += (size_t)*tail_base;
    }
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        out[ooff + i] = (O)in[in_off + i];
}

}  // namespace trtc
