// trtc_compact.cuh -- single-pass stable stream compaction and partition.
//
// Replaces the reference's compaction shape (internal/general_copy_if.cpp:26-64 and the
// partition scans of partition.cpp:29-125): a u32 flag scan through general_scan, a
// blocking copy of the count to the host, then a scatter kernel.  Here one kernel computes
// the flags from the tile it holds in registers, ranks the selected elements with warp
// ballots, finds the tile's output offset by decoupled look-back over selected counts and
// writes the selected elements (and, for partitions, the rejected ones at
// index - selected_before).  Inputs are read before a tile publishes anything, so the
// in-place forms (Remove, Remove_If, Unique, ...) need no copy of the input.
#pragma once
#include "trtc_scan.cuh"

namespace trtc {

enum CompactMode : int {
    CM_PRED = 0,             // pred(in[i])                       copy_if / partition
    CM_PRED_STENCIL = 1,     // pred(stencil[i])                  copy_if_stencil / partition_stencil
    CM_NOT_EQUAL = 2,        // in[i] != value                    remove / remove_copy
    CM_NOT_PRED = 3,         // !pred(in[i])                      remove_if / remove_copy_if
    CM_NOT_PRED_STENCIL = 4, // !pred(stencil[i])                 remove_if_stencil
    CM_UNIQUE = 5,           // i == 0 || in[i] != in[i-1]        unique (default)
    CM_UNIQUE_PRED = 6,      // i == 0 || !pred(in[i], in[i-1])   unique with binary_pred
    CM_TAIL = 7,             // i == n-1 || !pred(in[i], in[i+1]) reduce_by_key segment tails
};

// Element i of a view through the read-only path (ld.global.nc) when the view is contiguous
// and its elements are 4 or 8 bytes: the second array of the two-array forms is read at the
// selected elements only, and a read-only load can be issued ahead of the kernel's stores
// (which the compiler cannot prove do not alias it) instead of each one waiting behind them.
template <class T, class V>
TRTC_FORCEINLINE T ld_view_nc(const V& v, size_t i) {
    if constexpr (ViewTraits<V>::contiguous && sizeof(T) == 4) {
        const unsigned int b = __ldg(reinterpret_cast<const unsigned int*>(v._data + i));
        return *reinterpret_cast<const T*>(&b);
    } else if constexpr (ViewTraits<V>::contiguous && sizeof(T) == 8) {
        const unsigned long long b = __ldg(reinterpret_cast<const unsigned long long*>(v._data + i));
        return *reinterpret_cast<const T*>(&b);
    } else {
        return (T)v[i];
    }
}

// the element array of a contiguous view (nullptr for the others)
template <class T, class V>
TRTC_FORCEINLINE const T* view_ptr(const V& v) {
    if constexpr (ViewTraits<V>::contiguous) return reinterpret_cast<const T*>(v._data);
    else return nullptr;
}

// CT: type of the selected counts (32-bit while n < 2^32: flag and count then travel in one
// 64-bit look-back word)
template <int MODE, bool PARTITION, bool TWO, class InV, class StV, class Pred, class ValT, class OutV, class FalseV,
          class In2V, class Out2V, int BLOCK, int ITEMS, class CT = unsigned long long>
__global__ void __launch_bounds__(BLOCK) compact_kernel(InV in, StV stencil, Pred pred, ValT value, OutV out,
                                                        FalseV out_false, In2V in2, Out2V out2, size_t n,
                                                        LookbackState st) {
    typedef typename remove_cvref<typename InV::value_t>::type E;
    typedef typename remove_cvref<decltype(in2[0])>::type E2;
    constexpr int WARPS = BLOCK / 32;
    constexpr int TILE = BLOCK * ITEMS;
    __shared__ uint32_t s_slot[2];
    __shared__ uint32_t s_wcnt[WARPS];
    __shared__ CT s_pre;

    const size_t tile = claim_tile(st, s_slot);
    const size_t tile_base = tile * TILE;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const size_t wbase = tile_base + (size_t)warp * 32 * ITEMS;
    const uint32_t ltm = lanemask_lt();

    E v[ITEMS];
    E2 v2[TWO ? ITEMS : 1];
    bool f[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const size_t idx = wbase + (size_t)i * 32 + lane;
        const bool ok = idx < n;
        v[i] = ok ? (E)in[idx] : E();
        if constexpr (TWO) v2[i] = ok ? (E2)in2[idx] : E2();
    }
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const size_t idx = wbase + (size_t)i * 32 + lane;
        const bool ok = idx < n;
        bool sel = false;
        if constexpr (MODE == CM_PRED) sel = ok && (bool)pred(v[i]);
        else if constexpr (MODE == CM_PRED_STENCIL) sel = ok && (bool)pred(stencil[idx < n ? idx : 0]);
        else if constexpr (MODE == CM_NOT_EQUAL) sel = ok && !(v[i] == value);
        else if constexpr (MODE == CM_NOT_PRED) sel = ok && !(bool)pred(v[i]);
        else if constexpr (MODE == CM_NOT_PRED_STENCIL) sel = ok && !(bool)pred(stencil[idx < n ? idx : 0]);
        else if constexpr (MODE == CM_UNIQUE || MODE == CM_UNIQUE_PRED) {
            E prev = shfl_up_any(v[i], 1);
            const E last = i > 0 ? shfl_any(v[i > 0 ? i - 1 : 0], 31) : E();
            if (lane == 0) prev = (i > 0) ? last : ((ok && idx > 0) ? (E)in[idx - 1] : E());
            if constexpr (MODE == CM_UNIQUE) sel = ok && (idx == 0 || v[i] != prev);
            else sel = ok && (idx == 0 || !(bool)pred(v[i], prev));
        } else if constexpr (MODE == CM_TAIL) {
            E next = shfl_down_any(v[i], 1);
            const E first = i + 1 < ITEMS ? shfl_any(v[i + 1 < ITEMS ? i + 1 : i], 0) : E();
            if (lane == 31) next = (i + 1 < ITEMS) ? first : ((idx + 1 < n) ? (E)in[idx + 1] : E());
            sel = ok && (idx + 1 == n || !(bool)pred(v[i], next));
        }
        f[i] = sel;
    }
    // warp ranks
    uint32_t rank[ITEMS];
    uint32_t wc = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const uint32_t b = __ballot_sync(0xffffffffu, f[i]);
        rank[i] = wc + (uint32_t)__popc(b & ltm);
        wc += (uint32_t)__popc(b);
    }
    if (lane == 0) s_wcnt[warp] = wc;
    __syncthreads();

    if (warp == 0) {
        CT agg = 0;
        if (lane < (uint32_t)WARPS) agg = s_wcnt[lane];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) agg += __shfl_down_sync(0xffffffffu, agg, d);
        agg = __shfl_sync(0xffffffffu, agg, 0);
        CT pre = 0;
        Plus plus;
        if (tile > 0) {
            if (lane == 0) publish<CT>(st, tile, agg, false, false);
            bool dummy;
            pre = lookback_prefix<CT, Plus, false>(st, tile, plus, dummy).v;
        }
        if (lane == 0) {
            publish<CT>(st, tile, pre + agg, true, false);
            if (tile_base + TILE >= n && st.result) *reinterpret_cast<unsigned long long*>(st.result) = (unsigned long long)(pre + agg);
            s_pre = pre;
        }
    }
    __syncthreads();

    unsigned long long base = s_pre;
    for (uint32_t w = 0; w < warp; w++) base += s_wcnt[w];
    const size_t out_n = out.size();
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const size_t idx = wbase + (size_t)i * 32 + lane;
        if (idx >= n) continue;
        const unsigned long long before = base + rank[i];  // selected elements before idx
        if (f[i]) {
            if (before < out_n) {
                out[before] = v[i];
                if constexpr (TWO) {
                    if (before < (unsigned long long)out2.size()) out2[before] = v2[i];
                }
            }
        } else {
            if constexpr (PARTITION) {
                const unsigned long long fp = idx - before;
                if (fp < (unsigned long long)out_false.size()) out_false[fp] = v[i];
            }
        }
    }
}

#ifndef TRTC_COMPACT2_MINB
#define TRTC_COMPACT2_MINB 4  // resident CTAs per SM the two-phase kernel is compiled for
#endif
// Two-phase, persistent, software-pipelined form of compact_kernel for outputs that do not
// overlap the inputs (compiled for 4 resident CTAs per SM, the persistent grid's size): phase 1 reads a tile, evaluates the selection and publishes its count;
// phase 2 (after the look-back) reads the tile again -- normally from L2 -- and writes it.
// A CTA runs phase 1 of its next tile before the look-back of its current one, so the waits
// overlap HBM reads.  (In-place forms keep the one-pass kernel: a later tile may write into
// an earlier tile's range before that tile re-reads it.)
template <int MODE, bool PARTITION, bool TWO, class InV, class StV, class Pred, class ValT, class OutV, class FalseV,
          class In2V, class Out2V, int BLOCK, int ITEMS, class CT = unsigned long long>
__global__ void __launch_bounds__(BLOCK, TRTC_COMPACT2_MINB) compact2_kernel(InV in, StV stencil, Pred pred, ValT value, OutV out,
                                                         FalseV out_false, In2V in2, Out2V out2, size_t n,
                                                         size_t tiles, LookbackState st) {
    typedef typename remove_cvref<typename InV::value_t>::type E;
    typedef typename remove_cvref<decltype(in2[0])>::type E2;
    constexpr int WARPS = BLOCK / 32;
    constexpr int TILE = BLOCK * ITEMS;
    __shared__ unsigned long long s_ticket;
    __shared__ uint32_t s_wcnt[2][WARPS];
    __shared__ CT s_agg[2];
    __shared__ CT s_pre;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const uint32_t ltm = lanemask_lt();
    // 16-byte vector path for full, aligned tiles of 4-byte elements: lane l of a warp row
    // holds 4 consecutive elements.  Element-wise selections, and the neighbour tests of
    // unique (previous element) and of segment tails (next element), whose neighbours come
    // from the lane's own vector, the adjacent lane (shuffle), the adjacent row, or one global
    // load at the edge of the warp's segment; a second array (TWO) is read and written only
    // at the selected elements
    constexpr bool NEIGH = MODE == CM_UNIQUE || MODE == CM_UNIQUE_PRED || MODE == CM_TAIL;
    constexpr bool VECOK = ViewTraits<InV>::contiguous && ViewTraits<OutV>::contiguous && sizeof(E) == 4 && !PARTITION &&
                           (MODE == CM_PRED || MODE == CM_NOT_EQUAL || MODE == CM_NOT_PRED || NEIGH) &&
                           (!TWO || NEIGH);
    constexpr int VROWS = ITEMS / 4;
    typedef union { uint4 q; E t[4]; } Vec;
    // a contiguous second array of 4-byte elements (its rows can be read as 16-byte vectors)
    constexpr bool VEC2 = ViewTraits<In2V>::contiguous && sizeof(E2) == 4;
    // vector path: each warp gathers its selected elements in shared memory (placed so that
    // 16-byte aligned output addresses map to 16-byte aligned slots), then writes them with
    // 16-byte stores (scalar stores only at the run's ragged ends)
    constexpr int WSTAGE = 32 * ITEMS + 4;
    __shared__ __align__(16) E s_stage[VECOK ? WARPS * WSTAGE : 1];
    auto vec_fast = [&](size_t tile) -> bool {
        if constexpr (VECOK) return (tile + 1) * (size_t)TILE <= n && ((((size_t)in._data) & 15) == 0);
        else return false;
    };
    auto vsel = [&](const E& x) -> bool {
        if constexpr (MODE == CM_PRED) return (bool)pred(x);
        else if constexpr (MODE == CM_NOT_EQUAL) return !(x == value);
        else if constexpr (MODE == CM_NOT_PRED) return !(bool)pred(x);
        else return false;  // not used (the neighbour modes take row_flags)
    };
    // selections of row r of a warp segment starting at element wbase (rows u[0..VROWS) of
    // the segment in registers; edge_v: the element before the segment (unique) or after it
    // (tails), read by the caller where it exists)
    auto row_flags = [&](const Vec* u, int r, const E& edge_v, size_t wbase, bool (&f)[4]) {
        if constexpr (!NEIGH) {
#pragma unroll
            for (int e = 0; e < 4; e++) f[e] = vsel(u[r].t[e]);
        } else {
            const size_t i0 = wbase + (size_t)r * 128 + (size_t)lane * 4;
            if constexpr (MODE == CM_TAIL) {
                E nx = shfl_down_any(u[r].t[0], 1);
                const E nrow = (r + 1 < VROWS) ? shfl_any(u[r + 1 < VROWS ? r + 1 : r].t[0], 0) : edge_v;
                if (lane == 31) nx = nrow;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const E next = e < 3 ? u[r].t[e < 3 ? e + 1 : 3] : nx;
                    f[e] = i0 + e + 1 == n || !(bool)pred(u[r].t[e], next);
                }
            } else {
                E pv = shfl_up_any(u[r].t[3], 1);
                const E prow = r > 0 ? shfl_any(u[r > 0 ? r - 1 : 0].t[3], 31) : edge_v;
                if (lane == 0) pv = prow;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const E prev = e > 0 ? u[r].t[e > 0 ? e - 1 : 0] : pv;
                    if constexpr (MODE == CM_UNIQUE) f[e] = i0 + e == 0 || u[r].t[e] != prev;
                    else f[e] = i0 + e == 0 || !(bool)pred(u[r].t[e], prev);
                }
            }
        }
    };
    // the neighbour outside the warp segment [wbase, wbase + 32*ITEMS) (all lanes read it)
    auto edge_of = [&](size_t wbase) -> E {
        if constexpr (MODE == CM_TAIL) return wbase + 32 * ITEMS < n ? (E)in._data[wbase + 32 * ITEMS] : E();
        else if constexpr (NEIGH) return wbase > 0 ? (E)in._data[wbase - 1] : E();
        else return E();
    };

    auto claim = [&]() -> size_t {
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(st.tile_ctr, 1ull);
            if (t == (unsigned long long)tiles + gridDim.x - 1) atomicExch(st.tile_ctr, 0ull);
            s_ticket = t;
            // the input's tile ahead into L2 (the second array is read at selected elements only)
            if constexpr (ViewTraits<InV>::contiguous)
                if (st.pf_ahead) prefetch_l2_range(in._data, (size_t)(t + st.pf_ahead) * TILE, (size_t)TILE, n);
        }
        __syncthreads();
        return (size_t)s_ticket;
    };
    // loads the tile's elements of this thread and evaluates the selection
    auto load = [&](size_t tile, E (&v)[ITEMS], bool (&f)[ITEMS]) {
        const size_t wbase = tile * TILE + (size_t)warp * 32 * ITEMS;
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const size_t idx = wbase + (size_t)i * 32 + lane;
            v[i] = idx < n ? (E)in[idx] : E();
        }
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const size_t idx = wbase + (size_t)i * 32 + lane;
            const bool ok = idx < n;
            bool sel = false;
            if constexpr (MODE == CM_PRED) sel = ok && (bool)pred(v[i]);
            else if constexpr (MODE == CM_PRED_STENCIL) sel = ok && (bool)pred(stencil[idx < n ? idx : 0]);
            else if constexpr (MODE == CM_NOT_EQUAL) sel = ok && !(v[i] == value);
            else if constexpr (MODE == CM_NOT_PRED) sel = ok && !(bool)pred(v[i]);
            else if constexpr (MODE == CM_NOT_PRED_STENCIL) sel = ok && !(bool)pred(stencil[idx < n ? idx : 0]);
            else if constexpr (MODE == CM_UNIQUE || MODE == CM_UNIQUE_PRED) {
                E prev = shfl_up_any(v[i], 1);
                const E last = i > 0 ? shfl_any(v[i > 0 ? i - 1 : 0], 31) : E();
                if (lane == 0) prev = (i > 0) ? last : ((ok && idx > 0) ? (E)in[idx - 1] : E());
                if constexpr (MODE == CM_UNIQUE) sel = ok && (idx == 0 || v[i] != prev);
                else sel = ok && (idx == 0 || !(bool)pred(v[i], prev));
            } else if constexpr (MODE == CM_TAIL) {
                E next = shfl_down_any(v[i], 1);
                const E first = i + 1 < ITEMS ? shfl_any(v[i + 1 < ITEMS ? i + 1 : i], 0) : E();
                if (lane == 31) next = (i + 1 < ITEMS) ? first : ((idx + 1 < n) ? (E)in[idx + 1] : E());
                sel = ok && (idx + 1 == n || !(bool)pred(v[i], next));
            }
            f[i] = sel;
        }
    };
    auto phase1 = [&](size_t tile, int b) {
        uint32_t wc = 0;
        if (vec_fast(tile)) {
            if constexpr (VECOK) {
                const size_t wb = tile * TILE + (size_t)warp * 32 * ITEMS;
                const uint4* p = reinterpret_cast<const uint4*>(in._data + wb);
                uint32_t c = 0;
                if constexpr (NEIGH) {
                    Vec u[VROWS];
#pragma unroll
                    for (int r = 0; r < VROWS; r++) u[r].q = p[r * 32 + lane];
                    const E edge = edge_of(wb);
#pragma unroll
                    for (int r = 0; r < VROWS; r++) {
                        bool f[4];
                        row_flags(u, r, edge, wb, f);
                        uint32_t rc = 0;
#pragma unroll
                        for (int e = 0; e < 4; e++) rc += f[e] ? 1u : 0u;
                        c += rc;
                        // the second array's selected rows into L2 for phase 2 (one tile later)
                        if constexpr (TWO && VEC2)
                            if (rc) asm volatile("prefetch.global.L2 [%0];" ::"l"(view_ptr<E2>(in2) + wb + (size_t)r * 128 + (size_t)lane * 4));
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < VROWS; r++) {
                        Vec u;
                        u.q = p[r * 32 + lane];
#pragma unroll
                        for (int e = 0; e < 4; e++) c += vsel(u.t[e]) ? 1u : 0u;
                    }
                }
                wc = __reduce_add_sync(0xffffffffu, c);
            }
        } else {
            E v[ITEMS];
            bool f[ITEMS];
            load(tile, v, f);
#pragma unroll
            for (int i = 0; i < ITEMS; i++) wc += (uint32_t)__popc(__ballot_sync(0xffffffffu, f[i]));
        }
        if (lane == 0) s_wcnt[b][warp] = wc;
        __syncthreads();
        if (threadIdx.x == 0) {
            CT agg = 0;
            for (int w = 0; w < WARPS; w++) agg += s_wcnt[b][w];
            s_agg[b] = agg;
            if (tile == 0) {
                publish<CT>(st, 0, agg, true, false);
                if (tiles == 1 && st.result) *reinterpret_cast<unsigned long long*>(st.result) = (unsigned long long)agg;
            } else {
                publish<CT>(st, tile, agg, false, false);
            }
        }
    };

    size_t cur = claim();
    if (cur >= tiles) return;
    int buf = 0;
    phase1(cur, 0);
    while (true) {
        const size_t nxt = claim();
        if (nxt < tiles) phase1(nxt, buf ^ 1);
        if (warp == 0) {
            CT pre = 0;
            if (cur > 0) {
                Plus plus;
                bool dummy;
                pre = lookback_prefix<CT, Plus, false>(st, cur, plus, dummy).v;
                if (lane == 0) {
                    publish<CT>(st, cur, (CT)(pre + s_agg[buf]), true, false);
                    if (cur == tiles - 1 && st.result) *reinterpret_cast<unsigned long long*>(st.result) = (unsigned long long)(pre + s_agg[buf]);
                }
            }
            if (lane == 0) s_pre = pre;
        }
        __syncthreads();
        if (vec_fast(cur)) {
            if constexpr (VECOK) {
                unsigned long long run = s_pre;
                for (uint32_t w = 0; w < warp; w++) run += s_wcnt[buf][w];
                const size_t wb = cur * TILE + (size_t)warp * 32 * ITEMS;
                const uint4* p = reinterpret_cast<const uint4*>(in._data + wb);
                Vec u[VROWS];
#pragma unroll
                for (int r = 0; r < VROWS; r++) u[r].q = p[r * 32 + lane];
                const E edge = edge_of(wb);
                const unsigned long long out_n = out.size();
                E* sbuf = s_stage + warp * WSTAGE;
                // slot j of sbuf holds output element run + (j - s0)
                const uint32_t s0 = (uint32_t)((reinterpret_cast<size_t>(out._data + run) >> 2) & 3u);
                // two-array forms with a 16-byte aligned, contiguous 4-byte second array: every
                // row's selections first, then one 16-byte load per row holding a selected
                // element, all issued before any store (a load per selected element placed at
                // its store waits a memory round trip per row)
                constexpr bool PRE2 = TWO && VEC2;
                uint32_t fmask = 0;
                Vec u2[PRE2 ? VROWS : 1];
                const bool pre2 = PRE2 && ((reinterpret_cast<size_t>(view_ptr<E2>(in2) + wb) & 15u) == 0);
                if (PRE2 && pre2) {
#pragma unroll
                    for (int r = 0; r < VROWS; r++) {
                        bool f[4];
                        row_flags(u, r, edge, wb, f);
#pragma unroll
                        for (int e = 0; e < 4; e++) fmask |= (f[e] ? 1u : 0u) << (r * 4 + e);
                    }
#pragma unroll
                    for (int r = 0; r < (PRE2 ? VROWS : 1); r++)
                        if ((fmask >> (r * 4)) & 15u)
                            u2[r].q = __ldg(reinterpret_cast<const uint4*>(view_ptr<E2>(in2) + wb + (size_t)r * 128) + lane);
                }
                uint32_t tot = 0;
#pragma unroll
                for (int r = 0; r < VROWS; r++) {
                    bool f[4];
                    uint32_t c = 0;
                    if (PRE2 && pre2) {
#pragma unroll
                        for (int e = 0; e < 4; e++) f[e] = (fmask >> (r * 4 + e)) & 1u;
                    } else {
                        row_flags(u, r, edge, wb, f);
                    }
#pragma unroll
                    for (int e = 0; e < 4; e++) c += f[e] ? 1u : 0u;
                    uint32_t x = c;  // inclusive prefix of the lane counts
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
                        if (lane >= (uint32_t)d) x += y;
                    }
                    uint32_t pos = s0 + tot + (x - c);
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        if (!f[e]) continue;
                        if constexpr (TWO) {  // the second array at the selected element, stored singly
                            const unsigned long long g = run + (pos - s0);
                            if (g < (unsigned long long)out2.size()) {
                                if (PRE2 && pre2) out2[g] = *reinterpret_cast<const E2*>(&u2[PRE2 ? r : 0].t[e]);
                                else out2[g] = ld_view_nc<E2>(in2, wb + (size_t)r * 128 + (size_t)lane * 4 + e);
                            }
                        }
                        sbuf[pos++] = u[r].t[e];
                    }
                    tot += __shfl_sync(0xffffffffu, x, 31);
                }
                __syncwarp();
                const uint32_t end = s0 + tot;
                for (uint32_t j0 = lane * 4; j0 < end; j0 += 128) {
                    const unsigned long long g0 = run + j0 - s0;  // output index of slot j0 (j0 >= s0)
                    if (j0 >= s0 && j0 + 4 <= end && g0 + 4 <= out_n) {
                        *reinterpret_cast<uint4*>(out._data + g0) = *reinterpret_cast<const uint4*>(sbuf + j0);
                    } else {
#pragma unroll
                        for (uint32_t k = 0; k < 4; k++) {
                            const uint32_t j = j0 + k;
                            if (j >= s0 && j < end && run + (j - s0) < out_n) out._data[run + (j - s0)] = sbuf[j];
                        }
                    }
                }
                __syncwarp();  // the buffer is refilled by this warp's next tile
            }
        } else {
            E v[ITEMS];
            bool f[ITEMS];
            load(cur, v, f);
            // TWO: the second array is read at the selected elements only (the outputs never
            // overlap the inputs in this kernel); a register copy of the whole row set would
            // read all of it and spill
            const size_t wbase = cur * TILE + (size_t)warp * 32 * ITEMS;
            unsigned long long base = s_pre;
            for (uint32_t w = 0; w < warp; w++) base += s_wcnt[buf][w];
            const size_t out_n = out.size();
            uint32_t wc = 0;
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const uint32_t bal = __ballot_sync(0xffffffffu, f[i]);
                const size_t idx = wbase + (size_t)i * 32 + lane;
                const unsigned long long before = base + wc + (uint32_t)__popc(bal & ltm);
                wc += (uint32_t)__popc(bal);
                if (idx >= n) continue;
                if (f[i]) {
                    if (before < out_n) {
                        out[before] = v[i];
                        if constexpr (TWO) {
                            if (before < (unsigned long long)out2.size()) out2[before] = ld_view_nc<E2>(in2, idx);
                        }
                    }
                } else {
                    if constexpr (PARTITION) {
                        const unsigned long long fp = idx - before;
                        if (fp < (unsigned long long)out_false.size()) out_false[fp] = v[i];
                    }
                }
            }
        }
        if (nxt >= tiles) break;
        cur = nxt;
        buf ^= 1;
    }
}

// Partition in place: rejected elements were compacted into a temp buffer; move them
// behind the selected ones once the count is known on the device.
template <class E>
__global__ void partition_tail_kernel(const E* __restrict__ tmp, E* __restrict__ out, size_t n,
                                      const unsigned long long* count) {
    const unsigned long long c = *count;
    const size_t nf = n - (size_t)c;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += (size_t)gridDim.x * blockDim.x)
        out[c + i] = tmp[i];
}

}  // namespace trtc
