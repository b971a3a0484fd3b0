// trtc_scan.cuh -- single-pass scans (decoupled look-back), segmented scans and reductions.
//
// Replaces the reference's 512-element block scan + recursive block-sum scan + add-back
// (internal/general_scan.cpp:8-88), its segmented variant with an 'active' array
// (internal/general_scan_by_key.cpp:8-143) and its 256-wide recursive tree reduction
// (internal/general_reduce.cpp:30-95) with one pass over the data each.
//
// Tiles are claimed in launch order from an atomic counter, so a tile only ever waits for
// tiles that are already running.  Every wait is bounded (TRTC_SPIN_LIMIT) and reports an
// error instead of hanging.  Look-back flags are tagged with a per-call epoch so the flag
// array never needs clearing between calls.  Operators need only be associative: all
// combinations keep index order (older operand on the left), no identity element is used.
#pragma once

// Test hook of the two-phase scan: a build that defines TRTC_FAULT_SKIP_PUBLISH(tile) true for
// some tile leaves that tile's look-back word unpublished, so the bounded waits of the tiles
// after it run out (launch_faultinject.cu).  Every other build leaves it false.
#ifndef TRTC_FAULT_SKIP_PUBLISH
#define TRTC_FAULT_SKIP_PUBLISH(tile) false
#endif
#include "trtc_prelude.cuh"
#include "trtc_builtins.cuh"
#include "trtc_abi.h"

namespace trtc {


// ---------------------------------------------------------------- loaders
// A scan source: element i of the scanned sequence is get(fetch(i)) (a view read, optionally
// followed by the unary op of a transform scan), converted to the scan's value type T.
template <class InV, class T, class UOp, bool HAS_UOP>
struct ScanSrc {
    typedef typename remove_cvref<typename InV::value_t>::type E;
    static constexpr bool CONTIG = ViewTraits<InV>::contiguous;
    InV in;
    UOp uop;
    TRTC_FORCEINLINE T get(const E& raw) {
        if constexpr (HAS_UOP) return (T)uop(raw);
        else return (T)raw;
    }
    TRTC_FORCEINLINE E fetch(size_t i) { return in[i]; }
};

template <class E> struct VecWidth {
    static constexpr int V = (sizeof(E) == 1 || sizeof(E) == 2 || sizeof(E) == 4 || sizeof(E) == 8 || sizeof(E) == 16)
                                 ? (int)(16 / sizeof(E)) : 1;
};

template <class T> struct Opt { T v; bool h; };

// a ⊕ b with optional operands (either may be absent)
template <class T, class Op>
TRTC_FORCEINLINE void opt_combine(T& a, bool& ah, const T& b, bool bh, Op& op) {
    if (bh) { a = ah ? (T)op(a, b) : b; ah = true; }
}

// ---------------------------------------------------------------- look-back (warp 0)
// Returns the ordered combination of all tiles before `tile` (their values being inclusive
// prefixes or aggregates).  SEG: stop at the first tile holding a segment head as well, and
// combine with the segmented operator (a head in the right operand discards the left).
//
// One round trip polls TRTC_LB_K blocks of 32 consecutive predecessor tiles (coalesced
// relaxed loads, all in flight together): the inclusive frontier must advance as fast as
// tiles start on 148 SMs.  Values of <= 4 bytes travel in the same 64-bit word as their
// flag (no fence, no second load); larger values are read after one acquire fence.
#ifndef TRTC_LB_K
#define TRTC_LB_K 1
#endif
template <class T> struct LbPack { static constexpr bool value = sizeof(T) <= 4; };

template <class T>
TRTC_FORCEINLINE uint32_t lb_bits(const T& v) {
    union U { T t; uint32_t u; TRTC_FORCEINLINE U() : u(0) {} } c;
    c.t = v;
    return c.u;
}
template <class T>
TRTC_FORCEINLINE T lb_value(uint32_t u) {
    union U { T t; uint32_t u; TRTC_FORCEINLINE U() : u(0) {} } c;
    c.u = u;
    return c.t;
}
TRTC_FORCEINLINE uint32_t lb_state(uint32_t fw, uint32_t epoch8) {
    const uint32_t r = fw - epoch8;  // valid words: 1, 2, 5, 6
    return (fw >= epoch8 && r < 8u && (r & 3u) != 0u && (r & 3u) != 3u) ? r : 0u;
}

// Ordered combination of tiles 0..j_start (walking back from j_start).
template <class T, class Op, bool SEG>
__device__ inline Opt<T> lookback_walk(const LookbackState& st, long long j_start, Op& op, bool& seg_flag_out) {
    constexpr int K = TRTC_LB_K;
    constexpr bool PACK = LbPack<T>::value;
    const uint32_t lane = lane_id();
    T acc = T();
    bool has = false, acc_head = false, done = false;
    long long j0 = j_start;  // newest tile not yet combined
    while (!done && j0 >= 0) {
        // ---- poll K blocks of 32 tiles: lane l of block k holds tile j0 - 32k - l
        uint32_t code[K];
        T val[K];
        uint32_t spins = 0;
        while (true) {
            bool ready = true;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const long long j = j0 - 32ll * k - (long long)lane;
                code[k] = 8u;  // beyond tile 0
                if (j >= 0) {
                    if constexpr (PACK) {
                        const unsigned long long w = ld_relaxed(&st.packed[j]);
                        code[k] = lb_state((uint32_t)(w >> 32), st.epoch8);
                        val[k] = lb_value<T>((uint32_t)w);
                    } else {
                        code[k] = lb_state(ld_relaxed(&st.flags[j]), st.epoch8);
                    }
                    ready = ready && code[k] != 0u;
                }
            }
            if (__all_sync(0xffffffffu, ready)) break;
            if (!spin_continue(spins, st.err)) {
                report_error(st.err, TRTC_ERR_LOOKBACK_TIMEOUT);
#pragma unroll
                for (int k = 0; k < K; k++) if (code[k] == 0u) code[k] = 2u;
                break;
            }
        }
        if constexpr (!PACK) {
            fence_acq_rel();  // values are read after their flags
            const T* agg = reinterpret_cast<const T*>(st.agg);
            const T* inc = reinterpret_cast<const T*>(st.incl);
#pragma unroll
            for (int k = 0; k < K; k++) {
                const long long j = j0 - 32ll * k - (long long)lane;
                val[k] = T();
                if (j >= 0) val[k] = ((code[k] & 3u) == 2u) ? inc[j] : agg[j];
            }
        }
        // ---- combine block by block, newest first (older values are left operands)
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (done) continue;
            const uint32_t c = code[k];
            const bool beyond = c == 8u;
            const bool hd0 = SEG && !beyond && (c & 4u);
            const bool stop_here = beyond || (c & 3u) == 2u || hd0;
            const uint32_t stop_mask = __ballot_sync(0xffffffffu, stop_here);
            const int stop = stop_mask ? __ffs(stop_mask) - 1 : 31;
            T v = val[k];
            bool vh = (int)lane <= stop && !beyond;
            bool hd = hd0;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const T o = shfl_down_any(v, d);
                const int oh_i = __shfl_down_sync(0xffffffffu, (int)vh, d);
                const int ohd = __shfl_down_sync(0xffffffffu, (int)hd, d);
                const bool oh = oh_i && ((int)lane + d < 32);
                if ((lane & (2 * d - 1)) == 0 && oh) {
                    if (SEG) {
                        if (!vh) { v = o; hd = ohd; }
                        else if (!hd) { v = (T)op(o, v); hd = ohd; }
                    } else {
                        v = vh ? (T)op(o, v) : o;
                    }
                    vh = true;
                }
            }
            if (vh && lane == 0) {
                if (SEG) {
                    if (!has) { acc = v; acc_head = hd; }
                    else if (!acc_head) { acc = (T)op(v, acc); acc_head = hd; }
                } else {
                    acc = has ? (T)op(v, acc) : v;
                }
                has = true;
            }
            if (stop_mask) done = true;
        }
        j0 -= 32ll * K;
    }
    Opt<T> r;
    r.v = shfl_any(acc, 0);
    r.h = __shfl_sync(0xffffffffu, (int)has, 0) != 0;
    seg_flag_out = __shfl_sync(0xffffffffu, (int)acc_head, 0) != 0;
    return r;
}

template <class T, class Op, bool SEG>
__device__ inline Opt<T> lookback_prefix(const LookbackState& st, size_t tile, Op& op, bool& seg_flag_out) {
    return lookback_walk<T, Op, SEG>(st, (long long)tile - 1, op, seg_flag_out);
}

template <class T>
TRTC_FORCEINLINE void publish(const LookbackState& st, size_t tile, const T& v, bool inclusive, bool head) {
    const uint32_t fw = st.epoch8 + (inclusive ? 2u : 1u) + (head ? 4u : 0u);
    if constexpr (LbPack<T>::value) {
        // flag and value in one single-copy-atomic 64-bit store
        const unsigned long long w = ((unsigned long long)fw << 32) | (unsigned long long)lb_bits<T>(v);
        asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(&st.packed[tile]), "l"(w) : "memory");
    } else {
        T* dst = reinterpret_cast<T*>(inclusive ? st.incl : st.agg);
        dst[tile] = v;
        st_release(&st.flags[tile], fw);
    }
}

TRTC_FORCEINLINE size_t claim_tile(const LookbackState& st, uint32_t* s_slot) {
    __syncthreads();
    if (threadIdx.x == 0) {
        // tiles are handed out in launch order; the CTA that takes the last ticket resets
        // the counter for the next launch on this stream (every ticket is already taken)
        const unsigned long long t = atomicAdd(st.tile_ctr, 1ull);
        if (t == (unsigned long long)gridDim.x - 1) atomicExch(st.tile_ctr, 0ull);
        s_slot[0] = (uint32_t)t;
        s_slot[1] = (uint32_t)(t >> 32);
    }
    __syncthreads();
    return (size_t)s_slot[0] | ((size_t)s_slot[1] << 32);
}

// ---------------------------------------------------------------- scan kernel
// Element (warp w, chunk v, lane l, e) of a tile is tile_base + w*NV*32*VEC + v*32*VEC +
// l*VEC + e: a warp reads 32 consecutive 16-byte vectors per chunk (coalesced), and each
// lane owns VEC consecutive elements, folded in registers before the warp-level scan.
// MODE 0: inclusive.  MODE 1: exclusive with init (out[0] = init).  MODE 2: reduction only
// (no output; the last tile stores the total in st.result).  MODE 3: reduction of init, x0, x1, ...
template <class InV, class UOp, bool HAS_UOP, class OutV, class T, class Op, int MODE, int BLOCK, int NV>
__global__ void __launch_bounds__(BLOCK) scan_kernel(InV in, UOp uop, OutV out, size_t n, Op op, T init,
                                                     LookbackState st) {
    typedef ScanSrc<InV, T, UOp, HAS_UOP> Src;
    Src src;
    src.in = in;
    src.uop = uop;
    typedef typename Src::E E;
    constexpr int VEC = Src::CONTIG ? VecWidth<E>::V : 1;
    constexpr int WARPS = BLOCK / 32;
    constexpr int TILE = BLOCK * NV * VEC;
    __shared__ uint32_t s_slot[2];
    __shared__ T s_wagg[WARPS];
    __shared__ int s_whas[WARPS];
    __shared__ T s_pre;
    __shared__ int s_pre_has;

    const size_t tile = claim_tile(st, s_slot);
    const size_t tile_base = tile * TILE;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const size_t valid = (n - tile_base) < (size_t)TILE ? (n - tile_base) : (size_t)TILE;
    const bool full = valid == (size_t)TILE;
    const uint32_t woff = warp * (NV * 32 * VEC);

    T x[NV][VEC];
    // ---- load
    bool vec_ok = false;
    if constexpr (Src::CONTIG && VEC > 1) vec_ok = full && ((((size_t)src.in._data) & 15) == 0);
    if (vec_ok) {
        if constexpr (Src::CONTIG && VEC > 1) {
            const uint4* p = reinterpret_cast<const uint4*>(src.in._data + tile_base + woff);
#pragma unroll
            for (int v = 0; v < NV; v++) {
                union { uint4 q; E e[VEC]; } u;
                u.q = p[v * 32 + lane];
#pragma unroll
                for (int e = 0; e < VEC; e++) x[v][e] = src.get(u.e[e]);
            }
        }
    } else {
#pragma unroll
        for (int v = 0; v < NV; v++)
#pragma unroll
            for (int e = 0; e < VEC; e++) {
                const size_t r = woff + v * 32 * VEC + lane * VEC + e;
                x[v][e] = (r < valid) ? src.get(src.fetch(tile_base + r)) : T();
            }
    }

    // ---- thread folds + warp scans per chunk
    T pre[NV];
    bool pre_h[NV];
    T carry = T();
    bool carry_h = false;
#pragma unroll
    for (int v = 0; v < NV; v++) {
        const long long cs = (long long)woff + v * 32 * VEC;             // chunk start in tile
        const long long ls = cs + (long long)lane * VEC;                 // lane start
        long long nvl = (long long)valid - ls;
        nvl = nvl < 0 ? 0 : (nvl > VEC ? VEC : nvl);
#pragma unroll
        for (int e = 1; e < VEC; e++)
            if (e < nvl) x[v][e] = (T)op(x[v][e - 1], x[v][e]);
        const bool lane_valid = nvl > 0;
        // last valid element of the lane (selected with constant indices: a runtime index
        // would move the whole register array to local memory)
        T inc = x[v][0];
#pragma unroll
        for (int e = 1; e < VEC; e++)
            if (e < nvl) inc = x[v][e];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T y = shfl_up_any(inc, d);
            if ((int)lane >= d && lane_valid) inc = (T)op(y, inc);
        }
        const T ex = shfl_up_any(inc, 1);
        const bool ex_h = lane > 0;
        long long last_lane = ((long long)valid - cs - 1) / VEC;
        if ((long long)valid - cs <= 0) last_lane = -1;
        if (last_lane > 31) last_lane = 31;
        const T ctot = shfl_any(inc, last_lane < 0 ? 0 : (int)last_lane);
        pre[v] = carry;
        pre_h[v] = carry_h;
        opt_combine(pre[v], pre_h[v], ex, ex_h, op);
        if (last_lane >= 0) opt_combine(carry, carry_h, ctot, true, op);
    }
    if (lane == 0) { s_wagg[warp] = carry; s_whas[warp] = carry_h ? 1 : 0; }
    __syncthreads();

    // ---- tile aggregate, look-back, prefixes
    if (warp == 0) {
        T agg = T();
        bool agg_h = false;
        if (lane == 0)
            for (int w = 0; w < WARPS; w++) opt_combine(agg, agg_h, s_wagg[w], s_whas[w] != 0, op);
        agg = shfl_any(agg, 0);
        agg_h = __shfl_sync(0xffffffffu, (int)agg_h, 0) != 0;
        T tp = T();
        bool tp_h = false;
        if (tile == 0) {
            if (MODE == 1 || MODE == 3) { tp = init; tp_h = true; }
            T incl = tp;
            bool incl_h = tp_h;
            opt_combine(incl, incl_h, agg, agg_h, op);
            if (lane == 0) {
                publish<T>(st, 0, incl, true, false);
                if (MODE >= 2 && valid == n && st.result) *reinterpret_cast<T*>(st.result) = incl;
            }
        } else {
            if (lane == 0) publish<T>(st, tile, agg, false, false);
            bool dummy;
            const Opt<T> p = lookback_prefix<T, Op, false>(st, tile, op, dummy);
            tp = p.v;
            tp_h = p.h;
            T incl = tp;
            bool incl_h = tp_h;
            opt_combine(incl, incl_h, agg, agg_h, op);
            if (lane == 0) {
                publish<T>(st, tile, incl, true, false);
                if (MODE >= 2 && tile_base + valid == n && st.result) *reinterpret_cast<T*>(st.result) = incl;
            }
        }
        if (lane == 0) { s_pre = tp; s_pre_has = tp_h ? 1 : 0; }
    }
    if constexpr (MODE < 2) {  // reductions write no elements
        __syncthreads();

        // warp prefix = tile prefix ⊕ aggregates of earlier warps
        T wp = s_pre;
        bool wp_h = s_pre_has != 0;
        for (uint32_t w = 0; w < warp; w++) opt_combine(wp, wp_h, s_wagg[w], s_whas[w] != 0, op);

        // ---- outputs
        bool st_vec = false;
        if constexpr (ViewTraits<OutV>::contiguous && VEC > 1 && sizeof(T) == sizeof(E))
            st_vec = vec_ok && ((((size_t)out._data) & 15) == 0) && out._size >= n;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            T tp = wp;
            bool tp_h = wp_h;
            opt_combine(tp, tp_h, pre[v], pre_h[v], op);
            T y[VEC];
#pragma unroll
            for (int e = 0; e < VEC; e++) {
                if (MODE == 0) {
                    y[e] = tp_h ? (T)op(tp, x[v][e]) : x[v][e];
                } else {
                    y[e] = (e == 0) ? tp : (T)op(tp, x[v][e - 1]);
                }
            }
            if constexpr (ViewTraits<OutV>::contiguous && VEC > 1 && sizeof(T) == sizeof(E)) {
                if (st_vec) {
                    union { uint4 q; T t[VEC]; } u;
#pragma unroll
                    for (int e = 0; e < VEC; e++) u.t[e] = y[e];
                    reinterpret_cast<uint4*>(out._data + tile_base + woff)[v * 32 + lane] = u.q;
                    continue;
                }
            }
#pragma unroll
            for (int e = 0; e < VEC; e++) {
                const size_t r = woff + v * 32 * VEC + lane * VEC + e;
                if (r < valid && tile_base + r < (size_t)out.size()) out[tile_base + r] = y[e];
            }
        }
    }
}

// ---------------------------------------------------------------- two-phase tile scan
// Contiguous inputs of built-in element types.  Each warp owns a contiguous segment of
// 32 * ITEMS elements of the tile, read as ROWS rows of 32 lanes x one 16-byte vector.
// Phase 1 reads the tile and reduces it (only the warp totals survive) and publishes the
// tile aggregate.  Phase 2 looks back for the tile's prefix (warp 0), reads the tile again --
// it was read moments earlier and is normally still in L2 -- and writes the scan.  CTAs are
// persistent and software-pipelined: a CTA runs phase 1 of its next tile before the look-back
// of its current one, so the look-back waits overlap HBM reads instead of idling the SM, and
// no tile data is held in registers across a wait.  HBM traffic stays 4 B read + 4 B written per 4-byte element when the
// re-read hits L2.  COMM: the operator is also commutative (the built-in Plus / Maximum /
// Minimum), so phase 1 may fold each lane's vectors before the warp combines them.
#ifndef TRTC_SCAN2_HINT
#define TRTC_SCAN2_HINT 0
#endif
// Optional L2 policies: phase-1 lines are wanted again soon (evict last), phase-2 reads and
// the output are not (evict first).  Measured slower on B200 than the plain loads and
// streaming phase-2 loads / stores (0.614 vs 0.585 ms at 2^28 i32), so off by default.
TRTC_FORCEINLINE uint4 ld_phase1(const uint4* p) {
    if (TRTC_SCAN2_HINT) return ld_l2hint(p, l2_evict_last_policy());
    return *p;
}
TRTC_FORCEINLINE uint4 ld_phase2(const uint4* p) {
    if (TRTC_SCAN2_HINT) return ld_l2hint(p, l2_evict_first_policy());
    return __ldcs(p);
}
TRTC_FORCEINLINE void st_out(uint4* p, const uint4& v) {
    if (TRTC_SCAN2_HINT) st_l2hint(p, v, l2_evict_first_policy());
    else __stcs(p, v);
}

template <class T, class Op, int MODE, int BLOCK, int ITEMS, bool COMM>
__global__ void __launch_bounds__(BLOCK) scan2_kernel(const T* __restrict__ in, T* __restrict__ out, size_t n,
                                                      size_t tiles, Op op, T init, LookbackState st) {
    constexpr int VEC = VecWidth<T>::V;
    static_assert(VEC > 1 && ITEMS % VEC == 0, "16-byte vectors of T");
    constexpr int ROWS = ITEMS / VEC;
    constexpr int WARPS = BLOCK / 32;
    constexpr int WSEG = 32 * ITEMS;
    constexpr int TILE = BLOCK * ITEMS;
    typedef union { uint4 q; T t[VEC]; } Vec;
    __shared__ unsigned long long s_ticket;
    __shared__ T s_wtot[2][WARPS];
    __shared__ int s_wh[2][WARPS];
    __shared__ T s_woff[2][WARPS];
    __shared__ int s_woh[2][WARPS];
    __shared__ T s_agg[2];
    __shared__ int s_agg_h[2];
    __shared__ T s_pre;
    __shared__ int s_pre_h;

    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const bool aligned = ((((size_t)in) | ((size_t)out)) & 15) == 0;

    // Tickets are handed out in order; every CTA takes exactly one ticket >= tiles (which
    // ends its loop), so the CTA that takes the last of the tiles + gridDim.x tickets resets
    // the counter for the next launch on this stream.
    auto claim = [&]() -> size_t {
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(st.tile_ctr, 1ull);
            if (t == (unsigned long long)tiles + gridDim.x - 1) atomicExch(st.tile_ctr, 0ull);
            s_ticket = t;
            if (st.pf_ahead) prefetch_l2_range(in, (size_t)(t + st.pf_ahead) * TILE, (size_t)TILE, n);
        }
        __syncthreads();
        return (size_t)s_ticket;
    };
    auto warp_valid = [&](size_t tile) -> uint32_t {
        const long long wv = (long long)(n - tile * (size_t)TILE) - (long long)warp * WSEG;
        return wv <= 0 ? 0u : (wv >= WSEG ? (uint32_t)WSEG : (uint32_t)wv);
    };

    // ---- phase 1: warp totals (ordered), tile aggregate, publication
    auto phase1 = [&](size_t tile, int b) {
        const uint32_t wvalid = warp_valid(tile);
        const bool fast = aligned && wvalid == (uint32_t)WSEG;
        const T* win = in + tile * (size_t)TILE + (size_t)warp * WSEG;
        T wt = T();
        bool wt_h = false;
        if (fast) {
            if constexpr (COMM) {
                Vec v[ROWS];
#pragma unroll
                for (int r = 0; r < ROWS; r++) v[r].q = ld_phase1(reinterpret_cast<const uint4*>(win) + r * 32 + lane);
                T a = v[0].t[0];
#pragma unroll
                for (int r = 0; r < ROWS; r++)
#pragma unroll
                    for (int e = 0; e < VEC; e++)
                        if (r | e) a = (T)op(a, v[r].t[e]);
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) a = (T)op(a, shfl_xor_any(a, d));
                wt = a;
            } else {
#pragma unroll
                for (int r = 0; r < ROWS; r++) {
                    Vec v;
                    v.q = ld_phase1(reinterpret_cast<const uint4*>(win) + r * 32 + lane);
                    T a = v.t[0];
#pragma unroll
                    for (int e = 1; e < VEC; e++) a = (T)op(a, v.t[e]);
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {  // ordered tree: lane l combines l and l + d
                        const T o = shfl_down_any(a, d);
                        if ((lane & (2 * d - 1)) == 0) a = (T)op(a, o);
                    }
                    a = shfl_any(a, 0);
                    wt = r ? (T)op(wt, a) : a;
                }
            }
            wt_h = true;
        } else {
            for (int r = 0; r < ROWS; r++) {
                T a = T();
                bool ah = false;
#pragma unroll
                for (int e = 0; e < VEC; e++) {
                    const uint32_t i = (uint32_t)r * 32u * VEC + lane * VEC + e;
                    if (i < wvalid) opt_combine(a, ah, win[i], true, op);
                }
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const T o = shfl_down_any(a, d);
                    const bool oh = __shfl_down_sync(0xffffffffu, (int)ah, d) != 0 && lane + d < 32;
                    if ((lane & (2 * d - 1)) == 0) opt_combine(a, ah, o, oh, op);
                }
                a = shfl_any(a, 0);
                ah = __shfl_sync(0xffffffffu, (int)ah, 0) != 0;
                opt_combine(wt, wt_h, a, ah, op);
            }
        }
        if (lane == 0) { s_wtot[b][warp] = wt; s_wh[b][warp] = wt_h ? 1 : 0; }
        __syncthreads();
        if (threadIdx.x == 0) {
            T agg = T();
            bool agg_h = false;
            for (int w = 0; w < WARPS; w++) {
                s_woff[b][w] = agg;
                s_woh[b][w] = agg_h ? 1 : 0;
                opt_combine(agg, agg_h, s_wtot[b][w], s_wh[b][w] != 0, op);
            }
            s_agg[b] = agg;
            s_agg_h[b] = agg_h ? 1 : 0;
            if (tile == 0) {
                T incl = init;
                bool incl_h = MODE == 1;
                if (!incl_h) incl = T();
                opt_combine(incl, incl_h, agg, agg_h, op);
                publish<T>(st, 0, incl, true, false);
            } else {
                if (!TRTC_FAULT_SKIP_PUBLISH(tile)) publish<T>(st, tile, agg, false, false);
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
        // look-back of the current tile (warp 0)
        if (warp == 0) {
            T tp = T();
            bool tp_h = false;
            if (cur == 0) {
                if (MODE == 1) { tp = init; tp_h = true; }
            } else {
                bool dummy;
                const Opt<T> p = lookback_prefix<T, Op, false>(st, cur, op, dummy);
                tp = p.v;
                tp_h = p.h;
                T incl = tp;
                bool incl_h = tp_h;
                opt_combine(incl, incl_h, s_agg[buf], s_agg_h[buf] != 0, op);
                if (lane == 0 && !TRTC_FAULT_SKIP_PUBLISH(cur)) publish<T>(st, cur, incl, true, false);
            }
            if (lane == 0) { s_pre = tp; s_pre_h = tp_h ? 1 : 0; }
        }
        __syncthreads();
        // re-read and write the current tile
        {
            const uint32_t wvalid = warp_valid(cur);
            const bool fast = aligned && wvalid == (uint32_t)WSEG;
            const T* win = in + cur * (size_t)TILE + (size_t)warp * WSEG;
            T* wout = out + cur * (size_t)TILE + (size_t)warp * WSEG;
            T carry = s_pre;
            bool carry_h = s_pre_h != 0;
            opt_combine(carry, carry_h, s_woff[buf][warp], s_woh[buf][warp] != 0, op);
            if (fast) {
                Vec v2[ROWS];
#pragma unroll
                for (int r = 0; r < ROWS; r++) v2[r].q = ld_phase2(reinterpret_cast<const uint4*>(win) + r * 32 + lane);
#pragma unroll
                for (int r = 0; r < ROWS; r++) {
                    T xi[VEC];  // inclusive within the lane's vector
                    xi[0] = v2[r].t[0];
#pragma unroll
                    for (int e = 1; e < VEC; e++) xi[e] = (T)op(xi[e - 1], v2[r].t[e]);
                    T incl = xi[VEC - 1];
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const T y = shfl_up_any(incl, d);
                        if (lane >= (uint32_t)d) incl = (T)op(y, incl);
                    }
                    const T ex = shfl_up_any(incl, 1);
                    const T row_tot = shfl_any(incl, 31);
                    // base = carry ⊕ (lanes before this one)
                    T base = ex;
                    bool base_h = lane > 0;
                    if (carry_h) { base = lane > 0 ? (T)op(carry, ex) : carry; base_h = true; }
                    Vec o;
#pragma unroll
                    for (int e = 0; e < VEC; e++) {
                        if (MODE == 0) o.t[e] = base_h ? (T)op(base, xi[e]) : xi[e];
                        else o.t[e] = (e == 0) ? base : (T)op(base, xi[e - 1]);
                    }
                    st_out(reinterpret_cast<uint4*>(wout) + r * 32 + lane, o.q);
                    carry = carry_h ? (T)op(carry, row_tot) : row_tot;
                    carry_h = true;
                }
            } else {
                for (int r = 0; r < ROWS; r++) {
                    const uint32_t i0 = (uint32_t)r * 32u * VEC + lane * VEC;
                    T xi[VEC];
                    T run = T();
                    bool run_h = false;
#pragma unroll
                    for (int e = 0; e < VEC; e++) {
                        if (i0 + e < wvalid) opt_combine(run, run_h, win[i0 + e], true, op);
                        xi[e] = run;
                    }
                    T incl = run;
                    bool incl_h = run_h;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const T y = shfl_up_any(incl, d);
                        const bool yh = __shfl_up_sync(0xffffffffu, (int)incl_h, d) != 0;
                        if (lane >= (uint32_t)d && yh) { incl = incl_h ? (T)op(y, incl) : y; incl_h = true; }
                    }
                    const T ex = shfl_up_any(incl, 1);
                    const bool ex_h = __shfl_up_sync(0xffffffffu, (int)incl_h, 1) != 0 && lane > 0;
                    const T row_tot = shfl_any(incl, 31);
                    const bool row_h = __shfl_sync(0xffffffffu, (int)incl_h, 31) != 0;
                    T base = carry;
                    bool base_h = carry_h;
                    opt_combine(base, base_h, ex, ex_h, op);
#pragma unroll
                    for (int e = 0; e < VEC; e++) {
                        if (i0 + e >= wvalid) continue;
                        T y;
                        if (MODE == 0) y = base_h ? (T)op(base, xi[e]) : xi[e];
                        else if (e == 0) y = base;
                        else y = base_h ? (T)op(base, xi[e - 1]) : xi[e - 1];
                        wout[i0 + e] = y;
                    }
                    opt_combine(carry, carry_h, row_tot, row_h, op);
                }
            }
        }
        if (nxt >= tiles) break;
        cur = nxt;
        buf ^= 1;
    }
}

// ---------------------------------------------------------------- segmented scan kernel
// Segments continue at i while pred(key[i-1], key[i]) (default EqualTo; a head starts a new
// segment).  MODE 0: inclusive.  MODE 1: exclusive, out[head] = init, otherwise
// init ⊕ (segment values before i).  Keys and values are read through their views.
template <class KV, class InV, class OutV, class T, class Pred, class Op, int MODE, int BLOCK, int NV>
__global__ void __launch_bounds__(BLOCK) scan_by_key_kernel(KV keys, InV vals, OutV out, size_t n, Pred pred, Op op,
                                                           T init, LookbackState st) {
    typedef ScanSrc<InV, T, Nothing, false> Src;
    Src src;
    src.in = vals;
    typedef typename Src::E E;
    typedef typename remove_cvref<typename KV::value_t>::type K;
    constexpr bool CONTIG = Src::CONTIG && ViewTraits<KV>::contiguous && VecWidth<E>::V > 1 && VecWidth<K>::V > 1;
    // lane chunk width: 16 bytes of the narrower type (the wider one takes several vectors)
    constexpr int VEC = CONTIG ? (VecWidth<E>::V > VecWidth<K>::V ? VecWidth<E>::V : VecWidth<K>::V) : 1;
    constexpr int WARPS = BLOCK / 32;
    constexpr int TILE = BLOCK * NV * VEC;
    __shared__ uint32_t s_slot[2];
    __shared__ T s_wagg[WARPS];
    __shared__ int s_whas[WARPS], s_whd[WARPS];
    __shared__ T s_pre;
    __shared__ int s_pre_has, s_pre_hd;

    const size_t tile = claim_tile(st, s_slot);
    const size_t tile_base = tile * TILE;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const size_t valid = (n - tile_base) < (size_t)TILE ? (n - tile_base) : (size_t)TILE;
    const bool full = valid == (size_t)TILE;
    const uint32_t woff = warp * (NV * 32 * VEC);

    T x[NV][VEC];
    K k[NV][VEC];
    bool vec_ok = false;
    if constexpr (CONTIG && VEC > 1)
        vec_ok = full && ((((size_t)src.in._data) & 15) == 0) && ((((size_t)keys._data) & 15) == 0);
    if (vec_ok) {
        if constexpr (CONTIG && VEC > 1) {
            constexpr int KV4 = VEC * (int)sizeof(K) / 16;  // 16-byte vectors of keys per chunk-lane
            constexpr int EV4 = VEC * (int)sizeof(E) / 16;
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const size_t r0 = tile_base + woff + v * 32 * VEC + lane * VEC;
                union { uint4 q[KV4 > 0 ? KV4 : 1]; K e[VEC]; } uk;
                union { uint4 q[EV4 > 0 ? EV4 : 1]; E e[VEC]; } ue;
#pragma unroll
                for (int q = 0; q < KV4; q++) uk.q[q] = reinterpret_cast<const uint4*>(keys._data + r0)[q];
#pragma unroll
                for (int q = 0; q < EV4; q++) ue.q[q] = reinterpret_cast<const uint4*>(src.in._data + r0)[q];
#pragma unroll
                for (int e = 0; e < VEC; e++) { k[v][e] = uk.e[e]; x[v][e] = src.get(ue.e[e]); }
            }
        }
    } else {
#pragma unroll
        for (int v = 0; v < NV; v++)
#pragma unroll
            for (int e = 0; e < VEC; e++) {
                const size_t r = woff + v * 32 * VEC + lane * VEC + e;
                if (r < valid) { k[v][e] = keys[tile_base + r]; x[v][e] = src.get(src.fetch(tile_base + r)); }
                else { k[v][e] = K(); x[v][e] = T(); }
            }
    }

    // heads: compare with the previous element's key
    bool h[NV][VEC];
    K carry_key = K();
#pragma unroll
    for (int v = 0; v < NV; v++) {
        const size_t ls = woff + v * 32 * VEC + lane * VEC;
        K prev = shfl_up_any(k[v][VEC - 1], 1);
        const K last31 = shfl_any(k[v][VEC - 1], 31);
        if (lane == 0) {
            if (v > 0) prev = carry_key;
            else if (tile_base + ls > 0 && tile_base + ls - 1 < n) prev = keys[tile_base + ls - 1];
        }
        carry_key = last31;
#pragma unroll
        for (int e = 0; e < VEC; e++) {
            const size_t gi = tile_base + ls + e;
            const K pk = e == 0 ? prev : k[v][e - 1];
            h[v][e] = (gi == 0) || !pred(pk, k[v][e]);
        }
    }

    // thread folds + segmented warp scans
    T pre[NV];
    bool pre_h[NV], pre_hd[NV];
    T xin[NV][VEC];  // inclusive value of each element within its thread chunk
    T carry = T();
    bool carry_h = false, carry_hd = false;
#pragma unroll
    for (int v = 0; v < NV; v++) {
        const long long cs = (long long)woff + v * 32 * VEC;
        const long long ls = cs + (long long)lane * VEC;
        long long nvl = (long long)valid - ls;
        nvl = nvl < 0 ? 0 : (nvl > VEC ? VEC : nvl);
        bool thd = h[v][0];
        xin[v][0] = x[v][0];
#pragma unroll
        for (int e = 1; e < VEC; e++) {
            xin[v][e] = (e < nvl && !h[v][e]) ? (T)op(xin[v][e - 1], x[v][e]) : x[v][e];
            if (e < nvl) thd = thd || h[v][e];
        }
        const bool lane_valid = nvl > 0;
        T inc = xin[v][0];
#pragma unroll
        for (int e = 1; e < VEC; e++)
            if (e < nvl) inc = xin[v][e];
        bool ihd = thd;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T y = shfl_up_any(inc, d);
            const int yhd = __shfl_up_sync(0xffffffffu, (int)ihd, d);
            if ((int)lane >= d && lane_valid) {
                if (!ihd) inc = (T)op(y, inc);
                ihd = ihd || yhd;
            }
        }
        const T ex = shfl_up_any(inc, 1);
        const int exhd = __shfl_up_sync(0xffffffffu, (int)ihd, 1);
        long long last_lane = ((long long)valid - cs - 1) / VEC;
        if ((long long)valid - cs <= 0) last_lane = -1;
        if (last_lane > 31) last_lane = 31;
        const int ll = last_lane < 0 ? 0 : (int)last_lane;
        const T ctot = shfl_any(inc, ll);
        const int ctothd = __shfl_sync(0xffffffffu, (int)ihd, ll);
        // thread prefix = carry ⊕seg ex
        pre[v] = carry; pre_h[v] = carry_h; pre_hd[v] = carry_hd;
        if (lane > 0) {
            if (!pre_h[v] || exhd) { pre[v] = ex; pre_hd[v] = exhd || (pre_h[v] && pre_hd[v]); }
            else { pre[v] = (T)op(pre[v], ex); }
            pre_h[v] = true;
        }
        if (last_lane >= 0) {
            if (!carry_h || ctothd) { carry = ctot; carry_hd = ctothd || (carry_h && carry_hd); }
            else carry = (T)op(carry, ctot);
            carry_h = true;
        }
    }
    if (lane == 0) { s_wagg[warp] = carry; s_whas[warp] = carry_h ? 1 : 0; s_whd[warp] = carry_hd ? 1 : 0; }
    __syncthreads();

    if (warp == 0) {
        T agg = T();
        bool agg_h = false, agg_hd = false;
        if (lane == 0)
            for (int w = 0; w < WARPS; w++) {
                if (!s_whas[w]) continue;
                if (!agg_h || s_whd[w]) { agg = s_wagg[w]; agg_hd = s_whd[w] || (agg_h && agg_hd); }
                else agg = (T)op(agg, s_wagg[w]);
                agg_h = true;
            }
        agg = shfl_any(agg, 0);
        agg_h = __shfl_sync(0xffffffffu, (int)agg_h, 0) != 0;
        agg_hd = __shfl_sync(0xffffffffu, (int)agg_hd, 0) != 0;
        T tp = T();
        bool tp_h = false, tp_hd = false;
        if (tile > 0) {
            if (lane == 0) publish<T>(st, tile, agg, false, agg_hd);
            const Opt<T> p = lookback_prefix<T, Op, true>(st, tile, op, tp_hd);
            tp = p.v;
            tp_h = p.h;
        }
        // inclusive of this tile = tp ⊕seg agg
        T incl = tp;
        bool incl_hd = tp_hd;
        if (!tp_h || agg_hd) { incl = agg; incl_hd = agg_hd || (tp_h && tp_hd); }
        else incl = (T)op(tp, agg);
        if (lane == 0) {
            publish<T>(st, tile, incl, true, incl_hd);
            s_pre = tp; s_pre_has = tp_h ? 1 : 0; s_pre_hd = tp_hd ? 1 : 0;
        }
    }
    __syncthreads();

    T wp = s_pre;
    bool wp_h = s_pre_has != 0;
    for (uint32_t w = 0; w < warp; w++) {
        if (!s_whas[w]) continue;
        if (!wp_h || s_whd[w]) wp = s_wagg[w];
        else wp = (T)op(wp, s_wagg[w]);
        wp_h = true;
    }
#pragma unroll
    for (int v = 0; v < NV; v++) {
        // thread prefix (running inclusive value of the element before this lane's first)
        T tp = wp;
        bool tp_h = wp_h;
        if (pre_h[v]) {
            if (!tp_h || pre_hd[v]) tp = pre[v];
            else tp = (T)op(tp, pre[v]);
            tp_h = true;
        }
        T run = tp;  // inclusive value of the previous element
#pragma unroll
        for (int e = 0; e < VEC; e++) {
            const size_t r = woff + v * 32 * VEC + lane * VEC + e;
            T cur;  // inclusive value of this element
            if (h[v][e]) cur = x[v][e];
            else if (e == 0) cur = tp_h ? (T)op(tp, x[v][e]) : x[v][e];
            else cur = (T)op(run, x[v][e]);
            T y;
            if (MODE == 0) y = cur;
            else y = h[v][e] ? init : (T)op(init, run);
            run = cur;
            if (r < valid && tile_base + r < (size_t)out.size()) out[tile_base + r] = y;
        }
    }
}

// ---------------------------------------------------------------- two-phase segmented scan
// scan_by_key for contiguous keys and values of one element size (4 or 8 bytes) under the
// built-in EqualTo / Plus, in the persistent software-pipelined form of scan2_kernel:
// phase 1 reads a tile (16-byte loads of keys and values) and publishes its segmented
// aggregate -- the sum after its last segment head, with a head flag -- phase 2 looks back
// (segmented: the walk stops at the first tile holding a head), re-reads the tile (normally
// from L2) and writes it.  No tile data is held in registers across a wait.  A full warp
// segment of aligned arrays is scanned in blocked order (each lane ITEMS consecutive
// elements, re-laid out through shared memory); the rest of the last tile, and every element
// of unaligned arrays, is scanned row by row with scalar loads; elements past n count as
// heads of value T() and are not stored, so they never reach a valid output.
#ifndef TRTC_SBK2_AHEAD
#define TRTC_SBK2_AHEAD 0  // draw the next tile's ticket during the look-back instead of after
#endif
#ifndef TRTC_SBK2_MINB  // resident CTAs per SM the kernel is compiled for (48 registers at 5)
#define TRTC_SBK2_MINB(bytes) ((bytes) == 8 ? 4 : 5)
#endif
// full aligned warp segments are re-laid out through shared memory so that each lane holds
// ITEMS consecutive elements: one warp-wide segmented scan per segment instead of one per
// 16-byte row
#ifndef TRTC_SBK2_BLOCKED
#define TRTC_SBK2_BLOCKED 1
#endif
template <class K, class T, int MODE, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK, TRTC_SBK2_MINB(sizeof(T))) sbk2_kernel(const K* __restrict__ keys, const T* vals, T* out,
                                                                     size_t n, size_t tiles, T init, LookbackState st) {
    static_assert(sizeof(K) == sizeof(T) && (sizeof(T) == 4 || sizeof(T) == 8), "keys and values of one width");
    constexpr int VEC = VecWidth<T>::V;
    static_assert(ITEMS % VEC == 0, "whole 16-byte vectors per lane");
    constexpr int ROWS = ITEMS / VEC;
    constexpr int WARPS = BLOCK / 32;
    constexpr int WSEG = 32 * ITEMS;
    constexpr int TILE = BLOCK * ITEMS;
    typedef union { uint4 q; T t[VEC]; } VecT;
    typedef union { uint4 q; K k[VEC]; } VecK;
    __shared__ unsigned long long s_ticket;
    __shared__ T s_wtot[2][WARPS];
    __shared__ int s_whd[2][WARPS];
    __shared__ T s_woff[2][WARPS];
    __shared__ int s_woh[2][WARPS], s_wohd[2][WARPS];
    __shared__ T s_agg[2];
    __shared__ int s_agg_hd[2];
    __shared__ T s_pre;
    __shared__ int s_pre_h;
    constexpr int SB = TRTC_SBK2_BLOCKED ? WARPS * WSEG : VEC;
    __shared__ __align__(16) K s_bk[SB];  // per-warp staging of the blocked re-layout
    __shared__ __align__(16) T s_bv[SB];
    Plus op;
    EqualTo eq;

    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const bool aligned = ((((size_t)keys) | ((size_t)vals) | ((size_t)out)) & 15) == 0;

    auto claim = [&]() -> size_t {
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(st.tile_ctr, 1ull);
            if (t == (unsigned long long)tiles + gridDim.x - 1) atomicExch(st.tile_ctr, 0ull);
            s_ticket = t;
            if (st.pf_ahead) {
                prefetch_l2_range(keys, (size_t)(t + st.pf_ahead) * TILE, (size_t)TILE, n);
                prefetch_l2_range(vals, (size_t)(t + st.pf_ahead) * TILE, (size_t)TILE, n);
            }
        }
        __syncthreads();
        return (size_t)s_ticket;
    };
    // fast rows are loaded up front (all 16-byte loads of the warp segment in flight at once)
    auto preload = [&](size_t wstart, bool phase2, VecK (&kq)[ROWS], VecT (&vq)[ROWS]) {
#pragma unroll
        for (int r = 0; r < ROWS; r++) {
            const size_t i0 = wstart + (size_t)r * 32 * VEC + (size_t)lane * VEC;
            kq[r].q = reinterpret_cast<const uint4*>(keys + i0)[0];
            vq[r].q = phase2 ? __ldcs(reinterpret_cast<const uint4*>(vals + i0)) : reinterpret_cast<const uint4*>(vals + i0)[0];
        }
    };
    // one row of the warp's segment: lane l holds elements wstart + r*32*VEC + l*VEC + e;
    // hd[e]: element e starts a segment; prevk_row: key before the row's first element
    auto load_row = [&](size_t wstart, int r, bool fast, K prevk_row, const VecK& kq, const VecT& vq, K (&k)[VEC],
                        T (&x)[VEC], bool (&hd)[VEC]) {
        const size_t i0 = wstart + (size_t)r * 32 * VEC + (size_t)lane * VEC;
        if (fast) {
#pragma unroll
            for (int e = 0; e < VEC; e++) { k[e] = kq.k[e]; x[e] = vq.t[e]; }
        } else {
#pragma unroll
            for (int e = 0; e < VEC; e++) {
                const bool ok = i0 + e < n;
                k[e] = ok ? keys[i0 + e] : K();
                x[e] = ok ? vals[i0 + e] : T();
            }
        }
        K pk = shfl_up_any(k[VEC - 1], 1);
        if (lane == 0) pk = prevk_row;
#pragma unroll
        for (int e = 0; e < VEC; e++) {
            const K before = e == 0 ? pk : k[e - 1];
            hd[e] = !(bool)eq(before, k[e]);
            if (!fast) hd[e] = hd[e] || i0 + e >= n;
        }
        if (i0 == 0) hd[0] = true;
    };
    auto first_key = [&](size_t wstart) -> K { return wstart > 0 && wstart - 1 < n ? keys[wstart - 1] : K(); };
    // a full aligned warp segment in blocked order: lane l receives elements
    // wstart + l*ITEMS .. + ITEMS-1 (16-byte row loads, staged in shared memory: row r, lane l
    // writes 16-byte slot r*32+l; lane l reads slots l*ROWS .. l*ROWS+ROWS-1).  Returns the
    // lane's head mask (bit j: element j starts a segment).
    auto load_blocked = [&](size_t wstart, bool phase2, K (&k)[ITEMS], T (&x)[ITEMS]) -> uint32_t {
        static_assert(ITEMS <= 32, "head mask");
        VecK kq[ROWS];
        VecT vq[ROWS];
        preload(wstart, phase2, kq, vq);
        uint4* sk4 = reinterpret_cast<uint4*>(s_bk + warp * WSEG);
        uint4* sv4 = reinterpret_cast<uint4*>(s_bv + warp * WSEG);
#pragma unroll
        for (int r = 0; r < ROWS; r++) {
            sk4[r * 32 + lane] = kq[r].q;
            sv4[r * 32 + lane] = vq[r].q;
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < ROWS; q++) {
            VecK a;
            VecT b;
            a.q = sk4[lane * ROWS + q];
            b.q = sv4[lane * ROWS + q];
#pragma unroll
            for (int e = 0; e < VEC; e++) {
                k[q * VEC + e] = a.k[e];
                x[q * VEC + e] = b.t[e];
            }
        }
        K pk = shfl_up_any(k[ITEMS - 1], 1);
        if (lane == 0) pk = first_key(wstart);
        uint32_t hd = 0;
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            const K before = j == 0 ? pk : k[j - 1];
            if (!(bool)eq(before, k[j])) hd |= 1u << j;
        }
        if (wstart == 0 && lane == 0) hd |= 1u;
        return hd;
    };
    // the lane's value after its last head (all its elements when it holds none)
    auto lane_fold = [&](const T (&x)[ITEMS], uint32_t hd) -> T {
        T a = x[0];
#pragma unroll
        for (int j = 1; j < ITEMS; j++) a = ((hd >> j) & 1u) ? x[j] : (T)op(a, x[j]);
        return a;
    };

    // ---- phase 1: segmented warp aggregates (ordered), tile aggregate, publication
    auto phase1 = [&](size_t tile, int b) {
        const size_t wstart = tile * (size_t)TILE + (size_t)warp * WSEG;
        const bool fast = aligned && wstart + WSEG <= n;
        T wt = T();
        bool wt_h = false, wt_hd = false;
        if (TRTC_SBK2_BLOCKED && fast) {
            K k[ITEMS];
            T x[ITEMS];
            const uint32_t hd = load_blocked(wstart, false, k, x);
            T a = lane_fold(x, hd);
            // the segment's value after its last head: lanes from the last lane holding a head
            // (lane 0 when none) summed by a butterfly
            const uint32_t hm = __ballot_sync(0xffffffffu, hd != 0u);
            const uint32_t last = hm ? 31u - __clz(hm) : 0u;
            a = lane >= last ? a : T();
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) a = (T)op(a, shfl_xor_any(a, d));
            wt = a;
            wt_hd = hm != 0u;
        } else {
            K prevk = first_key(wstart);
            VecK kq[ROWS];
            VecT vq[ROWS];
            if (fast) preload(wstart, false, kq, vq);
#pragma unroll
            for (int r = 0; r < ROWS; r++) {
                K k[VEC];
                T x[VEC];
                bool hd[VEC];
                load_row(wstart, r, fast, prevk, kq[r], vq[r], k, x, hd);
                prevk = shfl_any(k[VEC - 1], 31);
                // lane fold (value after the lane's last head)
                T a = x[0];
                bool ahd = hd[0];
#pragma unroll
                for (int e = 1; e < VEC; e++) {
                    if (hd[e]) { a = x[e]; ahd = true; }
                    else a = (T)op(a, x[e]);
                }
                // the row's value after its last head: the lanes from the last lane holding a
                // head (lane 0 when none) summed by a butterfly (Plus, T() its identity)
                const uint32_t hm = __ballot_sync(0xffffffffu, ahd);
                const uint32_t last = hm ? 31u - __clz(hm) : 0u;
                a = lane >= last ? a : T();
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) a = (T)op(a, shfl_xor_any(a, d));
                ahd = hm != 0;
                if (!wt_h || ahd) wt = a;
                else wt = (T)op(wt, a);
                wt_h = true;
                wt_hd = wt_hd || ahd;
            }
        }
        if (lane == 0) { s_wtot[b][warp] = wt; s_whd[b][warp] = wt_hd ? 1 : 0; }
        __syncthreads();
        if (threadIdx.x == 0) {
            T agg = T();
            bool agg_h = false, agg_hd = false;
            for (int w = 0; w < WARPS; w++) {
                s_woff[b][w] = agg;
                s_woh[b][w] = agg_h ? 1 : 0;
                s_wohd[b][w] = agg_hd ? 1 : 0;
                const bool whd = s_whd[b][w] != 0;
                agg = (!agg_h || whd) ? s_wtot[b][w] : (T)op(agg, s_wtot[b][w]);
                agg_h = true;
                agg_hd = agg_hd || whd;
            }
            s_agg[b] = agg;
            s_agg_hd[b] = agg_hd ? 1 : 0;
            publish<T>(st, tile, agg, tile == 0, agg_hd);
        }
    };

    size_t cur = claim();
    if (cur >= tiles) return;
    int buf = 0;
    phase1(cur, 0);
#if TRTC_SBK2_AHEAD
    // the ticket after next is drawn by thread 0 during the look-back (its latency then hides
    // behind the look-back's) and read after the barrier that follows it; a CTA stops drawing
    // once it holds a ticket >= tiles, so each CTA still takes exactly one such ticket
    size_t nxt = claim();
#endif
    while (true) {
#if !TRTC_SBK2_AHEAD
        const size_t nxt = claim();
#endif
        if (nxt < tiles) phase1(nxt, buf ^ 1);
        // segmented look-back of the current tile (warp 0): the running segment value entering it
        if (warp == 0) {
            T tp = T();
            bool tp_h = false;
            if (cur > 0) {
                bool tp_hd = false;
                const Opt<T> p = lookback_prefix<T, Plus, true>(st, cur, op, tp_hd);
                tp = p.v;
                tp_h = p.h;
                T incl = tp;
                if (s_agg_hd[buf] || !tp_h) incl = s_agg[buf];
                else incl = (T)op(tp, s_agg[buf]);
                if (lane == 0) publish<T>(st, cur, incl, true, tp_hd || s_agg_hd[buf] != 0);
            }
            if (lane == 0) { s_pre = tp; s_pre_h = tp_h ? 1 : 0; }
#if TRTC_SBK2_AHEAD
            if (lane == 0) {
                unsigned long long t = ~0ull;
                if (nxt < tiles) {
                    t = atomicAdd(st.tile_ctr, 1ull);
                    if (t == (unsigned long long)tiles + gridDim.x - 1) atomicExch(st.tile_ctr, 0ull);
                }
                s_ticket = t;
            }
#endif
        }
        __syncthreads();
#if TRTC_SBK2_AHEAD
        const size_t nxt2 = (size_t)s_ticket;
#endif
        // re-read and write the current tile
        {
            const size_t wstart = cur * (size_t)TILE + (size_t)warp * WSEG;
            const bool fast = aligned && wstart + WSEG <= n;
            // carry into the warp = tile prefix, then the tile's earlier warps (segmented)
            T carry = s_pre;
            bool carry_h = s_pre_h != 0;
            if (s_woh[buf][warp]) {
                if (s_wohd[buf][warp] || !carry_h) carry = s_woff[buf][warp];
                else carry = (T)op(carry, s_woff[buf][warp]);
                carry_h = true;
            }
            if (TRTC_SBK2_BLOCKED && fast) {
                K k[ITEMS];
                T x[ITEMS];
                const uint32_t hd = load_blocked(wstart, true, k, x);
                const T a = lane_fold(x, hd);
                // inclusive segmented scan over the lanes (as in the row form below)
                const uint32_t hm = __ballot_sync(0xffffffffu, hd != 0u);
                const uint32_t le = lane == 31u ? 0xffffffffu : ((2u << lane) - 1u);  // lanes <= l
                T inc = a;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const T y = shfl_up_any(inc, d);
                    if (lane >= (uint32_t)d) {
                        const uint32_t win = le & ~((1u << (lane - (uint32_t)d + 1u)) - 1u);
                        if ((hm & win) == 0u) inc = (T)op(y, inc);
                    }
                }
                const T ex = shfl_up_any(inc, 1);
                const bool exhd = (hm & (le >> 1)) != 0u;  // a head in lanes < l
                T run = carry;
                bool run_h = carry_h;
                if (lane > 0) {
                    run = (exhd || !run_h) ? ex : (T)op(run, ex);
                    run_h = true;
                }
#pragma unroll
                for (int j = 0; j < ITEMS; j++) {
                    const bool h = (hd >> j) & 1u;
                    const T c = h ? x[j] : (run_h ? (T)op(run, x[j]) : x[j]);
                    const T y = MODE == 0 ? c : (h ? init : (T)op(init, run));
                    x[j] = y;
                    run = c;
                    run_h = true;
                }
                // back to rows through the lane's own staging slots, then 16-byte stores
                uint4* sv4 = reinterpret_cast<uint4*>(s_bv + warp * WSEG);
#pragma unroll
                for (int q = 0; q < ROWS; q++) {
                    VecT o;
#pragma unroll
                    for (int e = 0; e < VEC; e++) o.t[e] = x[q * VEC + e];
                    sv4[lane * ROWS + q] = o.q;
                }
                __syncwarp();
#pragma unroll
                for (int r = 0; r < ROWS; r++)
                    __stcs(reinterpret_cast<uint4*>(out + wstart + (size_t)(r * 32 + (int)lane) * VEC), sv4[r * 32 + lane]);
            } else {
                K prevk = first_key(wstart);
                VecK kq[ROWS];
                VecT vq[ROWS];
                if (fast) preload(wstart, true, kq, vq);
#pragma unroll
                for (int r = 0; r < ROWS; r++) {
                    K k[VEC];
                    T x[VEC];
                    bool hd[VEC];
                    load_row(wstart, r, fast, prevk, kq[r], vq[r], k, x, hd);
                    prevk = shfl_any(k[VEC - 1], 31);
                    T a = x[0];
                    bool ahd = hd[0];
#pragma unroll
                    for (int e = 1; e < VEC; e++) {
                        if (hd[e]) { a = x[e]; ahd = true; }
                        else a = (T)op(a, x[e]);
                    }
                    // inclusive segmented scan over the lanes: at distance d, lane l holds lanes
                    // (l-d, l] and takes in (l-2d, l-d] only if no lane of its window holds a head
                    const uint32_t hm = __ballot_sync(0xffffffffu, ahd);
                    const uint32_t le = lane == 31u ? 0xffffffffu : ((2u << lane) - 1u);  // lanes <= l
                    T inc = a;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const T y = shfl_up_any(inc, d);
                        if (lane >= (uint32_t)d) {
                            const uint32_t win = le & ~((1u << (lane - (uint32_t)d + 1u)) - 1u);
                            if ((hm & win) == 0u) inc = (T)op(y, inc);
                        }
                    }
                    const T ex = shfl_up_any(inc, 1);
                    const bool exhd = (hm & (le >> 1)) != 0u;  // a head in lanes < l
                    const T row_tot = shfl_any(inc, 31);
                    const bool row_hd = hm != 0u;
                    // running value entering this lane's first element
                    T run = carry;
                    bool run_h = carry_h;
                    if (lane > 0) {
                        run = (exhd || !run_h) ? ex : (T)op(run, ex);
                        run_h = true;
                    }
                    T y[VEC];
#pragma unroll
                    for (int e = 0; e < VEC; e++) {
                        const T c = hd[e] ? x[e] : (run_h ? (T)op(run, x[e]) : x[e]);
                        if (MODE == 0) y[e] = c;
                        else y[e] = hd[e] ? init : (T)op(init, run);
                        run = c;
                        run_h = true;
                    }
                    const size_t i0 = wstart + (size_t)r * 32 * VEC + (size_t)lane * VEC;
                    if (fast) {
                        VecT o;
#pragma unroll
                        for (int e = 0; e < VEC; e++) o.t[e] = y[e];
                        __stcs(reinterpret_cast<uint4*>(out + i0), o.q);
                    } else {
#pragma unroll
                        for (int e = 0; e < VEC; e++)
                            if (i0 + e < n) out[i0 + e] = y[e];
                    }
                    carry = (row_hd || !carry_h) ? row_tot : (T)op(carry, row_tot);
                    carry_h = true;
                }
            }
        }
        if (nxt >= tiles) break;
        cur = nxt;
#if TRTC_SBK2_AHEAD
        nxt = nxt2;
#endif
        buf ^= 1;
    }
}

// ---------------------------------------------------------------- commutative reduce
// independent 16-byte loads in flight per thread (B200, 2^28 f32 per launch: 0.1851-0.1855 /
// 0.1824-0.1833 / 0.1828 / 0.1817 ms at 4 / 8 / 12 / 16; 34-52 registers, no spills)
#ifndef TRTC_REDUCE_UNROLL
#define TRTC_REDUCE_UNROLL 16
#endif
// Built-in commutative operators over contiguous input: 16-byte loads, VEC independent
// per-thread accumulators (shorter FP accumulation chains), warp/block trees, one partial
// per CTA, and the last CTA to finish folds the partials (no second launch).
template <class E, class T, class Op, class UOp, bool HAS_UOP, int BLOCK>
__global__ void __launch_bounds__(BLOCK) reduce_kernel(const E* __restrict__ in, size_t n, Op op, UOp uop, T* partials,
                                                       int* partial_has, uint32_t* done_ctr, T* result, int has_init,
                                                       T init) {
    constexpr int VEC = VecWidth<E>::V;
    constexpr int WARPS = BLOCK / 32;
    __shared__ T s_w[WARPS];
    __shared__ int s_wh[WARPS];
    __shared__ bool s_last;
    auto get = [&](const E& e) -> T {
        if constexpr (HAS_UOP) return (T)uop(e);
        else return (T)e;
    };
    T acc[VEC];
    bool acc_h = false;
    const bool aligned = ((((size_t)in) & 15) == 0);
    const size_t nvec = aligned ? n / VEC : 0;
    const size_t gtid = (size_t)blockIdx.x * BLOCK + threadIdx.x, gsz = (size_t)gridDim.x * BLOCK;
    size_t vi = gtid;
    if (vi < nvec) {
        union { uint4 q; E e[VEC]; } u;
        u.q = reinterpret_cast<const uint4*>(in)[vi];
#pragma unroll
        for (int e = 0; e < VEC; e++) acc[e] = get(u.e[e]);
        acc_h = true;
        // U independent 16-byte loads in flight per thread
        constexpr int U = TRTC_REDUCE_UNROLL;
        for (vi += gsz; vi + (U - 1) * gsz < nvec; vi += U * gsz) {
            union { uint4 q; E e[VEC]; } w[U];
#pragma unroll
            for (int r = 0; r < U; r++) w[r].q = reinterpret_cast<const uint4*>(in)[vi + r * gsz];
#pragma unroll
            for (int r = 0; r < U; r++)
#pragma unroll
                for (int e = 0; e < VEC; e++) acc[e] = (T)op(acc[e], get(w[r].e[e]));
        }
        for (; vi < nvec; vi += gsz) {
            u.q = reinterpret_cast<const uint4*>(in)[vi];
#pragma unroll
            for (int e = 0; e < VEC; e++) acc[e] = (T)op(acc[e], get(u.e[e]));
        }
    }
    T a = acc[0];
    if (acc_h) {
#pragma unroll
        for (int e = 1; e < VEC; e++) a = (T)op(a, acc[e]);
    }
    for (size_t i = nvec * VEC + gtid; i < n; i += gsz) {
        const T t = get(in[i]);
        a = acc_h ? (T)op(a, t) : t;
        acc_h = true;
    }
    // warp tree
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const T o = shfl_down_any(a, d);
        const int oh = __shfl_down_sync(0xffffffffu, (int)acc_h, d);
        if ((int)lane_id() + d < 32 && oh) { a = acc_h ? (T)op(a, o) : o; acc_h = true; }
    }
    const uint32_t warp = threadIdx.x >> 5;
    if (lane_id() == 0) { s_w[warp] = a; s_wh[warp] = acc_h ? 1 : 0; }
    __syncthreads();
    if (threadIdx.x == 0) {
        T b = T();
        bool bh = false;
        for (int w = 0; w < WARPS; w++) opt_combine(b, bh, s_w[w], s_wh[w] != 0, op);
        partials[blockIdx.x] = b;
        partial_has[blockIdx.x] = bh ? 1 : 0;
        __threadfence();
        const uint32_t prev = atomicAdd(done_ctr, 1u);
        s_last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    // the last CTA folds the partials with all its threads (the operator is commutative)
    __threadfence();
    T r = T();
    bool rh = false;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += BLOCK) {
        const T p = *(volatile T*)&partials[b];
        const int ph = *(volatile int*)&partial_has[b];
        opt_combine(r, rh, p, ph != 0, op);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const T o = shfl_down_any(r, d);
        const int oh = __shfl_down_sync(0xffffffffu, (int)rh, d);
        if ((int)lane_id() + d < 32 && oh) { r = rh ? (T)op(r, o) : o; rh = true; }
    }
    __syncthreads();  // s_w / s_wh are reused
    if (lane_id() == 0) { s_w[warp] = r; s_wh[warp] = rh ? 1 : 0; }
    __syncthreads();
    if (threadIdx.x == 0) {
        T t = init;
        bool th = has_init != 0;
        for (int w = 0; w < WARPS; w++) opt_combine(t, th, s_w[w], s_wh[w] != 0, op);
        *result = t;
        *done_ctr = 0;  // leaves the counter ready for the next call
    }
}

}  // namespace trtc
