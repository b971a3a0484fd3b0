// trtc_radix.cuh -- onesweep LSD radix sort (8-bit digits) for the built-in key types.
//
// Replaces the reference's 1-bit-per-pass split sort (internal/radix_sort.cpp:165-553),
// producing the identical stable order:
//   * hist kernel: one read of the keys builds the 256-bin histogram of every digit of the
//     ordered key code (RadixKey<K>::ordered), flags NaNs, and clears the first look-back
//     status array;
//   * plan kernel: marks digits whose histogram has a bucket holding every key as no-ops
//     (the reference's varying-bit mask, internal/radix_sort.cpp:11-45, at digit granularity),
//     scans the histograms into bucket bases and picks the ping-pong buffer of every pass so
//     the result lands in the caller's buffer without a host round trip;
//   * min-tree + count kernels (float/double, only when a NaN is present): the reference
//     offsets keys by keys[TRTC_Min_Element], whose 256-wide tree (extrema.cpp:5-13 over
//     internal/general_reduce.cpp:55-95) can select a non-minimum when NaNs sit in left slots;
//     the sorted order is then a rotation, applied by the last digit pass's scatter;
//   * one pass kernel per digit: a CTA takes tiles in launch order from an atomic counter,
//     ranks its keys with warp multisplit (bit ballots), publishes per-digit counts,
//     looks back across earlier tiles for its global offsets (decoupled look-back with
//     release/acquire flags and bounded spins), stages the tile in shared memory in digit
//     order (a full tile's 4-byte payloads arrive there by one TMA bulk copy issued when the
//     tile starts) and writes it out in bucket runs.
#pragma once
#include "trtc_prelude.cuh"

namespace trtc {

struct SortPlan {
    uint32_t active_mask;      // bit p: digit pass p moves data
    uint32_t num_active;
    int32_t ordinal[8];        // running index of active pass p (selects the status array)
    uint32_t src_sel[8];       // buffer set a pass reads: 0 caller, 1 temp A, 2 temp B
    uint32_t dst_sel[8];
    int32_t last_pass;         // last active pass (applies the rotation)
    uint32_t copy_back;        // one active pass only: result sits in temp A
    uint32_t base[8][256];     // exclusive bucket starts of every pass
};

// Per-call control block; the host zeroes it (one memset) before every sort.
struct SortCtrl {
    uint32_t hist[8][256];
    uint32_t tile_ctr[8];
    uint32_t nan_flag;
    uint32_t err;
    unsigned long long rot_count;   // keys ordered strictly below the selected minimum
    SortPlan plan;
};

struct SortBufs {
    void* keys[3];
    void* vals[3];
    uint32_t* err;   // host-visible error word
};

template <class S> struct StatusBits;
template <> struct StatusBits<uint32_t> {
    static constexpr int SHIFT = 30;
    static constexpr uint32_t MASK = 0x3FFFFFFFu;
};
template <> struct StatusBits<unsigned long long> {
    static constexpr int SHIFT = 62;
    static constexpr unsigned long long MASK = 0x3FFFFFFFFFFFFFFFull;
};

template <class K, bool DESC>
TRTC_FORCEINLINE uint32_t radix_digit(typename RadixKey<K>::B k, int shift) {
    typename RadixKey<K>::U u = RadixKey<K>::ordered(k);
    if (DESC) u = ~u;
    return (uint32_t)(u >> shift) & 0xFFu;
}

// inclusive scan over the 256 threads of a (sub)block; threads >= 256 must also call it
template <int BLOCK>
__device__ inline uint32_t block_excl_scan_256(uint32_t v, uint32_t* s_wsum) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (t < 256 && lane == 31) s_wsum[w] = x;
    __syncthreads();
    uint32_t pre = 0;
    if (t < 256)
        for (int i = 0; i < w; i++) pre += s_wsum[i];
    __syncthreads();
    return pre + x - v;
}

// ------------------------------------------------------------------ histogram
// One CTA per SM.  Every lane of a warp owns a private column of the shared histogram
// (bin b of digit p at word (p*256 + b)*COPIES + lane % COPIES), so the shared-memory atomics
// of a warp never collide on an address or a bank (COPIES = 32; 16 for 8-digit keys, whose
// lanes l and l+16 may share a word), whatever the key distribution.  Loads are 16-byte
// vectors, UNROLL of them in flight per thread.
template <class K> struct HistCopies { enum { V = RadixKey<K>::DIGITS > 4 ? 16 : 32 }; };

template <class K, bool DESC, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) radix_hist_kernel(const typename RadixKey<K>::B* __restrict__ keys, size_t n,
                                                              SortCtrl* ctrl, uint4* status0, size_t status_vec4) {
    typedef RadixKey<K> RK;
    typedef typename RK::B KB;
    constexpr int D = RK::DIGITS;
    constexpr int C = HistCopies<K>::V;
    constexpr int VEC = 16 / (int)sizeof(KB);
    constexpr int UNROLL = 4;
    extern __shared__ __align__(16) uint32_t s_hist[];  // [D][256][C]
    __shared__ uint32_t s_nan;
    for (int i = threadIdx.x; i < D * 256 * C; i += BLOCK) s_hist[i] = 0;
    if (threadIdx.x == 0) s_nan = 0;

    // clear the first look-back status array (the pass kernels clear the next one)
    for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < status_vec4; i += (size_t)gridDim.x * BLOCK)
        status0[i] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();

    uint32_t* col = s_hist + (threadIdx.x & (C - 1));
    bool any_nan = false;
    auto count_key = [&](KB k) {
        if (RK::is_nan(k)) any_nan = true;
        typename RK::U u = RK::ordered(k);
        if (DESC) u = ~u;
#pragma unroll
        for (int p = 0; p < D; p++) {
            const uint32_t w = (p < 4) ? (uint32_t)u : (uint32_t)((unsigned long long)u >> 32);
            const uint32_t d = __byte_perm(w, 0u, 0x4440u | (uint32_t)(p & 3));
            atomicAdd(col + (p * 256 + d) * C, 1u);
        }
    };

    const size_t nvec = ((((size_t)keys) & 15) == 0) ? n / VEC : 0;
    const uint4* kv = reinterpret_cast<const uint4*>(keys);
    const size_t stride = (size_t)gridDim.x * BLOCK;
    size_t v = (size_t)blockIdx.x * BLOCK + threadIdx.x;
    for (; v + (UNROLL - 1) * stride < nvec; v += UNROLL * stride) {
        union { uint4 q; KB k[VEC]; } u[UNROLL];
#pragma unroll
        for (int r = 0; r < UNROLL; r++) u[r].q = kv[v + r * stride];
#pragma unroll
        for (int r = 0; r < UNROLL; r++)
#pragma unroll
            for (int e = 0; e < VEC; e++) count_key(u[r].k[e]);
    }
    for (; v < nvec; v += stride) {
        union { uint4 q; KB k[VEC]; } u;
        u.q = kv[v];
#pragma unroll
        for (int e = 0; e < VEC; e++) count_key(u.k[e]);
    }
    // scalar tail (and unaligned inputs)
    for (size_t i = nvec * VEC + (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += stride) count_key(keys[i]);
    if (any_nan) s_nan = 1;
    __syncthreads();
    // fold the columns (rotated start: the lanes of a warp read different banks)
    for (int b = threadIdx.x; b < D * 256; b += BLOCK) {
        uint32_t sum = 0;
#pragma unroll 8
        for (int c = 0; c < C; c++) sum += s_hist[b * C + ((c + b) & (C - 1))];
        if (sum) atomicAdd(&ctrl->hist[0][0] + b, sum);
    }
    if (threadIdx.x == 0 && s_nan) atomicOr(&ctrl->nan_flag, 1u);
}

// ------------------------------------------------------------------ plan (1 block of 256)
template <int D>
__global__ void __launch_bounds__(256) radix_plan_kernel(SortCtrl* ctrl, size_t n) {
    __shared__ uint32_t s_wsum[8];
    __shared__ uint32_t s_active[8];
    const int t = threadIdx.x;
    for (int p = 0; p < D; p++) {
        const uint32_t c = ctrl->hist[p][t];
        const int full = __syncthreads_or(c == (uint32_t)n);
        const uint32_t ex = block_excl_scan_256<256>(c, s_wsum);
        ctrl->plan.base[p][t] = ex;
        if (t == 0) s_active[p] = full ? 0u : 1u;
    }
    __syncthreads();
    if (t == 0) {
        SortPlan& pl = ctrl->plan;
        uint32_t mask = 0;
        for (int p = 0; p < D; p++) mask |= s_active[p] << p;
        const int a = __popc(mask);
        pl.active_mask = mask;
        pl.num_active = (uint32_t)a;
        pl.copy_back = (a == 1) ? 1u : 0u;
        pl.last_pass = -1;
        int j = 0;
        uint32_t cur = 0;
        for (int p = 0; p < 8; p++) {
            pl.ordinal[p] = 0; pl.src_sel[p] = 0; pl.dst_sel[p] = 0;
            if (p >= D || !((mask >> p) & 1u)) continue;
            uint32_t dst;
            if (a == 1) dst = 1;
            else if ((a & 1) == 0) dst = (j & 1) ? 0u : 1u;
            else if (j == 0) dst = 1;
            else if (j == 1) dst = 2;
            else if (j == 2) dst = 0;
            else dst = (j & 1) ? 1u : 0u;
            pl.ordinal[p] = j;
            pl.src_sel[p] = cur;
            pl.dst_sel[p] = dst;
            pl.last_pass = p;
            cur = dst;
            j++;
        }
    }
}

// ------------------------------------------------------------------ Min_Element tree
// Exact replica of the reference's index reduction order: consecutive blocks of 256, inside
// a block the strided tree s = 128..1 with "if (tid < s && i + s < n) h[tid] = op(h[tid],
// h[tid+s])", op(i1, i2) = v[i2] < v[i1] ? i2 : i1.  One warp handles one 256-block: lane l
// holds slots l, l+32, ..., l+224.  FIRST: read keys; otherwise read a previous round.
// One warp applies the tree to one 256-block of L <= 256 slots; load(t, v, i) yields slot t
// (t < L).  Lane 0 holds the block's (value, index) on return.
template <class K, class Load>
TRTC_FORCEINLINE void min_tree_warp256(Load load, uint32_t L, K& out_v, unsigned long long& out_i) {
    const uint32_t lane = threadIdx.x & 31u;
    K v[8];
    unsigned long long ix[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint32_t t = lane + 32u * k;
        if (t < L) load(t, v[k], ix[k]);
        else { v[k] = K(); ix[k] = 0; }
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (lane + 32u * k + 128u < L && v[k + 4] < v[k]) { v[k] = v[k + 4]; ix[k] = ix[k + 4]; }
#pragma unroll
    for (int k = 0; k < 2; k++)
        if (lane + 32u * k + 64u < L && v[k + 2] < v[k]) { v[k] = v[k + 2]; ix[k] = ix[k + 2]; }
    if (lane + 32u < L && v[1] < v[0]) { v[0] = v[1]; ix[0] = ix[1]; }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const K ov = shfl_down_any(v[0], s);
        const unsigned long long oi = __shfl_down_sync(0xffffffffu, ix[0], s);
        if (lane < (uint32_t)s && lane + s < L && ov < v[0]) { v[0] = ov; ix[0] = oi; }
    }
    out_v = v[0];
    out_i = ix[0];
}

template <class K, bool FIRST, bool NAN_GATE>
__global__ void __launch_bounds__(256) min_tree_kernel(const typename RadixKey<K>::B* __restrict__ keys,
                                                        const K* __restrict__ in_v,
                                                        const unsigned long long* __restrict__ in_i, size_t m,
                                                        K* __restrict__ out_v, unsigned long long* __restrict__ out_i,
                                                        const SortCtrl* ctrl) {
    if (NAN_GATE && ctrl->nan_flag == 0) return;
    const uint32_t lane = threadIdx.x & 31u;
    const size_t nb = (m + 255) / 256;
    const size_t warps_total = (size_t)gridDim.x * (blockDim.x / 32);
    for (size_t b = (size_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); b < nb; b += warps_total) {
        const size_t base = b * 256;
        const uint32_t L = (uint32_t)((m - base) < 256 ? (m - base) : 256);
        K rv;
        unsigned long long ri;
        min_tree_warp256<K>(
            [&](uint32_t t, K& v, unsigned long long& i) {
                if constexpr (FIRST) { v = RadixKey<K>::value(keys[base + t]); i = base + t; }
                else { v = in_v[base + t]; i = in_i[base + t]; }
            },
            L, rv, ri);
        if (lane == 0) { out_v[b] = rv; out_i[b] = ri; }
    }
}

// number of keys whose ordered code is below the selected minimum's (NaN case only).
// 16-byte loads, four per thread in flight (a scalar grid-stride loop kept too few bytes in
// flight to reach HBM bandwidth); ragged head and tail elements are read one by one.
template <class K, int BLOCK>
__global__ void __launch_bounds__(BLOCK) radix_count_below_kernel(const typename RadixKey<K>::B* __restrict__ keys, size_t n,
                                                                  const unsigned long long* min_idx, SortCtrl* ctrl) {
    if (ctrl->nan_flag == 0) return;
    typedef RadixKey<K> RK;
    typedef typename RK::B KB;
    constexpr int PER = 16 / sizeof(KB);
    const typename RK::U tm = RK::ordered(keys[*min_idx]);
    const size_t mis = ((16u - ((size_t)keys & 15u)) & 15u) / sizeof(KB);
    const size_t head = mis < n ? mis : n;
    const size_t nvec = (n - head) / PER;
    const size_t body_end = head + nvec * PER;
    const uint4* __restrict__ vp = reinterpret_cast<const uint4*>(keys + head);
    const size_t tid = (size_t)blockIdx.x * BLOCK + threadIdx.x, stride = (size_t)gridDim.x * BLOCK;
    unsigned long long c = 0;
    if (tid < head) c += RK::ordered(keys[tid]) < tm ? 1ull : 0ull;
    for (size_t i = tid; i < nvec; i += 4 * stride) {
        uint4 q[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (i + u * stride < nvec) q[u] = vp[i + u * stride];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (i + u * stride >= nvec) continue;
            union { uint4 v; KB k[PER]; } w;
            w.v = q[u];
#pragma unroll
            for (int e = 0; e < PER; e++) c += RK::ordered(w.k[e]) < tm ? 1ull : 0ull;
        }
    }
    if (body_end + tid < n) c += RK::ordered(keys[body_end + tid]) < tm ? 1ull : 0ull;  // tail < PER elements
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
    if ((threadIdx.x & 31u) == 0 && c) atomicAdd(&ctrl->rot_count, c);
}

// ------------------------------------------------------------------ one digit pass
// 4- or 8-byte asynchronous copy global -> shared (cp.async, L1-allocating)
template <class V>
TRTC_FORCEINLINE void cp_async_elem(V* smem_dst, const V* gsrc) {
    static_assert(sizeof(V) == 4 || sizeof(V) == 8, "cp.async element of 4 or 8 bytes");
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gsrc), "n"((int)sizeof(V)) : "memory");
}
TRTC_FORCEINLINE void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Bulk copy global -> shared by the tensor memory accelerator (cp.async.bulk, no
// multicast), completing on a shared-memory mbarrier.  Both addresses 16-byte aligned, the
// size a multiple of 16.  The copy's shared-memory writes do not use the SM's load/store
// pipe.
TRTC_FORCEINLINE uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
TRTC_FORCEINLINE void mbar_init_one(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
    // make the initialised barrier visible to the copy engine (async proxy)
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
TRTC_FORCEINLINE void bulk_load_g2s(void* sdst, const void* gsrc, uint32_t bytes, unsigned long long* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(sdst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
TRTC_FORCEINLINE bool mbar_try_wait(unsigned long long* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for phase `parity` of the barrier; false when the poll budget is spent
TRTC_FORCEINLINE bool mbar_wait_bounded(unsigned long long* bar, uint32_t parity, const uint32_t* err) {
    uint32_t spins = 0;
    while (!mbar_try_wait(bar, parity))
        if (!spin_continue(spins, err)) return false;
    return true;
}

// Digit of byte `pass` of the ordered key code: one byte permute on the 32-bit half that
// holds it (sel = 0x4440 | byte index within the half).
template <class K, bool DESC>
TRTC_FORCEINLINE uint32_t radix_digit_sel(typename RadixKey<K>::B k, uint32_t sel, bool hi) {
    const typename RadixKey<K>::U u = RadixKey<K>::ordered(k);
    uint32_t w;
    if constexpr (sizeof(typename RadixKey<K>::U) == 8) w = hi ? (uint32_t)(u >> 32) : (uint32_t)u;
    else w = (uint32_t)u;
    const uint32_t d = __byte_perm(w, 0u, sel);
    return DESC ? (d ^ 0xFFu) : d;
}

template <bool B> struct BoolC { static constexpr bool value = B; };

#ifndef TRTC_RADIX_MINB  // resident CTAs per SM the pass kernel is compiled for
#define TRTC_RADIX_MINB(items) ((items) >= 24 ? 2 : 4)
#endif
#ifndef TRTC_RADIX_LB
#define TRTC_RADIX_LB 4  // predecessor tiles polled per look-back round
#endif
// Peer groups of equal digit inside a warp come from two methods that load different
// pipes: items i with i % MIXP < MIXB use eight bit ballots (ALU and vote instructions),
// the others atomicOr their lane bit into a per-warp mask per digit in shared memory (LSU).
// Measured on B200 (2^28 u32 pairs): masks alone move the pass onto the LSU pipe, ballots
// alone onto issue; one item in three on ballots balances them for pairs, one in five for
// keys alone (no payload traffic on the LSU pipe; 2^28 u32 keys 4.605 -> 4.569 ms, pairs
// 5.701 -> 5.727 ms at one in five).  __match_any_sync was 50 % slower than either.
#ifndef TRTC_RADIX_MIXP
#define TRTC_RADIX_MIXP 3
#endif
#ifndef TRTC_RADIX_MIXP_KEYS
#define TRTC_RADIX_MIXP_KEYS 5
#endif
#ifndef TRTC_RADIX_MIXB
#define TRTC_RADIX_MIXB 1
#endif
// ranks of item i are resolved (shuffle from the group leader) RWIN items after its atomic:
// the window covers the atomic's latency and bounds the live per-item state (resolving all
// ranks after the loop spilled)
#ifndef TRTC_RADIX_RWIN
#define TRTC_RADIX_RWIN 4
#endif
// payloads copied global -> staging slot with cp.async after the block scan (no registers
// held across the ranking, which makes room for 4 CTAs per SM) instead of loaded into
// registers before it
#ifndef TRTC_RADIX_VASYNC
#define TRTC_RADIX_VASYNC 1
#endif
// 4-byte payloads of a full tile: one bulk copy (cp.async.bulk) of the tile's payloads into
// the payload staging area, issued when the tile starts and overlapped with the ranking;
// at staging every thread reads its payloads from there (consecutive words) and, after a
// barrier, writes them to their staging slots.  Replaces the per-element cp.async copies
// and their scattered shared-memory writes through the load/store pipe.
#ifndef TRTC_RADIX_VBULK
#define TRTC_RADIX_VBULK 1
#endif
// the digit masks: two alternating sets of 256 words per warp, placed in the key/payload
// staging area (idle during the ranking) when it is large enough, else after the counters
template <int BLOCK>
constexpr size_t radix_match_words() { return (size_t)(BLOCK / 32) * 2 * 256; }
template <class KB, class V, bool HAS_VALS, int BLOCK, int TILE>
constexpr size_t radix_match_smem() {
    return (TRTC_RADIX_MIXB < TRTC_RADIX_MIXP &&
            (size_t)TILE * (sizeof(KB) + (HAS_VALS ? sizeof(V) : 0)) < radix_match_words<BLOCK>() * 4)
               ? radix_match_words<BLOCK>() * 4 : (size_t)0;
}
// the bulk payload path needs 4-byte payloads, a tile of whole 16-byte chunks, and digit
// masks that do not overlap the payload area (it is filled during the ranking)
template <class KB, class V, bool HAS_VALS, int BLOCK, int TILE>
constexpr bool radix_vbulk() {
    return TRTC_RADIX_VBULK && HAS_VALS && sizeof(V) == 4 && ((size_t)TILE * sizeof(V)) % 16 == 0 &&
           (TRTC_RADIX_MIXB >= TRTC_RADIX_MIXP || radix_match_smem<KB, V, HAS_VALS, BLOCK, TILE>() != 0 ||
            (size_t)TILE * sizeof(KB) >= radix_match_words<BLOCK>() * 4);
}

// HAS_VALS: move a 4- or 8-byte payload with the keys.  vals_from_index: the payload of the
// first active pass is the element index (used to sort a permutation for odd value sizes).
//
// Per tile (BLOCK threads x ITEMS keys, warp-striped: key i of lane l of warp w sits at
// tile_base + w*32*ITEMS + i*32 + l):
//   1. load the keys; rank every key inside its warp (peers of equal digit from bit
//      ballots or shared-memory digit masks, one shared-memory atomicAdd per peer group on
//      the warp's digit counters);
//   2. (payloads are not held in registers across the ranking: a full tile's 4-byte
//      payloads arrive by one bulk copy issued at the tile's start, others are copied
//      with cp.async in step 4)
//   3. one thread per digit: tile count, publication of the tile aggregate, block-wide
//      exclusive scan of the counts, warp offsets folded into the warp counters;
//   4. stage keys (and payloads) in shared memory in digit order; then, one thread per
//      digit, decoupled look-back for the digit's global offset, publication of the
//      inclusive prefix, and a range check of the digit's destination run against n;
//   5. write the tile out in bucket runs: consecutive threads write consecutive slots of a
//      digit's run.
template <class K, class V, bool HAS_VALS, bool DESC, int BLOCK, int ITEMS, class ST>
__global__ void __launch_bounds__(BLOCK, TRTC_RADIX_MINB(ITEMS)) radix_pass_kernel(SortBufs bufs, size_t n, SortCtrl* ctrl, int pass,
                                                           ST* status0, ST* status1, int vals_from_index,
                                                           uint32_t pf_tiles) {
    static_assert(BLOCK == 256, "one thread per digit");
    constexpr int TILE = BLOCK * ITEMS;
    constexpr int WARPS = BLOCK / 32;
    constexpr int MIXP = HAS_VALS ? TRTC_RADIX_MIXP : TRTC_RADIX_MIXP_KEYS;
    static_assert(TRTC_RADIX_MIXB < TRTC_RADIX_MIXP_KEYS || TRTC_RADIX_MIXB >= TRTC_RADIX_MIXP,
                  "keys-only and pair sorts agree on whether digit masks are used");
    constexpr bool FLOATKEY = is_same<K, float>::value || is_same<K, double>::value;
    typedef StatusBits<ST> SB;
    typedef typename RadixKey<K>::B KB;
    // element positions: 32-bit while n < 2^30 (ST = uint32_t), else 64-bit
    typedef typename conditional<(sizeof(ST) == 8), unsigned long long, uint32_t>::type IX;
    const SortPlan& plan = ctrl->plan;
    if (!((plan.active_mask >> pass) & 1u)) return;

    extern __shared__ __align__(16) unsigned char smem[];
    KB* s_keys = reinterpret_cast<KB*>(smem);
    V* s_vals = reinterpret_cast<V*>(smem + sizeof(KB) * TILE);
    uint32_t* s_whist = reinterpret_cast<uint32_t*>(smem + sizeof(KB) * TILE + (HAS_VALS ? sizeof(V) * TILE : 0));
    // digit masks (see radix_match_smem)
    uint32_t* s_wmatch = radix_match_smem<KB, V, HAS_VALS, BLOCK, TILE>() ? s_whist + WARPS * 256
                                                                         : reinterpret_cast<uint32_t*>(smem);
    __shared__ IX s_adj[256];
    __shared__ uint32_t s_wsum[8];
    __shared__ uint32_t s_tile;
    __shared__ __align__(8) unsigned long long s_vbar;  // completion of the bulk payload copy
    constexpr bool VB = radix_vbulk<KB, V, HAS_VALS, BLOCK, TILE>();

    const int ord = plan.ordinal[pass];
    ST* st = (ord & 1) ? status1 : status0;
    ST* st_next = (ord & 1) ? status0 : status1;
    // buffer selection with selects (a runtime index into the parameter array would copy
    // it to local memory)
    const uint32_t ss = plan.src_sel[pass], ds = plan.dst_sel[pass];
    const KB* __restrict__ src_k =
        reinterpret_cast<const KB*>(ss == 0 ? bufs.keys[0] : (ss == 1 ? bufs.keys[1] : bufs.keys[2]));
    KB* __restrict__ dst_k = reinterpret_cast<KB*>(ds == 0 ? bufs.keys[0] : (ds == 1 ? bufs.keys[1] : bufs.keys[2]));
    const V* __restrict__ src_v =
        reinterpret_cast<const V*>(ss == 0 ? bufs.vals[0] : (ss == 1 ? bufs.vals[1] : bufs.vals[2]));
    V* __restrict__ dst_v = reinterpret_cast<V*>(ds == 0 ? bufs.vals[0] : (ds == 1 ? bufs.vals[1] : bufs.vals[2]));
    const uint32_t sel = 0x4440u | (uint32_t)(pass & 3);
    const bool hi = pass >= 4;
    const bool index_payload = HAS_VALS && vals_from_index && ord == 0;
    IX rot = 0;
    if (FLOATKEY && pass == plan.last_pass && ctrl->rot_count) {
        const unsigned long long k = ctrl->rot_count % n;
        rot = (IX)(DESC ? k : (k ? n - k : 0));
    }

    if (threadIdx.x == 0) s_tile = atomicAdd(&ctrl->tile_ctr[ord], 1u);
    for (int i = threadIdx.x; i < WARPS * 256; i += BLOCK) s_whist[i] = 0;
    if (TRTC_RADIX_MIXB < TRTC_RADIX_MIXP)
        for (int i = threadIdx.x; i < (int)radix_match_words<BLOCK>(); i += BLOCK) s_wmatch[i] = 0;
    __syncthreads();
    const size_t tile = s_tile;
    st_next[tile * 256 + threadIdx.x] = 0;

    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const size_t tile_base = tile * TILE;
    const size_t wbase = tile_base + (size_t)warp * 32 * ITEMS;
    const KB* __restrict__ wk = src_k + wbase;
    const bool full = tile_base + TILE <= n;
    const uint32_t tile_n = full ? (uint32_t)TILE : (uint32_t)(n - tile_base);
    // tiles are claimed in order, so the tile pf_tiles ahead (a fraction of the ~4 tiles per
    // SM in flight) starts a few tile durations later: one TMA bulk prefetch brings its keys
    // and payloads into L2 now, and its CTA's loads then wait on L2 instead of HBM (whole
    // tiles inside [0, n) only; the prefetch is a hint and changes no result)
    if (pf_tiles && threadIdx.x == 32) {
        const size_t fb = tile_base + (size_t)pf_tiles * TILE;
        prefetch_l2_range(src_k, fb, (size_t)TILE, n);
        if (HAS_VALS && !index_payload) prefetch_l2_range(src_v, fb, (size_t)TILE, n);
    }
    // uniform over the CTA: full tile, loaded payloads, 16-byte aligned source
    const bool vbulk = VB && full && !index_payload && ((reinterpret_cast<uintptr_t>(src_v + tile_base) & 15u) == 0);
    if (vbulk && threadIdx.x == 0) {
        mbar_init_one(&s_vbar);
        bulk_load_g2s(s_vals, src_v + tile_base, (uint32_t)(TILE * sizeof(V)), &s_vbar);
    }
    // keys of this warp inside the tile (partial tiles only)
    const uint32_t warp_n = full ? 32u * ITEMS
                                 : (tile_n > warp * 32u * ITEMS ? min(tile_n - warp * 32u * ITEMS, 32u * ITEMS) : 0u);

    KB keys[ITEMS];
    uint32_t rank[ITEMS];
    V vals[HAS_VALS ? ITEMS : 1];
    uint32_t* wh = s_whist + warp * 256;

    // ---- 1. load + warp multisplit ranking
    auto rank_tile = [&](auto full_c) {
        constexpr bool FULL = decltype(full_c)::value;
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t r = (uint32_t)i * 32u + lane;
            keys[i] = (FULL || r < warp_n) ? wk[r] : KB(0);
        }
        const uint32_t ltm = lanemask_lt();
        uint32_t info[ITEMS];  // rank among peers | group leader lane << 8
        constexpr int RW = (TRTC_RADIX_RWIN > 0 && TRTC_RADIX_RWIN < ITEMS) ? TRTC_RADIX_RWIN : ITEMS;
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t d = radix_digit_sel<K, DESC>(keys[i], sel, hi);
            uint32_t peers;
            if ((i % MIXP) < TRTC_RADIX_MIXB) {
                peers = FULL ? 0xffffffffu : __ballot_sync(0xffffffffu, (uint32_t)i * 32u + lane < warp_n);
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    const bool bit = (d >> b) & 1u;
                    const uint32_t bb = __ballot_sync(0xffffffffu, bit);
                    peers &= bit ? bb : ~bb;
                }
            } else {
                const bool valid = FULL || (uint32_t)i * 32u + lane < warp_n;
                // the two mask sets alternate over the mask-ranked items, so a set is reused
                // only after the other set's item and its two warp barriers
                const int ors_before = i - ((i / MIXP) * TRTC_RADIX_MIXB +
                                            ((i % MIXP) < TRTC_RADIX_MIXB ? (i % MIXP) : TRTC_RADIX_MIXB));
                uint32_t* wm = s_wmatch + warp * 512 + (ors_before & 1) * 256;
                if (valid) atomicOr(&wm[d], 1u << lane);
                __syncwarp();
                peers = valid ? wm[d] : 0u;
                __syncwarp();
                if (valid && lane == 31u - __clz(peers)) wm[d] = 0u;
            }
            // the highest lane of a group adds the group's size to the warp's digit counter
            const uint32_t leader = 31u - __clz(peers);
            info[i] = (uint32_t)__popc(peers & ltm) | (leader << 8);
            rank[i] = 0;
            if (lane == leader && (FULL || (uint32_t)i * 32u + lane < warp_n))
                rank[i] = atomicAdd(&wh[d], (uint32_t)__popc(peers));
            if (i >= RW) {
                const int j = i - RW;
                rank[j] = __shfl_sync(0xffffffffu, rank[j], (int)(info[j] >> 8)) + (info[j] & 0xFFu);
            }
        }
#pragma unroll
        for (int j = ITEMS - RW; j < ITEMS; j++)
            rank[j] = __shfl_sync(0xffffffffu, rank[j], (int)(info[j] >> 8)) + (info[j] & 0xFFu);
        // ---- 2. payload loads, consumed only at staging
        if constexpr (HAS_VALS && !TRTC_RADIX_VASYNC) {
            const V* __restrict__ wv = src_v + wbase;
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const uint32_t r = (uint32_t)i * 32u + lane;
                if (FULL || r < warp_n) vals[i] = index_payload ? (V)(wbase + r) : wv[r];
            }
        }
    };
    if (full) rank_tile(BoolC<true>());
    else rank_tile(BoolC<false>());
    __syncthreads();

    // ---- 3. one thread per digit: tile count, aggregate, block scan, warp offsets
    const uint32_t d_me = threadIdx.x;
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < WARPS; w++) cnt += s_whist[w * 256 + d_me];
    st_relaxed(&st[tile * 256 + d_me], ((ST)(tile == 0 ? 2u : 1u) << SB::SHIFT) | (ST)cnt);
    const uint32_t start = block_excl_scan_256<BLOCK>(cnt, s_wsum);
    {
        uint32_t run = start;
#pragma unroll
        for (int w = 0; w < WARPS; w++) {
            const uint32_t c = s_whist[w * 256 + d_me];
            s_whist[w * 256 + d_me] = run;
            run += c;
        }
    }
    __syncthreads();

    // ---- 4. stage in digit order
    bool bad = false;
    if (vbulk) {
        // keys to their slots (rank[] becomes the slot), then the payloads: read from the
        // bulk-copied tile in the keys' striped order, a barrier, written to the same slots
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            rank[i] += wh[radix_digit_sel<K, DESC>(keys[i], sel, hi)];
            s_keys[rank[i]] = keys[i];
        }
        if (!mbar_wait_bounded(&s_vbar, 0u, bufs.err)) {
            report_error(bufs.err, TRTC_ERR_BULK_COPY_TIMEOUT);
            bad = true;
        }
        V pv[VB ? ITEMS : 1];
        const V* wraw = s_vals + warp * 32u * ITEMS + lane;
#pragma unroll
        for (int i = 0; i < (VB ? ITEMS : 1); i++) pv[i] = wraw[i * 32];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < (VB ? ITEMS : 1); i++) s_vals[rank[i]] = pv[i];
    } else {
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            if (full || (uint32_t)i * 32u + lane < warp_n) {
                const uint32_t d = radix_digit_sel<K, DESC>(keys[i], sel, hi);
                const uint32_t pos = wh[d] + rank[i];
                s_keys[pos] = keys[i];
                if constexpr (HAS_VALS) {
                    if constexpr (TRTC_RADIX_VASYNC) {
                        const uint32_t r = (uint32_t)i * 32u + lane;
                        if (index_payload) s_vals[pos] = (V)(wbase + r);
                        else cp_async_elem(&s_vals[pos], src_v + wbase + r);
                    } else {
                        s_vals[pos] = vals[i];
                    }
                }
            }
        }
        if constexpr (HAS_VALS && TRTC_RADIX_VASYNC) cp_async_wait_all();  // before the barrier below
    }

    // ---- decoupled look-back for the digit's global offset.  Each round polls LB
    // predecessor tiles at once (independent loads), so the inclusive-prefix frontier
    // advances LB tiles per memory round trip.
    {
        constexpr int LB = TRTC_RADIX_LB;
        ST excl = 0;
        if (tile > 0) {
            long long j = (long long)tile - 1;  // newest tile not yet accumulated
            uint32_t spins = 0;
            bool done = false;
            while (!done) {
                ST s[LB];
#pragma unroll
                for (int k = 0; k < LB; k++)
                    s[k] = (j - k >= 0) ? ld_relaxed(&st[(size_t)(j - k) * 256 + d_me]) : ((ST)2u << SB::SHIFT);
                int used = 0;
#pragma unroll
                for (int k = 0; k < LB; k++) {
                    if (done || used != k) continue;  // stop at the first tile not yet published
                    const uint32_t f = (uint32_t)(s[k] >> SB::SHIFT);
                    if (f == 0) continue;
                    excl += s[k] & SB::MASK;
                    used = k + 1;
                    if (f == 2) done = true;
                }
                j -= used;
                if (!done && j < 0) done = true;
                if (!done && used == 0) {
                    if (!spin_continue(spins, bufs.err)) { report_error(bufs.err, TRTC_ERR_LOOKBACK_TIMEOUT); bad = true; break; }
                }
            }
            st_relaxed(&st[tile * 256 + d_me], ((ST)2u << SB::SHIFT) | (excl + (ST)cnt));
        }
        // the digit's destination run must lie inside [0, n)
        const unsigned long long lo = (unsigned long long)plan.base[pass][d_me] + (unsigned long long)excl;
        if (lo + cnt > (unsigned long long)n) bad = true;
        s_adj[d_me] = (IX)lo - (IX)start;
    }
    if (__syncthreads_or(bad)) {  // also completes the staging
        if (threadIdx.x == 0) report_error(bufs.err, TRTC_ERR_BAD_PLAN);
        return;
    }

    // ---- 5. write out in bucket runs
    auto write_tile = [&](auto full_c) {
        constexpr bool FULL = decltype(full_c)::value;
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t k = (uint32_t)i * BLOCK + threadIdx.x;
            if (FULL || k < tile_n) {
                const KB key = s_keys[k];
                const uint32_t d = radix_digit_sel<K, DESC>(key, sel, hi);
                IX dst = s_adj[d] + (IX)k;
                if constexpr (FLOATKEY) {
                    dst += rot;
                    if (dst >= (IX)n) dst -= (IX)n;
                }
                dst_k[dst] = key;
                if (HAS_VALS) dst_v[dst] = s_vals[k];
            }
        }
    };
    if (full) write_tile(BoolC<true>());
    else write_tile(BoolC<false>());
}

// single active pass: the result sits in temp A and is copied back to the caller's buffers
template <class K, class V, bool HAS_VALS>
__global__ void radix_copyback_kernel(SortBufs bufs, size_t n, const SortCtrl* ctrl) {
    if (!ctrl->plan.copy_back) return;
    typedef typename RadixKey<K>::B KB;
    const KB* sk = reinterpret_cast<const KB*>(bufs.keys[1]);
    KB* dk = reinterpret_cast<KB*>(bufs.keys[0]);
    const V* sv = reinterpret_cast<const V*>(bufs.vals[1]);
    V* dv = reinterpret_cast<V*>(bufs.vals[0]);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        dk[i] = sk[i];
        if (HAS_VALS) dv[i] = sv[i];
    }
}

// payloads of other sizes: values[i] = values_orig[perm[i]] through a temp copy
static __global__ void radix_gather_bytes_kernel(const unsigned char* __restrict__ vals, unsigned char* __restrict__ tmp,
                                          const uint32_t* __restrict__ perm, size_t n, int esize, const SortCtrl* ctrl) {
    if (ctrl->plan.num_active == 0) return;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t s = perm[i];
        if (s >= n) continue;
        for (int b = 0; b < esize; b++) tmp[i * esize + b] = vals[s * esize + b];
    }
}
static __global__ void radix_copy_bytes_gated_kernel(const unsigned char* __restrict__ src, unsigned char* __restrict__ dst,
                                              size_t nbytes, const SortCtrl* ctrl) {
    if (ctrl->plan.num_active == 0) return;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nbytes; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

}  // namespace trtc
