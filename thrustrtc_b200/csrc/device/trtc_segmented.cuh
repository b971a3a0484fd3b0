// trtc_segmented.cuh -- batched segmented sort + scan: many independent segments of one
// key/value array, each stably sorted by key and then exclusive-scanned (Plus) over its
// sorted values, in one persistent launch fed by a device work queue.
//
// The reference sorts one vector per call (internal/radix_sort.cpp:165-553) and scans one
// vector per call (internal/general_scan.cpp:8-88); a batch there is one call pair per
// segment.  Here a CTA takes a segment id from the queue and sorts the whole segment itself,
// in one of six size classes (ITEMS and warp_small are the tuning table's; launch_segmented.cu):
//   * segments of at most `warp_small` (0 or 32) keys: one warp, a bitonic network over
//     (code, index) pairs, no digit counters (seg_warp_bitonic);
//   * segments of at most 32 * ITEMS keys: one warp, four 8-bit LSD passes of ballot
//     ranking with per-warp counters (seg_warp_sort_scan); a CTA's eight warps take eight
//     such segments at once;
//   * segments of at most 64 * ITEMS / 128 * ITEMS keys: a group of two / four warps, the
//     same passes with the group's counters scanned by the group and named barriers of the
//     group only (seg_group_sort_scan); a CTA's four / two groups take as many segments;
//   * small segments (<= 256 * ITEMS keys) are sorted on chip: four 8-bit LSD passes of
//     warp multisplit ranking + shared-memory scatter, with the tile re-laid out so that
//     every warp gets keys whatever the segment length; then the values are scanned and
//     keys, values and scan are written once;
//   * larger segments are sorted by the CTA in global memory: one read builds all digit
//     histograms, then four chunked, stable scatter passes ping-pong between the segment and
//     a temp array (mostly L2-resident for segments of up to a few MB), then a chunked
//     scan with a running carry.
// The queue lists the segments by class, largest first, so the longest work starts first and
// a CTA's batch of small segments shares one class.
#pragma once
#include "trtc_prelude.cuh"
#include "trtc_radix.cuh"

namespace trtc {

// One segment given by its own arrays (list mode, used by the request server): keys k and
// 4-byte values v sorted in place, out = exclusive scan of the sorted values (or nullptr),
// n elements, toff = the segment's offset in the temp arrays.
struct SegItem {
    void* k;
    void* v;
    void* out;
    unsigned long long n;
    unsigned long long toff;
};

// size classes of a segment of `len` keys (items = keys per thread of a CTA tile): 0 one
// warp, 1 / 2 two / four warps, 3 the CTA on chip, 4 + k the CTA through global memory with
// floor(log2 len) = floor(log2 (256 items)) + k.  The work queue lists the classes from the
// largest down, so the longest segments start first.
enum { SEG_CLASSES = 32 };
TRTC_FORCEINLINE uint32_t seg_class(unsigned long long len, uint32_t items) {
    const unsigned long long tile = 256ull * items;
    if (len > tile) {
        const int k = (63 - __clzll((long long)len)) - (63 - __clzll((long long)tile));
        return 4u + (uint32_t)min(k, SEG_CLASSES - 5);
    }
    return len > 128ull * items ? 3u : len > 64ull * items ? 2u : len > 32ull * items ? 1u : 0u;
}

struct SegCtrl {
    unsigned long long next;                   // work-queue cursor
    unsigned long long count[SEG_CLASSES];     // segments per class
    unsigned long long placed[SEG_CLASSES];    // segments of a class placed so far
    unsigned long long pad;
};

// per-class segment counts (block histogram, one atomic per class and block)
template <class OFF>
__global__ void __launch_bounds__(256) seg_class_count_kernel(const OFF* __restrict__ off, unsigned long long nseg,
                                                              uint32_t items, SegCtrl* ctrl) {
    __shared__ unsigned long long s_c[SEG_CLASSES];
    if (threadIdx.x < SEG_CLASSES) s_c[threadIdx.x] = 0;
    __syncthreads();
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < nseg;
         i += (unsigned long long)gridDim.x * blockDim.x)
        atomicAdd(&s_c[seg_class((unsigned long long)(off[i + 1] - off[i]), items)], 1ull);
    __syncthreads();
    if (threadIdx.x < SEG_CLASSES && s_c[threadIdx.x]) atomicAdd(&ctrl->count[threadIdx.x], s_c[threadIdx.x]);
}

// queue[] = the segments ordered by class, largest class first (order inside a class is free)
template <class OFF>
__global__ void __launch_bounds__(256) seg_queue_kernel(const OFF* __restrict__ off, unsigned long long nseg,
                                                        uint32_t items, uint32_t* __restrict__ queue, SegCtrl* ctrl) {
    __shared__ unsigned long long s_start[SEG_CLASSES];
    if (threadIdx.x == 0) {
        unsigned long long run = 0;
        for (int c = SEG_CLASSES - 1; c >= 0; c--) { s_start[c] = run; run += ctrl->count[c]; }
    }
    __syncthreads();
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < nseg;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t c = seg_class((unsigned long long)(off[i + 1] - off[i]), items);
        queue[s_start[c] + atomicAdd(&ctrl->placed[c], 1ull)] = (uint32_t)i;
    }
}

// Ranks IT (<= ITEMS) warp-striped items per thread of a tile of `tile_n` keys: element
// e = warp*32*IT + i*32 + lane.  On return pos[i] is the item's position in the digit-sorted
// tile (stable), s_cnt[d] / s_start[d] the tile's digit counts and exclusive starts.
template <class K, bool DESC, int ITEMS>
__device__ inline void seg_rank_tile(const typename RadixKey<K>::B (&keys)[ITEMS], uint32_t (&pos)[ITEMS], int IT,
                                     uint32_t tile_n, uint32_t sel, bool hi, uint32_t* s_whist, uint32_t* s_cnt,
                                     uint32_t* s_start, uint32_t* s_wsum) {
    constexpr int WARPS = 8;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < WARPS * 256; i += 256) s_whist[i] = 0;
    __syncthreads();
    uint32_t* wh = s_whist + warp * 256;
    const uint32_t ltm = lanemask_lt();
    const uint32_t wbase = warp * 32u * (uint32_t)IT;
    uint32_t info[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        pos[i] = 0;
        info[i] = 0;
        if (i >= IT || wbase + (uint32_t)i * 32u >= tile_n) continue;  // warp-uniform
        const bool valid = wbase + (uint32_t)i * 32u + lane < tile_n;
        const uint32_t d = radix_digit_sel<K, DESC>(keys[i], sel, hi);
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const bool set = (d >> b) & 1u;
            const uint32_t bb = __ballot_sync(0xffffffffu, set);
            peers &= set ? bb : ~bb;
        }
        const uint32_t leader = 31u - __clz(peers);
        info[i] = (uint32_t)__popc(peers & ltm) | (leader << 8);
        if (valid && lane == leader) pos[i] = atomicAdd(&wh[d], (uint32_t)__popc(peers));
    }
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        if (i >= IT || wbase + (uint32_t)i * 32u >= tile_n) continue;
        pos[i] = __shfl_sync(0xffffffffu, pos[i], (int)(info[i] >> 8)) + (info[i] & 0xFFu);
    }
    __syncthreads();
    const uint32_t d = threadIdx.x;
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < WARPS; w++) cnt += s_whist[w * 256 + d];
    const uint32_t start = block_excl_scan_256<256>(cnt, s_wsum);
    s_cnt[d] = cnt;
    s_start[d] = start;
    uint32_t run = start;
#pragma unroll
    for (int w = 0; w < WARPS; w++) {
        const uint32_t c = s_whist[w * 256 + d];
        s_whist[w * 256 + d] = run;
        run += c;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        if (i >= IT || wbase + (uint32_t)i * 32u + lane >= tile_n) continue;
        pos[i] += wh[radix_digit_sel<K, DESC>(keys[i], sel, hi)];
    }
}

// exclusive Plus scan of s_v[0..len) into s_o (256 threads, len <= 256 * ITEMS), carry-in c
template <class V, int ITEMS>
__device__ inline V seg_block_excl_scan(const V* s_v, V* s_o, uint32_t len, V carry, V* s_part) {
    const uint32_t t = threadIdx.x;
    const uint32_t per = (len + 255u) / 256u;  // consecutive elements per thread
    const uint32_t b = t * per;
    V sum = V();
    for (uint32_t k = 0; k < per; k++)
        if (b + k < len) sum += s_v[b + k];
    // block exclusive scan of the thread sums (values of any width: two warp levels)
    const uint32_t lane = t & 31u, w = t >> 5;
    V x = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const V y = shfl_up_any(x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    if (lane == 31) s_part[w] = x;
    __syncthreads();
    V pre = carry;
    for (uint32_t i = 0; i < w; i++) pre += s_part[i];
    V total = carry;
    for (int i = 0; i < 8; i++) total += s_part[i];
    V run = pre + x - sum;
    for (uint32_t k = 0; k < per; k++)
        if (b + k < len) { s_o[b + k] = run; run += s_v[b + k]; }
    __syncthreads();
    return total;
}

// One warp sorts (stable LSD, 8-bit digits) and scans a segment of len <= 32 * ITEMS keys on
// its own: no block barrier, so the CTA's eight warps work on eight small segments at once.
// Element e = i*32 + lane sits in item i of the lane; sk / sv are this warp's staging slices
// (32 * ITEMS elements), wh its 256 digit counters.
template <class K, class V, bool DESC, int ITEMS>
__device__ inline void seg_warp_sort_scan(typename RadixKey<K>::B* gk, V* gv, V* gs, uint32_t len,
                                          typename RadixKey<K>::B* sk, V* sv, uint32_t* wh) {
    typedef typename RadixKey<K>::B KB;
    constexpr int D = RadixKey<K>::DIGITS;
    const uint32_t lane = threadIdx.x & 31u;
    const int IT = (int)((len + 31u) / 32u);  // items in use (warp-uniform)
    const uint32_t ltm = lanemask_lt();
    KB k[ITEMS];
    V v[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const uint32_t e = (uint32_t)i * 32u + lane;
        if (i < IT && e < len) { k[i] = gk[e]; v[i] = gv[e]; }
        else { k[i] = KB(0); v[i] = V(); }
    }
    for (int p = 0; p < D; p++) {
        const uint32_t sel = 0x4440u | (uint32_t)(p & 3);
        const bool hi = p >= 4;
#pragma unroll
        for (int j = 0; j < 8; j++) wh[j * 32 + lane] = 0;
        __syncwarp();
        uint32_t pos[ITEMS], info[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            pos[i] = 0;
            info[i] = 0;
            if (i >= IT) continue;
            const bool valid = (uint32_t)i * 32u + lane < len;
            const uint32_t d = radix_digit_sel<K, DESC>(k[i], sel, hi);
            uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const bool set = (d >> b) & 1u;
                const uint32_t bb = __ballot_sync(0xffffffffu, set);
                peers &= set ? bb : ~bb;
            }
            const uint32_t leader = 31u - __clz(peers | 1u);
            info[i] = (uint32_t)__popc(peers & ltm) | (leader << 8);
            if (valid && lane == leader) pos[i] = atomicAdd(&wh[d], (uint32_t)__popc(peers));
        }
#pragma unroll
        for (int i = 0; i < ITEMS; i++)
            if (i < IT) pos[i] = __shfl_sync(0xffffffffu, pos[i], (int)(info[i] >> 8)) + (info[i] & 0xFFu);
        __syncwarp();
        // exclusive scan of the 256 counters: lane owns digits 8*lane .. 8*lane+7
        uint32_t c[8], sum = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) { c[j] = wh[lane * 8 + j]; sum += c[j]; }
        uint32_t inc = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= (uint32_t)d) inc += y;
        }
        uint32_t run = inc - sum;
#pragma unroll
        for (int j = 0; j < 8; j++) { wh[lane * 8 + j] = run; run += c[j]; }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            if (i >= IT || (uint32_t)i * 32u + lane >= len) continue;
            const uint32_t q = pos[i] + wh[radix_digit_sel<K, DESC>(k[i], sel, hi)];
            sk[q] = k[i];
            sv[q] = v[i];
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t e = (uint32_t)i * 32u + lane;
            if (i < IT && e < len) { k[i] = sk[e]; v[i] = sv[e]; }
        }
        __syncwarp();
    }
    // exclusive scan of the sorted values, written with the sorted keys and values
    V carry = V();
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        if (i >= IT) continue;
        const uint32_t e = (uint32_t)i * 32u + lane;
        const bool valid = e < len;
        const V x = valid ? v[i] : V();
        V incl = x;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const V y = shfl_up_any(incl, d);
            if (lane >= (uint32_t)d) incl += y;
        }
        if (valid) {
            gk[e] = k[i];
            gv[e] = v[i];
            if (gs) gs[e] = carry + incl - x;
        }
        carry += shfl_any(incl, 31);
    }
}

// A group of G (2 or 4) warps sorts (stable LSD, 8-bit digits) and scans a segment of
// len <= 32 * G * ITEMS keys: the segment is cut into G consecutive warp chunks of 32 * IT
// elements (element e = wg*32*IT + i*32 + lane in item i of lane `lane` of the group's warp
// wg, IT = ceil(len / (32 G))); each warp ranks its chunk with ballots and its own 256 digit
// counters, the group scans the counters digit-major / warp-minor (so equal digits keep the
// chunk order), and the keys are scattered to the group's staging slice sk.  The values are
// not held in registers: they move between the group's two value slices va / vb (element e
// read from the current one, written to its new slot in the other).  Only the group's warps
// meet at its named barrier `bar` (1 + group index, 32 * G threads), so the CTA's 8 / G
// groups work on 8 / G segments at once.  s_wsum / s_vpart: one slot per warp of the CTA.
template <class K, class V, bool DESC, int ITEMS>
__device__ inline void seg_group_sort_scan(typename RadixKey<K>::B* gk, V* gv, V* gs, uint32_t len,
                                           typename RadixKey<K>::B* sk, V* va, V* vb, uint32_t* s_whist,
                                           uint32_t* s_wsum, V* s_vpart, uint32_t G, uint32_t bar) {
    // G is a runtime value (2 or 4): one copy of this code serves both group sizes, which
    // keeps the kernel inside its register budget
    typedef typename RadixKey<K>::B KB;
    constexpr int D = RadixKey<K>::DIGITS;
    const uint32_t GT = 32u * G;      // threads of the group
    const uint32_t DPT = 256u / GT;   // digits scanned per thread
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t wg = warp % G, gw0 = warp - wg;  // warp inside the group, the group's first warp
    const uint32_t gt = wg * 32u + lane;             // thread inside the group
    const uint32_t IT = (len + GT - 1u) / GT;        // items in use (group-uniform)
    const uint32_t wbase = wg * 32u * IT;
    const uint32_t wn = len > wbase ? min(len - wbase, 32u * IT) : 0u;  // elements of this warp
    uint32_t* wh = s_whist + warp * 256;
    const uint32_t ltm = lanemask_lt();
    // named barrier of the group (immediate ids, so the kernel reserves barriers 0-4 only)
    auto gsync = [&]() {
        switch (bar) {
            case 1: asm volatile("bar.sync 1, %0;\n" ::"r"(GT) : "memory"); break;
            case 2: asm volatile("bar.sync 2, %0;\n" ::"r"(GT) : "memory"); break;
            case 3: asm volatile("bar.sync 3, %0;\n" ::"r"(GT) : "memory"); break;
            default: asm volatile("bar.sync 4, %0;\n" ::"r"(GT) : "memory"); break;
        }
    };
    KB k[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const uint32_t r = (uint32_t)i * 32u + lane;
        if ((uint32_t)i < IT && r < wn) { k[i] = gk[wbase + r]; va[wbase + r] = gv[wbase + r]; }
        else k[i] = KB(0);
    }
    for (int p = 0; p < D; p++) {
        const uint32_t sel = 0x4440u | (uint32_t)(p & 3);
        const bool hi = p >= 4;
#pragma unroll
        for (int j = 0; j < 8; j++) wh[j * 32 + lane] = 0;
        __syncwarp();
        uint32_t pos[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            pos[i] = 0;
            if ((uint32_t)i >= IT || (uint32_t)i * 32u >= wn) continue;  // warp-uniform
            const bool valid = (uint32_t)i * 32u + lane < wn;
            const uint32_t d = radix_digit_sel<K, DESC>(k[i], sel, hi);
            uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const bool set = (d >> b) & 1u;
                const uint32_t bb = __ballot_sync(0xffffffffu, set);
                peers &= set ? bb : ~bb;
            }
            const uint32_t leader = 31u - __clz(peers | 1u);
            uint32_t base = 0;
            if (valid && lane == leader) base = atomicAdd(&wh[d], (uint32_t)__popc(peers));
            pos[i] = __shfl_sync(0xffffffffu, base, (int)leader) + (uint32_t)__popc(peers & ltm);
        }
        gsync();  // every warp's counters are complete
        // exclusive scan over (digit, warp): thread gt owns digits gt*DPT .. gt*DPT+DPT-1 (the
        // counts are read again below rather than held in registers)
        uint32_t tot = 0;
        for (uint32_t j = 0; j < DPT; j++)
            for (uint32_t w = 0; w < G; w++) tot += s_whist[(gw0 + w) * 256 + gt * DPT + j];
        uint32_t inc = tot;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= (uint32_t)d) inc += y;
        }
        if (lane == 31) s_wsum[warp] = inc;
        gsync();
        uint32_t run = inc - tot;
        for (uint32_t w = 0; w < wg; w++) run += s_wsum[gw0 + w];
        for (uint32_t j = 0; j < DPT; j++)
            for (uint32_t w = 0; w < G; w++) {
                uint32_t* cw = &s_whist[(gw0 + w) * 256 + gt * DPT + j];
                const uint32_t c = *cw;
                *cw = run;
                run += c;
            }
        gsync();  // digit starts of every warp are in place
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t r = (uint32_t)i * 32u + lane;
            if ((uint32_t)i >= IT || r >= wn) continue;
            const uint32_t q = pos[i] + wh[radix_digit_sel<K, DESC>(k[i], sel, hi)];
            sk[q] = k[i];
            vb[q] = va[wbase + r];
        }
        gsync();  // the pass's order is complete in sk / vb
        if (p + 1 < D) {
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const uint32_t r = (uint32_t)i * 32u + lane;
                if ((uint32_t)i < IT && r < wn) k[i] = sk[wbase + r];
            }
        }
        V* t = va; va = vb; vb = t;
        // the next pass writes sk / vb only after its first group barrier, which every warp
        // reaches after this reload
    }
    // exclusive scan of the sorted values (in va; the sorted keys are in sk): warp totals, the
    // group's offsets, then each warp's rows with a running carry; keys, values and scan
    // written in element order
    V wsum = V();
#pragma unroll 1
    for (uint32_t r = lane; r < wn; r += 32u) wsum += va[wbase + r];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) wsum += shfl_xor_any(wsum, d);
    if (lane == 0) s_vpart[warp] = wsum;
    gsync();
    V carry = V();
    for (uint32_t w = 0; w < wg; w++) carry += s_vpart[gw0 + w];
#pragma unroll 1
    for (uint32_t r0 = 0; r0 < wn; r0 += 32u) {  // rows of the warp's chunk (warp-uniform)
        const uint32_t r = r0 + lane;
        const bool valid = r < wn;
        const V x = valid ? va[wbase + r] : V();
        V incl = x;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const V y = shfl_up_any(incl, d);
            if (lane >= (uint32_t)d) incl += y;
        }
        if (valid) {
            gk[wbase + r] = sk[wbase + r];
            gv[wbase + r] = x;
            if (gs) gs[wbase + r] = carry + incl - x;
        }
        carry += shfl_any(incl, 31);
    }
    gsync();  // s_vpart and the staging slices are free for the group's next segment
}

// One warp sorts (and scans) a segment of len <= 32 keys without digit counters: a bitonic
// network over (ordered code, original index) pairs, one per lane.  The index makes every
// pair distinct, so the network's result is the stable order (equal codes keep their input
// order); padding lanes carry the largest code and indices >= len, so they sort last.  Each
// lane then takes its key and value from the lane that held the element (shuffles only: the
// segment may be sorted in place).
template <class K, class V, bool DESC>
__device__ inline void seg_warp_bitonic(typename RadixKey<K>::B* gk, V* gv, V* gs, uint32_t len) {
    typedef typename RadixKey<K>::B KB;
    typedef typename RadixKey<K>::U U;
    const uint32_t lane = threadIdx.x & 31u;
    const bool valid = lane < len;
    const KB key = valid ? gk[lane] : KB(0);
    const V val = valid ? gv[lane] : V();
    U code = ~U(0);
    if (valid) {
        code = RadixKey<K>::ordered(key);
        if (DESC) code = ~code;
    }
    uint32_t idx = lane;
#pragma unroll
    for (uint32_t k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const U oc = __shfl_xor_sync(0xffffffffu, code, (int)j);
            const uint32_t oi = __shfl_xor_sync(0xffffffffu, idx, (int)j);
            const bool other_less = oc < code || (oc == code && oi < idx);
            // blocks of k alternate direction; the lower lane of a pair keeps the smaller
            // element in an ascending block and the larger one in a descending block
            const bool asc = (lane & k) == 0, lower = (lane & j) == 0;
            if ((asc == lower) == other_less) { code = oc; idx = oi; }
        }
    }
    const KB sk = shfl_any(key, (int)idx);
    const V sv = shfl_any(val, (int)idx);
    const V x = valid ? sv : V();
    V incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const V y = shfl_up_any(incl, d);
        if (lane >= (uint32_t)d) incl += y;
    }
    if (valid) {
        gk[lane] = sk;
        gv[lane] = sv;
        if (gs) gs[lane] = incl - x;
    }
}

template <class K, class V, int ITEMS>
constexpr size_t seg_sort_scan_smem() {
    return (size_t)256 * ITEMS * (2 * sizeof(V) + sizeof(typename RadixKey<K>::B)) + 8 * 256 * 4;
}

// One persistent launch over the whole batch.  keys/vals: the concatenated segments (sorted
// in place); scan: receives the exclusive scans; tk/tv: temp arrays of n elements (large
// segments only).
// resident CTAs per SM the batched kernel is compiled for (B200, 100k lognormal segments at 8
// items, u32 keys: 2 CTAs (127 registers) 4.15 ms, 3 CTAs 3.53 ms, 4 CTAs (64 registers) 3.46 ms;
// 16 items need the shared memory of 3 CTAs; 8-byte keys keep 2 CTAs, which they fill without
// spilling)
#ifndef TRTC_SEG_MINB
#define TRTC_SEG_MINB(items, key_bytes) ((key_bytes) > 4 ? 2 : ((items) <= 8 ? 4 : 3))
#endif
// groups of two and four warps for the segments between one warp's share and a quarter of
// the CTA tile (0: those segments take the whole-CTA on-chip class)
#ifndef TRTC_SEG_GROUPS
#define TRTC_SEG_GROUPS 1
#endif
template <class K, class V, class OFF, bool DESC, int ITEMS, int MINB = TRTC_SEG_MINB(ITEMS, sizeof(K))>
__global__ void __launch_bounds__(256, MINB) seg_sort_scan_kernel(typename RadixKey<K>::B* __restrict__ keys,
                                                                V* __restrict__ vals, V* __restrict__ scan,
                                                                typename RadixKey<K>::B* __restrict__ tk,
                                                                V* __restrict__ tv, const OFF* __restrict__ off,
                                                                const uint32_t* __restrict__ queue,
                                                                unsigned long long nseg, SegCtrl* ctrl,
                                                                const SegItem* __restrict__ items,
                                                                uint32_t warp_small) {
    typedef typename RadixKey<K>::B KB;
    constexpr int TILE = 256 * ITEMS;
    constexpr int D = RadixKey<K>::DIGITS;
    extern __shared__ __align__(16) unsigned char seg_smem[];  // seg_sort_scan_smem<K, V, ITEMS>() bytes
    V* s_v = reinterpret_cast<V*>(seg_smem);
    V* s_o = s_v + TILE;
    KB* s_k = reinterpret_cast<KB*>(s_o + TILE);
    uint32_t* s_whist = reinterpret_cast<uint32_t*>(s_k + TILE);
    __shared__ uint32_t s_cnt[256], s_start[256], s_run[256];
    __shared__ uint32_t s_hist[D][256];
    __shared__ uint32_t s_wsum[8];
    __shared__ V s_part[8];
    __shared__ unsigned long long s_item;
    __shared__ unsigned long long s_batch, s_defer[8];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    constexpr uint32_t WSEG = 32u * ITEMS;  // segments up to this length are sorted by one warp

    // the arrays and length of queue entry `item`
    auto fetch = [&](unsigned long long item, KB*& gk, V*& gv, V*& gs, uint32_t& len, unsigned long long& base) {
        if (items) {  // list mode: segments in queue order, each with its own arrays
            const SegItem it = items[item];
            gk = reinterpret_cast<KB*>(it.k);
            gv = reinterpret_cast<V*>(it.v);
            gs = reinterpret_cast<V*>(it.out);
            len = (uint32_t)it.n;
            base = it.toff;
        } else {
            const uint32_t sid = queue[item];
            base = (unsigned long long)off[sid];
            len = (uint32_t)((unsigned long long)off[sid + 1] - base);
            gk = keys + base;
            gv = vals + base;
            gs = scan + base;
        }
    };

    // whole-CTA sort + scan of one segment (on chip up to TILE keys, else through global memory)
    auto block_segment = [&](KB* gk, V* gv, V* gs, uint32_t len, unsigned long long base) {
        if (len <= (uint32_t)TILE) {
            // ---------------- on-chip sort of a small segment
            const int IT = (int)((len + 255u) / 256u);
            const uint32_t wbase = warp * 32u * (uint32_t)IT;
            KB k[ITEMS];
            V v[ITEMS];
            uint32_t pos[ITEMS];
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const uint32_t e = wbase + (uint32_t)i * 32u + lane;
                if (i < IT && e < len) { k[i] = gk[e]; v[i] = gv[e]; }
                else { k[i] = KB(0); v[i] = V(); }
            }
            for (int p = 0; p < D; p++) {
                const uint32_t sel = 0x4440u | (uint32_t)(p & 3);
                seg_rank_tile<K, DESC, ITEMS>(k, pos, IT, len, sel, p >= 4, s_whist, s_cnt, s_start, s_wsum);
#pragma unroll
                for (int i = 0; i < ITEMS; i++) {
                    const uint32_t e = wbase + (uint32_t)i * 32u + lane;
                    if (i < IT && e < len) { s_k[pos[i]] = k[i]; s_v[pos[i]] = v[i]; }
                }
                __syncthreads();
                if (p + 1 < D) {
#pragma unroll
                    for (int i = 0; i < ITEMS; i++) {
                        const uint32_t e = wbase + (uint32_t)i * 32u + lane;
                        if (i < IT && e < len) { k[i] = s_k[e]; v[i] = s_v[e]; }
                    }
                }
                __syncthreads();
            }
            // s_k / s_v hold the sorted segment; exclusive scan of the values into s_o
            if (gs) seg_block_excl_scan<V, ITEMS>(s_v, s_o, len, V(), s_part);
            for (uint32_t e = threadIdx.x; e < len; e += 256) {
                gk[e] = s_k[e];
                gv[e] = s_v[e];
                if (gs) gs[e] = s_o[e];
            }
            return;
        }

        // ---------------- large segment: CTA-level LSD passes through global memory
        for (int i = threadIdx.x; i < D * 256; i += 256) (&s_hist[0][0])[i] = 0;
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < len; e += 256) {
            typename RadixKey<K>::U u = RadixKey<K>::ordered(gk[e]);
            if (DESC) u = ~u;
#pragma unroll
            for (int p = 0; p < D; p++) {
                const uint32_t w = (p < 4) ? (uint32_t)u : (uint32_t)((unsigned long long)u >> 32);
                atomicAdd(&s_hist[p][__byte_perm(w, 0u, 0x4440u | (uint32_t)(p & 3))], 1u);
            }
        }
        __syncthreads();
        KB* sk = gk;
        V* sv = gv;
        KB* dk = tk + base;
        V* dv = tv + base;
        for (int p = 0; p < D; p++) {
            const uint32_t sel = 0x4440u | (uint32_t)(p & 3);
            const bool hi = p >= 4;
            {
                const uint32_t c = s_hist[p][threadIdx.x];
                s_run[threadIdx.x] = block_excl_scan_256<256>(c, s_wsum);
            }
            __syncthreads();
            for (uint32_t cb = 0; cb < len; cb += TILE) {
                const uint32_t cn = min((uint32_t)TILE, len - cb);
                const uint32_t wbase = warp * 32u * ITEMS;
                KB k[ITEMS];
                V v[ITEMS];
                uint32_t pos[ITEMS];
#pragma unroll
                for (int i = 0; i < ITEMS; i++) {
                    const uint32_t e = wbase + (uint32_t)i * 32u + lane;
                    if (e < cn) { k[i] = sk[cb + e]; v[i] = sv[cb + e]; }
                    else { k[i] = KB(0); v[i] = V(); }
                }
                seg_rank_tile<K, DESC, ITEMS>(k, pos, ITEMS, cn, sel, hi, s_whist, s_cnt, s_start, s_wsum);
#pragma unroll
                for (int i = 0; i < ITEMS; i++) {
                    const uint32_t e = wbase + (uint32_t)i * 32u + lane;
                    if (e < cn) { s_k[pos[i]] = k[i]; s_v[pos[i]] = v[i]; }
                }
                __syncthreads();
                for (uint32_t e = threadIdx.x; e < cn; e += 256) {
                    const KB key = s_k[e];
                    const uint32_t d = radix_digit_sel<K, DESC>(key, sel, hi);
                    const uint32_t dst = s_run[d] + (e - s_start[d]);
                    dk[dst] = key;
                    dv[dst] = s_v[e];
                }
                __syncthreads();
                s_run[threadIdx.x] += s_cnt[threadIdx.x];
                __syncthreads();
            }
            KB* t1 = sk; sk = dk; dk = t1;
            V* t2 = sv; sv = dv; dv = t2;
        }
        // after D passes the segment is in sk/sv (the caller's arrays when D is even);
        // chunked exclusive scan with a running carry, writing keys and values back if needed
        V carry = V();
        for (uint32_t cb = 0; cb < len; cb += TILE) {
            const uint32_t cn = min((uint32_t)TILE, len - cb);
            for (uint32_t e = threadIdx.x; e < cn; e += 256) {
                s_v[e] = sv[cb + e];
                if (sk != gk) { gk[cb + e] = sk[cb + e]; gv[cb + e] = s_v[e]; }
            }
            __syncthreads();
            if (gs) {
                carry = seg_block_excl_scan<V, ITEMS>(s_v, s_o, cn, carry, s_part);
                for (uint32_t e = threadIdx.x; e < cn; e += 256) gs[cb + e] = s_o[e];
            }
            __syncthreads();
        }
    };

    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(&ctrl->next, 1ull);
        __syncthreads();
        const unsigned long long item = s_item;
        if (item >= nseg) return;
        KB* gk;
        V* gv;
        V* gs;
        uint32_t len;
        unsigned long long base;
        fetch(item, gk, gv, gs, len, base);
        if (len == 0) continue;
        if (len > (TRTC_SEG_GROUPS ? 4u : 1u) * WSEG) {
            block_segment(gk, gv, gs, len, base);
            continue;
        }
        // a small segment: the queue lists the classes from the largest down, so the entries
        // after it are no longer than its class.  The CTA splits into groups of G warps (one
        // warp up to WSEG keys, two up to 2 WSEG, four up to 4 WSEG), takes one more entry per
        // further group, and every group sorts one; an entry longer than its group's share
        // (list mode keeps the caller's order) is deferred to the whole CTA afterwards
        const uint32_t G = !TRTC_SEG_GROUPS ? 1u : len > 2u * WSEG ? 4u : (len > WSEG ? 2u : 1u);  // CTA-uniform
        if (threadIdx.x == 0) s_batch = atomicAdd(&ctrl->next, (unsigned long long)(8u / G - 1u));
        __syncthreads();
        const uint32_t grp = warp / G;
        const unsigned long long mine = grp == 0 ? item : s_batch + grp - 1;
        unsigned long long defer = ~0ull;
        if (mine < nseg) {
            KB* wk;
            V* wv;
            V* ws;
            uint32_t wl;
            unsigned long long wb;
            fetch(mine, wk, wv, ws, wl, wb);
            if (wl > G * WSEG) defer = mine;
            else if (wl > 0 && G == 1 && wl <= warp_small) seg_warp_bitonic<K, V, DESC>(wk, wv, ws, wl);
            else if (wl > 0 && G == 1)
                seg_warp_sort_scan<K, V, DESC, ITEMS>(wk, wv, ws, wl, s_k + warp * WSEG, s_v + warp * WSEG,
                                                      s_whist + warp * 256);
            else if (wl > 0)
                seg_group_sort_scan<K, V, DESC, ITEMS>(wk, wv, ws, wl, s_k + grp * G * WSEG, s_v + grp * G * WSEG,
                                                       s_o + grp * G * WSEG, s_whist, s_wsum, s_part, G, 1u + grp);
        }
        if (lane == 0) s_defer[warp] = (warp % G == 0) ? defer : ~0ull;
        __syncthreads();
        for (int w = 0; w < 8; w++) {
            const unsigned long long d = s_defer[w];
            if (d == ~0ull) continue;
            fetch(d, gk, gv, gs, len, base);
            block_segment(gk, gv, gs, len, base);
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------ NaN rotation (float keys)
// The reference sorts a float vector by (code(x) - code(m)) mod 2^w, m the element that its
// Min_Element tree selects (extrema.cpp:5-13 over internal/general_reduce.cpp:55-95).  With a
// NaN in a left slot the tree can select a non-minimum, and the sorted order is the code order
// rotated so that the keys ordered at or above m come first.  A segment sorted on its own gets
// the same rotation here: seg_rot_kernel (before the sort) replays the tree on every segment
// that holds a NaN and counts its keys ordered strictly below the selected one;
// seg_rotate_kernel (after the sort) rotates those segments by that count and redoes their
// exclusive scans.  Segments without a NaN are only read once, for the NaN test.
template <class K> struct SegMinSlot {
    K v;
    unsigned long long i;
};

// tree slots of a segment starting at element `base` (index `sid`): the rounds need at most
// ceil(L/256) + ceil(L/2^16) + ceil(L/2^24) + 1 slots, which fit between base/128 + 4*sid and
// the next segment's start; the whole area holds n/128 + 4*nseg + 4 slots
TRTC_FORCEINLINE unsigned long long seg_tree_base(unsigned long long base, unsigned long long sid) {
    return base / 128ull + 4ull * sid;
}
inline unsigned long long seg_tree_slots(unsigned long long n, unsigned long long nseg) {
    return n / 128ull + 4ull * nseg + 4ull;
}

template <class K, class OFF>
__global__ void __launch_bounds__(256) seg_rot_kernel(const typename RadixKey<K>::B* __restrict__ keys,
                                                      const OFF* __restrict__ off,
                                                      const SegItem* __restrict__ items, unsigned long long nseg,
                                                      SegMinSlot<K>* tree, uint32_t* __restrict__ rot) {
    typedef RadixKey<K> RK;
    typedef typename RK::B KB;
    __shared__ unsigned long long s_c[8];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (unsigned long long sid = blockIdx.x; sid < nseg; sid += gridDim.x) {
        const KB* gk;
        uint32_t len;
        unsigned long long base;
        if (items) {
            const SegItem it = items[sid];
            gk = reinterpret_cast<const KB*>(it.k);
            len = (uint32_t)it.n;
            base = it.toff;
        } else {
            base = (unsigned long long)off[sid];
            len = (uint32_t)((unsigned long long)off[sid + 1] - base);
            gk = keys + base;
        }
        bool nan = false;
        for (uint32_t e = threadIdx.x; e < len; e += 256) nan |= RK::is_nan(gk[e]);
        if (!__syncthreads_or(nan)) {
            if (threadIdx.x == 0) rot[sid] = 0;
            continue;
        }
        // round 1 over 256-blocks of the keys, then rounds over the block results (slots in
        // global memory, written and read by this CTA only, ordered by its barriers)
        SegMinSlot<K>* src = tree + seg_tree_base(base, sid);
        uint32_t m = (len + 255u) / 256u;
        for (uint32_t b = warp; b < m; b += 8) {
            const uint32_t L = min(256u, len - b * 256u);
            K rv;
            unsigned long long ri;
            min_tree_warp256<K>(
                [&](uint32_t t, K& v, unsigned long long& i) { v = RK::value(gk[b * 256u + t]); i = b * 256u + t; },
                L, rv, ri);
            if (lane == 0) { src[b].v = rv; src[b].i = ri; }
        }
        __syncthreads();
        while (m > 1) {
            SegMinSlot<K>* dst = src + m;
            const uint32_t nb = (m + 255u) / 256u;
            for (uint32_t b = warp; b < nb; b += 8) {
                const uint32_t L = min(256u, m - b * 256u);
                K rv;
                unsigned long long ri;
                min_tree_warp256<K>(
                    [&](uint32_t t, K& v, unsigned long long& i) { v = src[b * 256u + t].v; i = src[b * 256u + t].i; },
                    L, rv, ri);
                if (lane == 0) { dst[b].v = rv; dst[b].i = ri; }
            }
            __syncthreads();
            src = dst;
            m = nb;
        }
        const typename RK::U tm = RK::ordered(gk[src[0].i]);
        unsigned long long c = 0;
        for (uint32_t e = threadIdx.x; e < len; e += 256) c += RK::ordered(gk[e]) < tm ? 1ull : 0ull;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
        if (lane == 0) s_c[warp] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long t = 0;
            for (int w = 0; w < 8; w++) t += s_c[w];
            rot[sid] = (uint32_t)t;
        }
        __syncthreads();
    }
}

template <class K, class V, class OFF, bool DESC>
__global__ void __launch_bounds__(256) seg_rotate_kernel(typename RadixKey<K>::B* __restrict__ keys,
                                                         V* __restrict__ vals, V* __restrict__ scan,
                                                         typename RadixKey<K>::B* __restrict__ tk,
                                                         V* __restrict__ tv, const OFF* __restrict__ off,
                                                         const SegItem* __restrict__ items, unsigned long long nseg,
                                                         const uint32_t* __restrict__ rot) {
    typedef typename RadixKey<K>::B KB;
    constexpr int CH = 1024;
    __shared__ V s_v[CH], s_o[CH], s_part[8];
    for (unsigned long long sid = blockIdx.x; sid < nseg; sid += gridDim.x) {
        const uint32_t r = rot[sid];
        if (r == 0) continue;
        KB* gk;
        V *gv, *gs;
        uint32_t len;
        unsigned long long base;
        if (items) {
            const SegItem it = items[sid];
            gk = reinterpret_cast<KB*>(it.k);
            gv = reinterpret_cast<V*>(it.v);
            gs = reinterpret_cast<V*>(it.out);
            len = (uint32_t)it.n;
            base = it.toff;
        } else {
            base = (unsigned long long)off[sid];
            len = (uint32_t)((unsigned long long)off[sid + 1] - base);
            gk = keys + base;
            gv = vals + base;
            gs = scan + base;
        }
        for (uint32_t e = threadIdx.x; e < len; e += 256) { tk[base + e] = gk[e]; tv[base + e] = gv[e]; }
        __syncthreads();
        // ascending: sorted position p moves to p - r (mod len); descending: to p + r
        for (uint32_t e = threadIdx.x; e < len; e += 256) {
            uint32_t d = DESC ? e + r : e + (len - r);
            if (d >= len) d -= len;
            gk[d] = tk[base + e];
            gv[d] = tv[base + e];
        }
        __syncthreads();
        if (gs) {
            V carry = V();
            for (uint32_t cb = 0; cb < len; cb += CH) {
                const uint32_t cn = min((uint32_t)CH, len - cb);
                for (uint32_t e = threadIdx.x; e < cn; e += 256) s_v[e] = gv[cb + e];
                __syncthreads();
                carry = seg_block_excl_scan<V, CH / 256>(s_v, s_o, cn, carry, s_part);
                for (uint32_t e = threadIdx.x; e < cn; e += 256) gs[cb + e] = s_o[e];
                __syncthreads();
            }
        }
    }
}

// Exclusive Plus scans of many segments (list mode): a persistent CTA takes one segment at
// a time and scans it in chunks of 256 * ITEMS with a running carry.
template <class T, int ITEMS>
__global__ void __launch_bounds__(256) seg_scan_list_kernel(const SegItem* __restrict__ items, unsigned long long nseg,
                                                            SegCtrl* ctrl) {
    constexpr int TILE = 256 * ITEMS;
    __shared__ __align__(16) T s_v[TILE];
    __shared__ __align__(16) T s_o[TILE];
    __shared__ T s_part[8];
    __shared__ unsigned long long s_item;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(&ctrl->next, 1ull);
        __syncthreads();
        const unsigned long long item = s_item;
        if (item >= nseg) return;
        const SegItem it = items[item];
        const T* in = reinterpret_cast<const T*>(it.k);
        T* out = reinterpret_cast<T*>(it.out);
        T carry = T();
        for (unsigned long long cb = 0; cb < it.n; cb += TILE) {
            const uint32_t cn = (uint32_t)min((unsigned long long)TILE, it.n - cb);
            for (uint32_t e = threadIdx.x; e < cn; e += 256) s_v[e] = in[cb + e];
            __syncthreads();
            carry = seg_block_excl_scan<T, ITEMS>(s_v, s_o, cn, carry, s_part);
            for (uint32_t e = threadIdx.x; e < cn; e += 256) out[cb + e] = s_o[e];
            __syncthreads();
        }
    }
}

// Plus reductions of many segments (list mode); the result of segment i goes to
// *(T*)items[i].out.
template <class T>
__global__ void __launch_bounds__(256) seg_reduce_list_kernel(const SegItem* __restrict__ items, unsigned long long nseg,
                                                              SegCtrl* ctrl) {
    __shared__ T s_w[8];
    __shared__ unsigned long long s_item;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(&ctrl->next, 1ull);
        __syncthreads();
        const unsigned long long item = s_item;
        if (item >= nseg) return;
        const SegItem it = items[item];
        const T* in = reinterpret_cast<const T*>(it.k);
        T a = T();
        for (unsigned long long e = threadIdx.x; e < it.n; e += 256) a += in[e];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) a += shfl_down_any(a, d);
        if ((threadIdx.x & 31u) == 0) s_w[threadIdx.x >> 5] = a;
        __syncthreads();
        if (threadIdx.x == 0) {
            T t = s_w[0];
            for (int w = 1; w < 8; w++) t += s_w[w];
            *reinterpret_cast<T*>(it.out) = t;
        }
    }
}

}  // namespace trtc
