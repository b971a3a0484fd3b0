// launch_sort_impl.cuh -- host driver of the onesweep radix sort (nvcc instantiations).
#pragma once
#include <map>
#include <mutex>
#include "trtc_runtime.h"
#include "../device/trtc_radix.cuh"

namespace trtc_host {

// items per thread of a digit pass (tile = 256 * ITEMS keys), from sweeps on B200: 2^28 u32
// pairs 6.13 ms at 20 (4 CTAs/SM), 6.16 ms at 24 (3 CTAs/SM); 2^24 i64 keys + u32 values
// 1.48 ms at 8, 1.33 at 10, 1.18 at 12 (4 CTAs/SM), 1.18 at 16 (3 CTAs/SM, spills)
#ifndef TRTC_RADIX_ITEMS32
#define TRTC_RADIX_ITEMS32 20
#endif
#ifndef TRTC_RADIX_SMALL_N
#define TRTC_RADIX_SMALL_N (1ull << 18)  // up to this many keys, 4-byte keys use 8-item tiles
#endif
#ifndef TRTC_RADIX_ITEMS64
#define TRTC_RADIX_ITEMS64 12
#endif
template <class K> struct SortTuning { enum { ITEMS = sizeof(K) >= 8 ? TRTC_RADIX_ITEMS64 : TRTC_RADIX_ITEMS32 }; };

// Opts a kernel in to `bytes` of dynamic shared memory (needed as soon as static +
// dynamic exceeds 48 KB).  Tracked per kernel address: many instantiations share one type.
template <class F>
static void set_smem_attr_once(F* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<const void*, size_t> done;
    std::lock_guard<std::mutex> lk(mu);
    size_t& d = done[(const void*)kernel];
    if (bytes > d) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        d = bytes;
    }
}

// Runs the whole sort on stream s.  vals0 may be null (keys only).  vals_from_index: the
// payload is the element index (vals0 then receives the sorting permutation).
template <class K, class V, bool HAS_VALS, bool DESC, class ST, int ITEMS = SortTuning<K>::ITEMS>
static bool radix_sort_run(K* keys, V* vals0, size_t n, cudaStream_t s, int vals_from_index) {
    using namespace trtc;
    constexpr int BLOCK = 256;
    constexpr int TILE = BLOCK * ITEMS;
    constexpr int D = RadixKey<K>::DIGITS;
    constexpr bool FLOATKEY = is_same<K, float>::value || is_same<K, double>::value;
    typedef typename RadixKey<K>::B KB;
    const size_t tiles = (n + TILE - 1) / TILE;
    SortCtrl* ctrl = (SortCtrl*)sort_ctrl_ws(s, sizeof(SortCtrl));
    if (!ctrl) return false;
    const size_t status_bytes = ((tiles * 256 * sizeof(ST)) + 15) & ~(size_t)15;
    void* st0 = tmp_alloc(status_bytes, s);
    void* st1 = tmp_alloc(status_bytes, s);
    K* ka = (K*)tmp_alloc(n * sizeof(K), s);
    K* kb = D >= 3 ? (K*)tmp_alloc(n * sizeof(K), s) : nullptr;
    V* va = HAS_VALS ? (V*)tmp_alloc(n * sizeof(V), s) : nullptr;
    V* vb = (HAS_VALS && D >= 3) ? (V*)tmp_alloc(n * sizeof(V), s) : nullptr;
    bool ok = st0 && st1 && ka && (D < 3 || kb) && (!HAS_VALS || (va && (D < 3 || vb)));
    K* tv[2] = {nullptr, nullptr};
    unsigned long long* ti[2] = {nullptr, nullptr};
    const size_t nb1 = (n + 255) / 256;
    if (ok && FLOATKEY) {
        for (int i = 0; i < 2; i++) {
            tv[i] = (K*)tmp_alloc(nb1 * sizeof(K), s);
            ti[i] = (unsigned long long*)tmp_alloc(nb1 * 8, s);
            ok = ok && tv[i] && ti[i];
        }
    }
    if (ok) {
        SortBufs bufs;
        bufs.keys[0] = keys; bufs.keys[1] = ka; bufs.keys[2] = kb;
        bufs.vals[0] = vals0; bufs.vals[1] = va; bufs.vals[2] = vb;
        bufs.err = device_error_word();
        cudaMemsetAsync(ctrl, 0, sizeof(SortCtrl), s);
        const int sms = sm_count();
        constexpr int HBLOCK = 1024;
        size_t hgrid = (n + HBLOCK * 16 - 1) / (HBLOCK * 16);
        if (hgrid > (size_t)sms) hgrid = (size_t)sms;
        if (hgrid < 1) hgrid = 1;
        const size_t hsmem = (size_t)D * 256 * HistCopies<K>::V * 4;
        auto hist_kernel = radix_hist_kernel<K, DESC, HBLOCK>;
        set_smem_attr_once(hist_kernel, hsmem);
        ktimer_mark("", s);
        hist_kernel<<<(unsigned)hgrid, HBLOCK, hsmem, s>>>((const KB*)keys, n, ctrl, (uint4*)st0, status_bytes / 16);
        ktimer_mark("radix_hist_kernel", s);
        radix_plan_kernel<D><<<1, 256, 0, s>>>(ctrl, n);
        ktimer_mark("radix_plan_kernel", s);
        count_launch(2);
        if (FLOATKEY) {
            // the reference's Min_Element tree; only does work when a NaN was seen
            size_t m = n;
            int cur = 0;
            {
                const size_t nb = (m + 255) / 256;
                size_t g = (nb + 7) / 8;
                if (g > (size_t)sms * 16) g = (size_t)sms * 16;
                min_tree_kernel<K, true, true><<<(unsigned)g, 256, 0, s>>>((const KB*)keys, nullptr, nullptr, m, tv[cur],
                                                                           ti[cur], ctrl);
                count_launch();
                m = nb;
            }
            while (m > 1) {
                const size_t nb = (m + 255) / 256;
                size_t g = (nb + 7) / 8;
                if (g > (size_t)sms * 16) g = (size_t)sms * 16;
                min_tree_kernel<K, false, true><<<(unsigned)g, 256, 0, s>>>(nullptr, tv[cur], ti[cur], m, tv[cur ^ 1],
                                                                             ti[cur ^ 1], ctrl);
                count_launch();
                cur ^= 1;
                m = nb;
            }
            radix_count_below_kernel<K, 256><<<(unsigned)(sms * 8), 256, 0, s>>>((const KB*)keys, n, ti[cur], ctrl);
            count_launch();
            ktimer_mark("radix_nan_rotation", s);
        }
        const size_t smem = (size_t)TILE * sizeof(KB) + (HAS_VALS ? (size_t)TILE * sizeof(V) : 0) + (BLOCK / 32) * 256 * 4 +
                            radix_match_smem<KB, V, HAS_VALS, BLOCK, TILE>();
        auto pass_kernel = radix_pass_kernel<K, V, HAS_VALS, DESC, BLOCK, ITEMS, ST>;
        set_smem_attr_once(pass_kernel, smem);
        // L2 prefetch distance of the pass kernel: 1.5 tiles per SM ahead (B200, 2^28 u32 pairs:
        // 5.739 ms without, 5.585 ms at 222 tiles, within 0.2 % from 148 to 444 tiles, slower
        // again past one wave of resident CTAs as the prefetched tiles crowd L2)
        const uint32_t pf = tile_prefetch_ahead((size_t)sms * 3 / 2);
        for (int p = 0; p < D; p++) {
            pass_kernel<<<(unsigned)tiles, BLOCK, smem, s>>>(bufs, n, ctrl, p, (ST*)st0, (ST*)st1, vals_from_index, pf);
            ktimer_mark("radix_pass_kernel", s);
        }
        count_launch(D);
        size_t cg = (n + 255) / 256;
        if (cg > (size_t)sms * 8) cg = (size_t)sms * 8;
        radix_copyback_kernel<K, V, HAS_VALS><<<(unsigned)cg, 256, 0, s>>>(bufs, n, ctrl);
        count_launch();
        ktimer_mark("radix_copyback_kernel", s);
        ok = TRTC_CUDA(cudaGetLastError());
    }
    for (int i = 0; i < 2; i++) { tmp_free(tv[i], s); tmp_free(ti[i], s); }
    tmp_free(st0, s); tmp_free(st1, s);
    tmp_free(ka, s); tmp_free(kb, s); tmp_free(va, s); tmp_free(vb, s);
    return ok;
}

template <class K, bool DESC>
static bool radix_sort_dispatch(void* keys, void* vals, size_t vsize, size_t n, cudaStream_t s) {
    if (n >= (1ull << 32)) { set_error("sort: more than 2^32-1 keys"); return false; }
    const bool big = n >= (1ull << 30);
    if (big && sizeof(K) < 4) { set_error("sort: more than 2^30 narrow keys"); return false; }
    K* k = (K*)keys;
    // small sorts of 4-byte keys take 8-item tiles: a pass over few tiles is bound by one tile's
    // latency, which shorter ranking loops cut (B200: 2^16 pairs 0.069 -> 0.057 ms, 2^18 0.075 ->
    // 0.067 ms; from 2^20 up the 20-item tiles are faster)
    constexpr int SMALL_ITEMS = sizeof(K) == 4 ? 8 : SortTuning<K>::ITEMS;
    const bool small = n <= TRTC_RADIX_SMALL_N;
#define TRTC_SORT_RUN(V, HV, vp, fi)                                                                         \
    (big ? radix_sort_run<K, V, HV, DESC, typename trtc::conditional<(sizeof(K) >= 4), unsigned long long, uint32_t>::type>( \
               k, (V*)(vp), n, s, fi)                                                                        \
         : small ? radix_sort_run<K, V, HV, DESC, uint32_t, SMALL_ITEMS>(k, (V*)(vp), n, s, fi)             \
                 : radix_sort_run<K, V, HV, DESC, uint32_t>(k, (V*)(vp), n, s, fi))
    if (!vals) return TRTC_SORT_RUN(uint32_t, false, nullptr, 0);
    if (vsize == 4) return TRTC_SORT_RUN(uint32_t, true, vals, 0);
    if (vsize == 8) return TRTC_SORT_RUN(unsigned long long, true, vals, 0);
    // other payload sizes: sort a permutation, then gather
    uint32_t* perm = (uint32_t*)tmp_alloc(n * 4, s);
    unsigned char* tmpv = (unsigned char*)tmp_alloc(n * vsize, s);
    bool ok = perm && tmpv && TRTC_SORT_RUN(uint32_t, true, perm, 1);
    if (ok) {
        trtc::SortCtrl* ctrl = (trtc::SortCtrl*)sort_ctrl_ws(s, sizeof(trtc::SortCtrl));
        size_t g = (n + 255) / 256;
        if (g > (size_t)sm_count() * 8) g = (size_t)sm_count() * 8;
        trtc::radix_gather_bytes_kernel<<<(unsigned)g, 256, 0, s>>>((const unsigned char*)vals, tmpv, perm, n, (int)vsize, ctrl);
        trtc::radix_copy_bytes_gated_kernel<<<(unsigned)g, 256, 0, s>>>(tmpv, (unsigned char*)vals, n * vsize, ctrl);
        count_launch(2);
        ok = TRTC_CUDA(cudaGetLastError());
    }
    tmp_free(perm, s);
    tmp_free(tmpv, s);
    return ok;
#undef TRTC_SORT_RUN
}

// Standalone TRTC_Min_Element (extrema.cpp:5-13): the reference's exact tree order.
template <class K>
static bool min_element_run(const K* keys, size_t n, cudaStream_t s, unsigned long long* out_idx) {
    using namespace trtc;
    const size_t nb1 = (n + 255) / 256;
    K* tv[2];
    unsigned long long* ti[2];
    bool ok = true;
    for (int i = 0; i < 2; i++) {
        tv[i] = (K*)tmp_alloc(nb1 * sizeof(K), s);
        ti[i] = (unsigned long long*)tmp_alloc(nb1 * 8, s);
        ok = ok && tv[i] && ti[i];
    }
    if (ok) {
        const int sms = sm_count();
        size_t m = n;
        int cur = 0;
        bool first = true;
        while (first || m > 1) {
            const size_t nb = (m + 255) / 256;
            size_t g = (nb + 7) / 8;
            if (g > (size_t)sms * 16) g = (size_t)sms * 16;
            if (first)
                min_tree_kernel<K, true, false><<<(unsigned)g, 256, 0, s>>>((const typename RadixKey<K>::B*)keys, nullptr,
                                                                            nullptr, m, tv[0], ti[0], nullptr);
            else {
                min_tree_kernel<K, false, false><<<(unsigned)g, 256, 0, s>>>(nullptr, tv[cur], ti[cur], m, tv[cur ^ 1],
                                                                              ti[cur ^ 1], nullptr);
                cur ^= 1;
            }
            count_launch();
            first = false;
            m = nb;
        }
        ok = TRTC_CUDA(cudaMemcpyAsync(out_idx, ti[cur], 8, cudaMemcpyDeviceToHost, s)) &&
             TRTC_CUDA(cudaStreamSynchronize(s));
    }
    for (int i = 0; i < 2; i++) { tmp_free(tv[i], s); tmp_free(ti[i], s); }
    return ok;
}

}  // namespace trtc_host
