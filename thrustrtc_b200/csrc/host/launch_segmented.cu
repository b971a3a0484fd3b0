// launch_segmented.cu -- batched segmented sort + exclusive scan (one persistent launch over
// all segments, fed by a device work queue), its workspace sizing, and the autotuner that
// picks the tile configuration per key type from timed trial runs.
#include <map>
#include <mutex>
#include <vector>

#include "../device/trtc_segmented.cuh"
#include "trtc_launch.h"
#include "trtc_runtime.h"

namespace trtc_host {

using namespace trtc;

namespace {

constexpr int SEG_CONFIGS[] = {8, 16};  // items per thread: small-class limit 2048 or 4096 keys
std::mutex g_seg_mu;
std::map<int, int> g_seg_items;  // key type -> tuned items per thread

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

template <class K> constexpr bool is_float_key() { return is_same<K, float>::value || is_same<K, double>::value; }

// control block, queue, temp keys, temp values; float keys add the NaN-rotation counts and
// the Min_Element tree slots (seg_rot_kernel)
template <class K>
size_t ws_bytes(size_t n, size_t nseg) {
    size_t b = align256(sizeof(SegCtrl)) + align256(nseg * 4) + align256(n * sizeof(typename RadixKey<K>::B)) +
               align256(n * 4);
    if (is_float_key<K>()) b += align256(nseg * 4) + align256(seg_tree_slots(n, nseg) * sizeof(SegMinSlot<K>));
    return b;
}

template <class K, bool DESC, int ITEMS>
bool seg_run_cfg(void* keys, void* vals, void* scan, const unsigned long long* off, size_t nseg, size_t n, void* ws,
                 cudaStream_t s) {
    typedef typename RadixKey<K>::B KB;
    typedef uint32_t V;
    unsigned char* p = (unsigned char*)ws;
    SegCtrl* ctrl = (SegCtrl*)p;
    p += align256(sizeof(SegCtrl));
    uint32_t* queue = (uint32_t*)p;
    p += align256(nseg * 4);
    KB* tk = (KB*)p;
    p += align256(n * sizeof(KB));
    V* tv = (V*)p;
    p += align256(n * 4);
    uint32_t* rot = (uint32_t*)p;  // float keys only
    p += align256(nseg * 4);
    SegMinSlot<K>* tree = (SegMinSlot<K>*)p;
    if (!TRTC_CUDA(cudaMemsetAsync(ctrl, 0, sizeof(SegCtrl), s))) return false;
    const int sms = sm_count();
    const unsigned rgrid = (unsigned)(nseg < (size_t)sms * 8 ? nseg : (size_t)sms * 8);
    if constexpr (is_float_key<K>()) {
        // the reference's per-segment NaN rotation, counted on the unsorted keys
        ktimer_mark("", s);
        seg_rot_kernel<K, unsigned long long><<<rgrid, 256, 0, s>>>((const KB*)keys, off, nullptr, nseg, tree, rot);
        count_launch();
        ktimer_mark("seg_rot_kernel", s);
    }
    size_t qg = (nseg + 255) / 256;
    if (qg > (size_t)sms * 4) qg = (size_t)sms * 4;
    if (qg < 1) qg = 1;
    ktimer_mark("", s);
    seg_queue_kernel<unsigned long long><<<(unsigned)qg, 256, 0, s>>>(off, nseg, 256ull * ITEMS, queue, ctrl);
    ktimer_mark("seg_queue_kernel", s);
    constexpr size_t smem = seg_sort_scan_smem<K, V, ITEMS>();
    auto kernel = seg_sort_scan_kernel<K, V, unsigned long long, DESC, ITEMS>;
    static int per_sm = 0;
    if (per_sm == 0) {
        if (!TRTC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
            return false;
        if (!TRTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem))) return false;
        if (per_sm < 1) per_sm = 1;
    }
    size_t grid = (size_t)per_sm * sms;
    if (grid > nseg) grid = nseg;
    kernel<<<(unsigned)grid, 256, smem, s>>>((KB*)keys, (V*)vals, (V*)scan, tk, tv, off, queue, nseg, ctrl, nullptr);
    ktimer_mark("seg_sort_scan_kernel", s);
    count_launch(2);
    if constexpr (is_float_key<K>()) {
        seg_rotate_kernel<K, V, unsigned long long, DESC><<<rgrid, 256, 0, s>>>((KB*)keys, (V*)vals, (V*)scan, tk, tv,
                                                                             off, nullptr, nseg, rot);
        count_launch();
        ktimer_mark("seg_rotate_kernel", s);
    }
    return TRTC_CUDA(cudaGetLastError());
}

template <class K, bool DESC>
bool seg_run(int items, void* keys, void* vals, void* scan, const unsigned long long* off, size_t nseg, size_t n,
             void* ws, cudaStream_t s) {
    if (items == 16) return seg_run_cfg<K, DESC, 16>(keys, vals, scan, off, nseg, n, ws, s);
    return seg_run_cfg<K, DESC, 8>(keys, vals, scan, off, nseg, n, ws, s);
}

template <class K>
bool seg_dispatch_desc(int items, bool desc, void* keys, void* vals, void* scan, const unsigned long long* off,
                       size_t nseg, size_t n, void* ws, cudaStream_t s) {
    return desc ? seg_run<K, true>(items, keys, vals, scan, off, nseg, n, ws, s)
                : seg_run<K, false>(items, keys, vals, scan, off, nseg, n, ws, s);
}

bool seg_dispatch(int tc, int items, bool desc, void* keys, void* vals, void* scan, const unsigned long long* off,
                  size_t nseg, size_t n, void* ws, cudaStream_t s) {
    switch (tc) {
        case TC_U32: return seg_dispatch_desc<uint32_t>(items, desc, keys, vals, scan, off, nseg, n, ws, s);
        case TC_I32: return seg_dispatch_desc<int32_t>(items, desc, keys, vals, scan, off, nseg, n, ws, s);
        case TC_F32: return seg_dispatch_desc<float>(items, desc, keys, vals, scan, off, nseg, n, ws, s);
        case TC_U64: return seg_dispatch_desc<uint64_t>(items, desc, keys, vals, scan, off, nseg, n, ws, s);
        case TC_I64: return seg_dispatch_desc<int64_t>(items, desc, keys, vals, scan, off, nseg, n, ws, s);
        default: set_error("segmented_sort_scan: key type must be int32, uint32, float, int64 or uint64"); return false;
    }
}

__global__ void seg_fill_kernel(uint32_t* k, uint32_t* v, size_t words, unsigned long long seed) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x) {
        unsigned long long z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        k[i] = (uint32_t)z;
        if (v) v[i] = (uint32_t)(z >> 32);
    }
}

}  // namespace

size_t segmented_workspace_bytes(int tc, size_t n, size_t nseg) {
    if (tc == TC_F32) return ws_bytes<float>(n, nseg);
    return (tc == TC_U64 || tc == TC_I64) ? ws_bytes<uint64_t>(n, nseg) : ws_bytes<uint32_t>(n, nseg);
}

int segmented_tuned_items(int tc) {
    std::lock_guard<std::mutex> lk(g_seg_mu);
    auto it = g_seg_items.find(tc);
    return it == g_seg_items.end() ? 16 : it->second;
}

bool segmented_sort_scan_raw(int tc, void* keys, void* vals, void* scan, const unsigned long long* off, size_t nseg,
                             size_t n, void* ws, size_t ws_bytes_given, bool desc, cudaStream_t s) {
    if (nseg == 0 || n == 0) return true;
    if (nseg >= (1ull << 32)) { set_error("segmented_sort_scan: at most 2^32 - 1 segments"); return false; }
    if (n >= (1ull << 32)) { set_error("segmented_sort_scan: at most 2^32 - 1 elements"); return false; }
    if (ws_bytes_given < segmented_workspace_bytes(tc, n, nseg)) {
        set_error("segmented_sort_scan: workspace too small (see trtc_raw_segmented_workspace_bytes)");
        return false;
    }
    return seg_dispatch(tc, segmented_tuned_items(tc), desc, keys, vals, scan, off, nseg, n, ws, s);
}

// Times every configuration on a copy of the batch shape (random keys, the caller's segment
// offsets) and keeps the fastest for this key type.  Allocates its own scratch.
bool segmented_autotune(int tc, const unsigned long long* off, size_t nseg, size_t n, cudaStream_t s, int* chosen) {
    if (!ensure_device()) return false;
    if (nseg == 0 || n == 0) { *chosen = segmented_tuned_items(tc); return true; }
    const size_t ksz = (tc == TC_U64 || tc == TC_I64) ? 8 : 4;
    const size_t wsb = segmented_workspace_bytes(tc, n, nseg);
    void *k = nullptr, *v = nullptr, *sc = nullptr, *ws = nullptr;
    bool ok = TRTC_CUDA(cudaMalloc(&k, n * ksz)) && TRTC_CUDA(cudaMalloc(&v, n * 4)) &&
              TRTC_CUDA(cudaMalloc(&sc, n * 4)) && TRTC_CUDA(cudaMalloc(&ws, wsb));
    cudaEvent_t a = nullptr, b = nullptr;
    ok = ok && TRTC_CUDA(cudaEventCreate(&a)) && TRTC_CUDA(cudaEventCreate(&b));
    int best = 16;
    float best_ms = 1e30f;
    for (int cfg : SEG_CONFIGS) {
        if (!ok) break;
        float tot = 0.f;
        for (int rep = 0; ok && rep < 4; rep++) {
            seg_fill_kernel<<<sm_count() * 4, 256, 0, s>>>((uint32_t*)k, (uint32_t*)v, n * ksz / 4, 1234 + rep);
            ok = TRTC_CUDA(cudaEventRecord(a, s)) &&
                 seg_dispatch(tc, cfg, false, k, v, sc, off, nseg, n, ws, s) && TRTC_CUDA(cudaEventRecord(b, s)) &&
                 TRTC_CUDA(cudaEventSynchronize(b)) && check_device_errors(s, "segmented autotune");
            float ms = 0.f;
            if (ok && rep > 0 && TRTC_CUDA(cudaEventElapsedTime(&ms, a, b))) tot += ms;
        }
        if (ok && tot < best_ms) { best_ms = tot; best = cfg; }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(k); cudaFree(v); cudaFree(sc); cudaFree(ws);
    if (!ok) return false;
    {
        std::lock_guard<std::mutex> lk(g_seg_mu);
        g_seg_items[tc] = best;
    }
    *chosen = best;
    return true;
}

}  // namespace trtc_host
