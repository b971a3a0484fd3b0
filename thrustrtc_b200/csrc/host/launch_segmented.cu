// launch_segmented.cu -- batched segmented sort + exclusive scan (one persistent launch over
// all segments, fed by a device work queue), its workspace sizing, and the tuning table of
// size classes: per key type, the items per thread (which sets the class limits: one warp up
// to 32 x ITEMS keys, groups of two / four warps up to 64 / 128 x ITEMS, the CTA on chip up to
// 256 x ITEMS, the CTA through global memory beyond) and the limit of the counter-free warp
// class (0 or 32 keys), picked by an autotuner from timed trial runs on the batch's own segment lengths and
// kept as versioned JSON (compiled-in defaults until a table is loaded or tuned).  The digit
// width is 8 bits in every radix class: on-chip ranking spends one ballot per key bit whatever
// the width, so narrower digits only add scatter passes and wider ones outgrow a warp's
// counters.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../device/trtc_segmented.cuh"
#include "trtc_launch.h"
#include "trtc_runtime.h"

namespace trtc_host {

using namespace trtc;

namespace {

struct SegShape {
    int items;       // items per thread: one warp <= 32 x items, 2 / 4 warps <= 64 / 128 x items, CTA on chip <= 256 x items
    int warp_small;  // counter-free (bitonic) warp class limit: 0 (off) or 32 keys
    float ms;        // trial time that chose it (0: compiled-in default or loaded)
};
constexpr SegShape SEG_DEFAULT = {16, 32, 0.f};
constexpr SegShape SEG_CONFIGS[] = {{8, 0, 0.f}, {8, 32, 0.f}, {16, 0, 0.f}, {16, 32, 0.f}};
constexpr int SEG_TUNING_VERSION = 1;
std::mutex g_seg_mu;
std::map<int, SegShape> g_seg_tuning;  // key type -> tuned shape
bool g_seg_env_loaded = false;

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
                 uint32_t warp_small, cudaStream_t s) {
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
    seg_class_count_kernel<unsigned long long><<<(unsigned)qg, 256, 0, s>>>(off, nseg, (uint32_t)ITEMS, ctrl);
    seg_queue_kernel<unsigned long long><<<(unsigned)qg, 256, 0, s>>>(off, nseg, (uint32_t)ITEMS, queue, ctrl);
    count_launch(2);
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
    kernel<<<(unsigned)grid, 256, smem, s>>>((KB*)keys, (V*)vals, (V*)scan, tk, tv, off, queue, nseg, ctrl, nullptr,
                                             warp_small);
    ktimer_mark("seg_sort_scan_kernel", s);
    count_launch();
    if constexpr (is_float_key<K>()) {
        seg_rotate_kernel<K, V, unsigned long long, DESC><<<rgrid, 256, 0, s>>>((KB*)keys, (V*)vals, (V*)scan, tk, tv,
                                                                             off, nullptr, nseg, rot);
        count_launch();
        ktimer_mark("seg_rotate_kernel", s);
    }
    return TRTC_CUDA(cudaGetLastError());
}

template <class K, bool DESC>
bool seg_run(const SegShape& sh, void* keys, void* vals, void* scan, const unsigned long long* off, size_t nseg,
             size_t n, void* ws, cudaStream_t s) {
    const uint32_t ws_small = (uint32_t)sh.warp_small;
    if (sh.items == 16) return seg_run_cfg<K, DESC, 16>(keys, vals, scan, off, nseg, n, ws, ws_small, s);
    return seg_run_cfg<K, DESC, 8>(keys, vals, scan, off, nseg, n, ws, ws_small, s);
}

template <class K>
bool seg_dispatch_desc(const SegShape& sh, bool desc, void* keys, void* vals, void* scan,
                       const unsigned long long* off, size_t nseg, size_t n, void* ws, cudaStream_t s) {
    return desc ? seg_run<K, true>(sh, keys, vals, scan, off, nseg, n, ws, s)
                : seg_run<K, false>(sh, keys, vals, scan, off, nseg, n, ws, s);
}

bool seg_dispatch(int tc, const SegShape& sh, bool desc, void* keys, void* vals, void* scan,
                  const unsigned long long* off, size_t nseg, size_t n, void* ws, cudaStream_t s) {
    switch (tc) {
        case TC_U32: return seg_dispatch_desc<uint32_t>(sh, desc, keys, vals, scan, off, nseg, n, ws, s);
        case TC_I32: return seg_dispatch_desc<int32_t>(sh, desc, keys, vals, scan, off, nseg, n, ws, s);
        case TC_F32: return seg_dispatch_desc<float>(sh, desc, keys, vals, scan, off, nseg, n, ws, s);
        case TC_U64: return seg_dispatch_desc<uint64_t>(sh, desc, keys, vals, scan, off, nseg, n, ws, s);
        case TC_I64: return seg_dispatch_desc<int64_t>(sh, desc, keys, vals, scan, off, nseg, n, ws, s);
        default: set_error("segmented_sort_scan: key type must be int32, uint32, float, int64 or uint64"); return false;
    }
}

bool valid_shape(const SegShape& sh) { return (sh.items == 8 || sh.items == 16) && (sh.warp_small == 0 || sh.warp_small == 32); }

// The table as JSON: {"format": ..., "version": 1, "digit_bits": 8, "entries": [{"key_type":
// 5, "items": 16, "warp_small": 32, "ms": 3.1}, ...]}
std::string tuning_json_locked() {
    std::string j = "{\"format\": \"thrustrtc_b200.segmented_tuning\", \"version\": " +
                    std::to_string(SEG_TUNING_VERSION) +
                    ", \"classes\": [\"warp_bitonic: len <= warp_small\", \"warp_radix: len <= 32*items\", "
                    "\"group2_radix: len <= 64*items\", \"group4_radix: len <= 128*items\", "
                    "\"cta_onchip: len <= 256*items\", \"cta_global\"], \"digit_bits\": 8, \"entries\": [";
    bool first = true;
    for (const auto& kv : g_seg_tuning) {
        char buf[160];
        snprintf(buf, sizeof(buf), "%s{\"key_type\": %d, \"items\": %d, \"warp_small\": %d, \"ms\": %.4f}",
                 first ? "" : ", ", kv.first, kv.second.items, kv.second.warp_small, kv.second.ms);
        j += buf;
        first = false;
    }
    return j + "]}";
}

// Reads the entries of a table written by tuning_json_locked (tolerant of whitespace and key
// order inside an entry); rejects another format or version.
bool tuning_load_locked(const char* json) {
    const char* f = strstr(json, "\"thrustrtc_b200.segmented_tuning\"");
    const char* v = strstr(json, "\"version\"");
    if (!f || !v) { set_error("segmented tuning: not a thrustrtc_b200 segmented tuning table"); return false; }
    v = strchr(v, ':');
    if (!v || atoi(v + 1) != SEG_TUNING_VERSION) { set_error("segmented tuning: unsupported table version"); return false; }
    auto field = [](const char* b, const char* e, const char* name, int* out) {
        const char* p = strstr(b, name);
        if (!p || p > e) return false;
        p = strchr(p, ':');
        if (!p || p > e) return false;
        *out = atoi(p + 1);
        return true;
    };
    std::map<int, SegShape> t;
    const char* p = strstr(json, "\"entries\"");
    while (p && (p = strchr(p, '{')) != nullptr) {
        const char* e = strchr(p, '}');
        if (!e) break;
        int kt = 0, it = 0, wsm = 0;
        if (!field(p, e, "\"key_type\"", &kt) || !field(p, e, "\"items\"", &it) ||
            !field(p, e, "\"warp_small\"", &wsm)) {
            set_error("segmented tuning: malformed entry");
            return false;
        }
        SegShape sh{it, wsm, 0.f};
        if (!valid_shape(sh)) { set_error("segmented tuning: unsupported shape in the table"); return false; }
        t[kt] = sh;
        p = e + 1;
    }
    for (const auto& kv : t) g_seg_tuning[kv.first] = kv.second;
    return true;
}

// TRTC_SEG_TUNING_FILE: a table to load at the first batched call of the process
void load_env_tuning_locked() {
    if (g_seg_env_loaded) return;
    g_seg_env_loaded = true;
    const char* path = getenv("TRTC_SEG_TUNING_FILE");
    if (!path || !*path) return;
    FILE* fp = fopen(path, "rb");
    if (!fp) return;
    std::string text;
    char buf[4096];
    size_t r;
    while ((r = fread(buf, 1, sizeof(buf), fp)) > 0) text.append(buf, r);
    fclose(fp);
    tuning_load_locked(text.c_str());
}

SegShape tuned_shape(int tc) {
    std::lock_guard<std::mutex> lk(g_seg_mu);
    load_env_tuning_locked();
    auto it = g_seg_tuning.find(tc);
    return it == g_seg_tuning.end() ? SEG_DEFAULT : it->second;
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

int segmented_tuned_items(int tc) { return tuned_shape(tc).items; }

std::string segmented_tuning_json() {
    std::lock_guard<std::mutex> lk(g_seg_mu);
    load_env_tuning_locked();
    return tuning_json_locked();
}

bool segmented_tuning_load(const char* json) {
    if (!json) { set_error("segmented tuning: no table"); return false; }
    std::lock_guard<std::mutex> lk(g_seg_mu);
    g_seg_env_loaded = true;
    return tuning_load_locked(json);
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
    return seg_dispatch(tc, tuned_shape(tc), desc, keys, vals, scan, off, nseg, n, ws, s);
}

// Times every configuration on a copy of the batch shape (random keys, the caller's segment
// offsets) and keeps the fastest for this key type.  Allocates its own scratch.
bool segmented_autotune(int tc, const unsigned long long* off, size_t nseg, size_t n, cudaStream_t s, int* chosen) {
    if (!ensure_device()) return false;
    if (nseg == 0 || n == 0) { *chosen = segmented_tuned_items(tc); return true; }
    if (tc != TC_U32 && tc != TC_I32 && tc != TC_F32 && tc != TC_U64 && tc != TC_I64) {
        set_error("segmented autotune: key type must be int32, uint32, float, int64 or uint64");
        return false;
    }
    const size_t ksz = (tc == TC_U64 || tc == TC_I64) ? 8 : 4;
    const size_t wsb = segmented_workspace_bytes(tc, n, nseg);
    void *k = nullptr, *v = nullptr, *sc = nullptr, *ws = nullptr;
    bool ok = TRTC_CUDA(cudaMalloc(&k, n * ksz)) && TRTC_CUDA(cudaMalloc(&v, n * 4)) &&
              TRTC_CUDA(cudaMalloc(&sc, n * 4)) && TRTC_CUDA(cudaMalloc(&ws, wsb));
    cudaEvent_t a = nullptr, b = nullptr;
    ok = ok && TRTC_CUDA(cudaEventCreate(&a)) && TRTC_CUDA(cudaEventCreate(&b));
    SegShape best = SEG_DEFAULT;
    float best_ms = 1e30f;
    for (const SegShape& cfg : SEG_CONFIGS) {
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
        if (ok && tot < best_ms) { best_ms = tot; best = cfg; best.ms = tot / 3.f; }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(k); cudaFree(v); cudaFree(sc); cudaFree(ws);
    if (!ok) return false;
    {
        std::lock_guard<std::mutex> lk(g_seg_mu);
        g_seg_env_loaded = true;
        g_seg_tuning[tc] = best;
    }
    *chosen = best.items;
    return true;
}

}  // namespace trtc_host
