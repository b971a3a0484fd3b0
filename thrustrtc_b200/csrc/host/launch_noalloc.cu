// launch_noalloc.cu -- trtc_raw_scan_noalloc: the persistent two-phase look-back scan that
// trtc_raw_scan runs for 4-byte element types (scan2_kernel, 256 threads x 32 elements per
// tile), with its look-back scratch in file-scope device arrays instead of workspace from
// cudaMalloc.  The call allocates nothing: no cudaMalloc/cudaFree, no pinned host memory, no
// stream-ordered pool, no library routine that allocates.
//
// Scratch (in this module's static device memory, one copy per CUDA context that loads the
// library, held until the process exits):
//   g_na_packed[NA_MAX_TILES]  one 64-bit (flag << 32 | value) look-back word per tile,
//                              epoch-tagged; zero at module load, cleared again (stream-ordered
//                              memset) when the epoch wraps
//   g_na_tile_ctr              tile ticket counter; zero at module load, and the CTA that takes
//                              the launch's last ticket resets it to zero
// A tile holds 8192 elements, so the 32768 words (256 KiB) serve n <= 2^28.
//
// The arrays' names are host-side stand-ins in host code, not device addresses: the device
// addresses come from cudaGetSymbolAddress, looked up once per CUDA context (on the first call
// made in it, with that context current) and cached under the context's unique id, so a
// context created after cudaDeviceReset gets its own look-up.
#include <cuda.h>

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "../device/trtc_scan.cuh"
#include "trtc_launch.h"
#include "trtc_runtime.h"

using namespace trtc;
using namespace trtc_host;

namespace {

constexpr int NA_BLOCK = 256;
constexpr int NA_ITEMS = 32;                                       // elements per thread (4-byte)
constexpr unsigned long long NA_TILE = NA_BLOCK * NA_ITEMS;        // 8192 elements per tile
constexpr unsigned long long NA_MAX_TILES = 1ull << 15;
constexpr unsigned long long NA_MAX_N = NA_MAX_TILES * NA_TILE;    // 2^28
constexpr uint32_t NA_EPOCH_LIMIT = 1u << 28;                      // epoch * 8 must fit 32 bits

static __device__ __align__(256) unsigned long long g_na_packed[NA_MAX_TILES];
static __device__ __align__(256) unsigned long long g_na_tile_ctr[2];

struct NaScratch {
    unsigned long long* packed = nullptr;
    unsigned long long* tile_ctr = nullptr;
    uint32_t epoch = 0;
    uint32_t epoch_limit = NA_EPOCH_LIMIT;
    int sms = 0;
};
std::mutex g_na_mu;
std::map<unsigned long long, NaScratch> g_na;  // per CUDA context (unique context id)

typedef CUresult (*PFN_ctxGetCurrent)(CUcontext*);
typedef CUresult (*PFN_ctxGetId)(CUcontext, unsigned long long*);
PFN_ctxGetCurrent g_ctx_current = nullptr;
PFN_ctxGetId g_ctx_id = nullptr;

// Id of the current context (the driver's unique context id where available, else the handle).
// The runtime makes the device's primary context current on its first call, so a thread that
// has no context yet gets one from the symbol look-up below.
bool current_context_id(unsigned long long* id) {
    if (!g_ctx_current) {
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&g_ctx_current, cudaEnableDefault, &q) !=
                cudaSuccess || q != cudaDriverEntryPointSuccess) {
            g_ctx_current = nullptr;
            set_error("scan_noalloc: cuCtxGetCurrent is not available");
            return false;
        }
        if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&g_ctx_id, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            g_ctx_id = nullptr;
    }
    CUcontext ctx = nullptr;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS) ctx = nullptr;
    if (!ctx) {
        void* p = nullptr;
        if (!TRTC_CUDA(cudaGetSymbolAddress(&p, g_na_tile_ctr))) return false;
        if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) { set_error("scan_noalloc: no current CUDA context"); return false; }
    }
    unsigned long long v = 0;
    if (g_ctx_id && g_ctx_id(ctx, &v) == CUDA_SUCCESS) *id = v;
    else *id = (unsigned long long)(uintptr_t)ctx;
    return true;
}

// Set-up, once per context, with that context current: the device addresses of the arrays.
// TRTC_NOALLOC_EPOCH_LIMIT (an integer >= 2) lowers the epoch wrap, so a test reaches the
// clear-on-wrap path in a few calls instead of 2^28.
bool na_setup(NaScratch*& out) {
    unsigned long long id = 0;
    if (!current_context_id(&id)) return false;
    auto it = g_na.find(id);
    if (it != g_na.end()) { out = &it->second; return true; }
    NaScratch s;
    cudaError_t e = cudaGetSymbolAddress((void**)&s.packed, g_na_packed);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&s.tile_ctr, g_na_tile_ctr);
    if (e != cudaSuccess) {
        set_error(std::string("scan_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorName(e) + " (" +
                  cudaGetErrorString(e) + ")");
        return false;
    }
    int dev = 0;
    if (!TRTC_CUDA(cudaGetDevice(&dev)) ||
        !TRTC_CUDA(cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev)))
        return false;
    if (const char* lim = getenv("TRTC_NOALLOC_EPOCH_LIMIT")) {
        const long v = strtol(lim, nullptr, 10);
        if (v >= 2 && (unsigned long)v < NA_EPOCH_LIMIT) s.epoch_limit = (uint32_t)v;
    }
    out = &(g_na[id] = s);
    return true;
}

template <class T, class Op, int MODE>
bool na_scan_t(const NaScratch& sc, uint32_t epoch8, uint32_t* err, const void* in, void* out, size_t n,
               const void* init, cudaStream_t s) {
    static_assert(sizeof(T) == 4, "4-byte elements only");
    const size_t tiles = (n + NA_TILE - 1) / NA_TILE;
    LookbackState st;
    st.flags = nullptr;  // 4-byte values use the packed words only
    st.packed = sc.packed;
    st.agg = nullptr;
    st.incl = nullptr;
    st.tile_ctr = sc.tile_ctr;
    st.epoch8 = epoch8;
    st.err = err;
    st.result = nullptr;
    T ini = T();
    if (init) std::memcpy(&ini, init, sizeof(T));
    // persistent CTAs, as many as are resident at once (the grid of trtc_raw_scan)
    auto kernel = scan2_kernel<T, Op, MODE, NA_BLOCK, NA_ITEMS, true>;
    static int per_sm = 0;
    if (per_sm == 0 && !TRTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NA_BLOCK, 0)))
        return false;
    size_t grid = (size_t)(per_sm > 0 ? per_sm : 1) * (size_t)sc.sms;
    if (grid > tiles) grid = tiles;
    kernel<<<(unsigned)grid, NA_BLOCK, 0, s>>>((const T*)in, (T*)out, n, tiles, Op(), ini, st);
    count_launch();
    return TRTC_CUDA(cudaGetLastError());
}

template <class T>
bool na_scan_op(const NaScratch& sc, uint32_t epoch8, uint32_t* err, int op, int mode, const void* in, void* out,
                size_t n, const void* init, cudaStream_t s) {
    switch (op * 2 + mode) {
        case 0: return na_scan_t<T, Plus, 0>(sc, epoch8, err, in, out, n, init, s);
        case 1: return na_scan_t<T, Plus, 1>(sc, epoch8, err, in, out, n, init, s);
        case 2: return na_scan_t<T, Maximum, 0>(sc, epoch8, err, in, out, n, init, s);
        case 3: return na_scan_t<T, Maximum, 1>(sc, epoch8, err, in, out, n, init, s);
        case 4: return na_scan_t<T, Minimum, 0>(sc, epoch8, err, in, out, n, init, s);
        case 5: return na_scan_t<T, Minimum, 1>(sc, epoch8, err, in, out, n, init, s);
        default: set_error("scan_noalloc: unsupported operator (0 Plus, 1 Maximum, 2 Minimum)"); return false;
    }
}

}  // namespace

extern "C" int trtc_raw_scan_noalloc(int type, int op, int exclusive, const void* in, void* out,
                                     unsigned long long n, const void* init, unsigned int* status_dev,
                                     void* stream) {
    if (n == 0) { set_error("scan_noalloc: empty input"); return -1; }
    if (n > NA_MAX_N) {
        set_error("scan_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " + std::to_string(NA_MAX_N) +
                  " elements (static scratch of " + std::to_string(NA_MAX_TILES) + " tiles of " +
                  std::to_string(NA_TILE) + ")");
        return -1;
    }
    if (type != TC_I32 && type != TC_U32 && type != TC_F32) {
        set_error("scan_noalloc: element type must be int32 (4), uint32 (5) or float (8)");
        return -1;
    }
    if (op < 0 || op > 2) { set_error("scan_noalloc: unsupported operator (0 Plus, 1 Maximum, 2 Minimum)"); return -1; }
    const cudaStream_t s = (cudaStream_t)stream;
    NaScratch* sc = nullptr;
    uint32_t epoch8 = 0;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (!na_setup(sc)) return -1;
        if (++sc->epoch >= sc->epoch_limit) {
            // stream-ordered clear of the tile words (earlier calls on `s` finish first)
            if (!TRTC_CUDA(cudaMemsetAsync(sc->packed, 0, sizeof(g_na_packed), s))) return -1;
            sc->epoch = 1;
        }
        epoch8 = sc->epoch * 8u;
    }
    uint32_t* err = (uint32_t*)status_dev;  // NULL: device-side failures are not reported
    const int mode = exclusive ? 1 : 0;
    bool ok;
    switch (type) {
        case TC_I32: ok = na_scan_op<int32_t>(*sc, epoch8, err, op, mode, in, out, n, init, s); break;
        case TC_U32: ok = na_scan_op<uint32_t>(*sc, epoch8, err, op, mode, in, out, n, init, s); break;
        default: ok = na_scan_op<float>(*sc, epoch8, err, op, mode, in, out, n, init, s); break;
    }
    return ok ? 0 : -1;
}
