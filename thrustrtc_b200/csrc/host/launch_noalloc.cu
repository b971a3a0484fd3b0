// launch_noalloc.cu -- trtc_raw_scan_noalloc: the single-pass look-back scan of scan_raw for
// 4-byte element types, with its look-back scratch in a file-scope device array instead of
// workspace obtained from cudaMalloc.  The call allocates nothing: no cudaMalloc/cudaFree,
// no pinned host memory, no stream-ordered pool.
//
// Scratch (per device, in this module's static device memory):
//   g_na_packed[NA_MAX_TILES]  one 64-bit (flag << 32 | value) word per tile, epoch-tagged;
//                              zero at module load, cleared again when the epoch wraps
//   g_na_tile_ctr              tile ticket counter; must be zero before a launch.  It is zero
//                              at module load and the CTA that takes the last ticket resets it
// A tile holds 256 threads x 4 chunks x 4 elements = 4096 elements, so with 65536 tiles the
// largest accepted n is 2^28 elements (512 KiB of scratch).
#include <cstring>
#include <mutex>
#include <map>
#include <string>

#include "../device/trtc_scan.cuh"
#include "trtc_launch.h"
#include "trtc_runtime.h"

using namespace trtc;
using namespace trtc_host;

namespace {

constexpr int NA_BLOCK = 256;
constexpr int NA_NV = 4;                                   // 16-byte vectors per lane and tile
constexpr unsigned long long NA_TILE = NA_BLOCK * NA_NV * 4;  // elements per tile (4-byte types)
constexpr unsigned long long NA_MAX_TILES = 1ull << 16;
constexpr unsigned long long NA_MAX_N = NA_MAX_TILES * NA_TILE;  // 2^28
constexpr uint32_t NA_EPOCH_LIMIT = 1u << 28;               // epoch * 8 must fit 32 bits

static __device__ __align__(256) unsigned long long g_na_packed[NA_MAX_TILES];
static __device__ __align__(256) unsigned long long g_na_tile_ctr[2];

struct NaScratch {
    unsigned long long* packed = nullptr;
    unsigned long long* tile_ctr = nullptr;
    uint32_t epoch = 0;
};
std::mutex g_na_mu;
std::map<int, NaScratch> g_na;  // per device ordinal

// One-time set-up per device, with that device current: the addresses of the static arrays.
bool na_setup(int dev, NaScratch*& out) {
    auto it = g_na.find(dev);
    if (it != g_na.end()) { out = &it->second; return true; }
    NaScratch s;
    cudaError_t e = cudaGetSymbolAddress((void**)&s.packed, g_na_packed);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&s.tile_ctr, g_na_tile_ctr);
    if (e != cudaSuccess) {
        set_error(std::string("scan_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorName(e) + " (" +
                  cudaGetErrorString(e) + ")");
        return false;
    }
    out = &(g_na[dev] = s);
    return true;
}

template <class T, class Op, int MODE>
bool na_scan_t(const NaScratch& sc, uint32_t epoch8, uint32_t* err, const void* in, void* out, size_t n,
               const void* init, cudaStream_t s) {
    static_assert(sizeof(T) == 4 && VecWidth<T>::V == 4, "4-byte elements only (the tiling of scan_raw)");
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
    VectorView<T> iv = make_view<T>(const_cast<T*>((const T*)in), n);
    VectorView<T> ov = make_view<T>((T*)out, n);
    scan_kernel<VectorView<T>, Nothing, false, VectorView<T>, T, Op, MODE, NA_BLOCK, NA_NV>
        <<<(unsigned)tiles, NA_BLOCK, 0, s>>>(iv, Nothing(), ov, n, Op(), ini, st);
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
    int dev = 0;
    if (!TRTC_CUDA(cudaGetDevice(&dev))) return -1;
    NaScratch* sc = nullptr;
    uint32_t epoch8 = 0;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (!na_setup(dev, sc)) return -1;
        if (++sc->epoch >= NA_EPOCH_LIMIT) {
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
