// launch_faultinject.cu -- test hook for the bounded look-back waits.
//
// One launch of the two-phase scan (scan2_kernel) built in this file only, in which tile 2
// never publishes its look-back word and every wait gives up after 4096 polls instead of
// 2^22.  The tiles behind tile 2 wait for a flag that nothing sets; their waits run out,
// the kernel records TRTC_ERR_LOOKBACK_TIMEOUT in the library's device error word and runs
// to its end, and the host reads and clears that word.  Nothing faults, traps or hangs: the
// test checks that the call reports the failure and that the next call succeeds.
#define TRTC_SPIN_LIMIT (1u << 12)
#define TRTC_FAULT_SKIP_PUBLISH(tile) ((tile) == 2)
#include "../device/trtc_scan.cuh"
#include "trtc_launch.h"
#include "trtc_runtime.h"

using namespace trtc_host;

namespace {
// a distinct operator type, so this kernel is an instantiation of its own (this file builds
// the scan with different wait bounds and publication than the product instantiations)
struct PlusWithStalledTile : ::Plus {};
}  // namespace

extern "C" int trtc_test_scan_lookback_timeout(const int* in, int* out, unsigned long long n, void* stream) {
    constexpr int BLOCK = 256, ITEMS = 32, TILE = BLOCK * ITEMS;
    if (!ensure_device()) return -1;
    if (n < 4ull * TILE) { set_error("lookback timeout test: needs at least 4 tiles of 8192 elements"); return -1; }
    const cudaStream_t s = (cudaStream_t)stream;
    const size_t tiles = (n + TILE - 1) / TILE;
    uint32_t e8 = 0;
    LookbackWs* w = lookback_ws(s, tiles, sizeof(int), &e8);
    if (!w) return -1;
    trtc::LookbackState st;
    st.flags = w->flags;
    st.agg = w->agg;
    st.incl = w->incl;
    st.packed = w->packed;
    st.tile_ctr = w->tile_ctr;
    st.epoch8 = e8;
    st.err = device_error_word();
    st.result = w->result;
    size_t grid = (size_t)sm_count();
    if (grid > tiles) grid = tiles;
    trtc::scan2_kernel<int, PlusWithStalledTile, 0, BLOCK, ITEMS, true>
        <<<(unsigned)grid, BLOCK, 0, s>>>(in, out, (size_t)n, tiles, PlusWithStalledTile(), 0, st);
    count_launch();
    if (!TRTC_CUDA(cudaGetLastError())) return -1;
    return check_device_errors(s, "lookback timeout test") ? 0 : -1;
}
