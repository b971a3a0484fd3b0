// ref_launch_calc.cpp -- test infrastructure: the block-size and resident-block queries of the
// reference library (declared in its internal/launch_calc.h), answered by the CUDA driver.
//
// The reference computes these with a vendored copy of an occupancy calculator
// (internal/cuda_occupancy.h:618-632 and the functions after it) that knows compute
// capabilities 3.x to 8.x only; for a B200 (10.0) it returns CUDA_OCC_ERROR_UNKNOWN_DEVICE,
// internal/launch_calc.cpp ignores that status, the block size stays -1, and every kernel the
// reference launches through TRTCContext::launch_for fails without a message
// (internal/impl_context.inl:827-828).  oracle/build_ref.py therefore builds the reference with
// this file in place of internal/launch_calc.cpp.  Block sizes only decide how the reference
// spreads its grid-stride work (its reductions and scans fix their own 256/512-wide blocks), so
// the results it computes do not depend on them.
#include <dlfcn.h>
#include <cstddef>
#include <cstdio>

#include "launch_calc.h"

namespace {

typedef size_t (*B2DSize)(int);
typedef int (*PFN_max_potential_block_size)(int*, int*, void*, B2DSize, size_t, int);
typedef int (*PFN_max_active_blocks)(int*, void*, int, size_t);

struct DriverOccupancy {
    PFN_max_potential_block_size block_size = nullptr;
    PFN_max_active_blocks active_blocks = nullptr;
    DriverOccupancy() {
        void* h = dlopen("libcuda.so.1", RTLD_LAZY | RTLD_NOLOAD);
        if (!h) h = dlopen("libcuda.so.1", RTLD_LAZY);
        if (!h) h = dlopen("libcuda.so", RTLD_LAZY);
        if (!h) return;
        block_size = (PFN_max_potential_block_size)dlsym(h, "cuOccupancyMaxPotentialBlockSize");
        active_blocks = (PFN_max_active_blocks)dlsym(h, "cuOccupancyMaxActiveBlocksPerMultiprocessor");
    }
};

const DriverOccupancy& driver() {
    static DriverOccupancy d;
    return d;
}

}  // namespace

bool launch_calc(CUfunction func, unsigned sharedMemBytes, int& sizeBlock) {
    const DriverOccupancy& d = driver();
    if (!d.block_size) {
        printf("ref_launch_calc: cuOccupancyMaxPotentialBlockSize not found\n");
        return false;
    }
    int min_grid = 0, bs = 0;
    const int r = d.block_size(&min_grid, &bs, (void*)func, nullptr, (size_t)sharedMemBytes, 0);
    if (r != 0 || bs <= 0) {
        printf("ref_launch_calc: cuOccupancyMaxPotentialBlockSize failed (%d)\n", r);
        return false;
    }
    sizeBlock = bs;
    return true;
}

bool persist_calc(CUfunction func, unsigned sharedMemBytes, int sizeBlock, int& numBlocks) {
    const DriverOccupancy& d = driver();
    CUdevice dev;
    int sms = 0, per_sm = 0;
    if (!d.active_blocks || cuCtxGetDevice(&dev) != CUDA_SUCCESS ||
        cuDeviceGetAttribute(&sms, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, dev) != CUDA_SUCCESS ||
        d.active_blocks(&per_sm, (void*)func, sizeBlock, (size_t)sharedMemBytes) != 0) {
        printf("ref_launch_calc: occupancy query failed\n");
        return false;
    }
    numBlocks = per_sm * sms;
    return true;
}
