// trtc_abi.h -- plain structs passed by value from host code to kernels.  No device code:
// included by the kernel headers (nvcc and NVRTC) and by host .cpp files, so both sides
// agree on the byte layout of these kernel parameters.
#pragma once

namespace trtc {

struct LookbackState {
    unsigned int* flags;            // [tiles] flag word: epoch8 + state (1 aggregate, 2 inclusive)
                                    //         + 4 when the tile holds a segment head
    unsigned long long* packed;     // [tiles] values of <= 4 bytes: (flag word << 32) | value bits
    void* agg;                      // [tiles] aggregates of larger values
    void* incl;                     // [tiles] inclusive prefixes of larger values
    unsigned long long* tile_ctr;   // tile ticket counter (zero between launches)
    unsigned int epoch8;            // per-launch epoch * 8: stale flags never look valid
    unsigned int* err;              // host-visible error word
    void* result;                   // optional: the last tile stores the grand total here
    unsigned int pf_ahead = 0;      // persistent tile kernels: when a CTA claims tile t, it
                                    // prefetches tile t + pf_ahead into L2 (0: none)
};

}  // namespace trtc
