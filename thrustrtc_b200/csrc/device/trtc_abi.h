// trtc_abi.h -- plain structs passed by value from host code to kernels.  No device code:
// included by the kernel headers (nvcc and NVRTC) and by host .cpp files, so both sides
// agree on the byte layout of these kernel parameters.
#pragma once

namespace trtc {

struct LookbackState {
    unsigned int* flags;            // [tiles] epoch4 + 1 (aggregate) / epoch4 + 2 (inclusive)
    void* agg;                      // [tiles] tile aggregates (value type of the scan)
    void* incl;                     // [tiles] inclusive prefixes
    unsigned char* heads;           // [tiles] segmented scans: tile contains a segment head
    unsigned long long* tile_ctr;   // tile ticket counter (zero between launches)
    unsigned int epoch4;
    unsigned int* err;              // host-visible error word
    void* result;                   // optional: the last tile stores the grand total here
};

}  // namespace trtc
