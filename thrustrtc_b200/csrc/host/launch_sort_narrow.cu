// launch_sort_narrow.cu -- radix sort instantiations for the narrow key types.
#include "launch_sort_impl.cuh"
#include "trtc_launch.h"

namespace trtc_host {

bool sort_raw_narrow(int tc, void* keys, void* vals, size_t vsize, size_t n, bool desc, cudaStream_t s) {
    switch (tc) {
        case TC_U8: return desc ? radix_sort_dispatch<uint8_t, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<uint8_t, false>(keys, vals, vsize, n, s);
        case TC_I8: return desc ? radix_sort_dispatch<int8_t, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<int8_t, false>(keys, vals, vsize, n, s);
        case TC_U16: return desc ? radix_sort_dispatch<uint16_t, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<uint16_t, false>(keys, vals, vsize, n, s);
        case TC_I16: return desc ? radix_sort_dispatch<int16_t, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<int16_t, false>(keys, vals, vsize, n, s);
        default: set_error("sort: unsupported key type"); return false;
    }
}

}  // namespace trtc_host
