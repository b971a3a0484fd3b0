// launch_sort_64.cu -- radix sort instantiations for the 64 key types.
#include "launch_sort_impl.cuh"
#include "trtc_launch.h"

namespace trtc_host {

bool sort_raw_64(int tc, void* keys, void* vals, size_t vsize, size_t n, bool desc, cudaStream_t s) {
    switch (tc) {
        case TC_U64: return desc ? radix_sort_dispatch<uint64_t, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<uint64_t, false>(keys, vals, vsize, n, s);
        case TC_I64: return desc ? radix_sort_dispatch<int64_t, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<int64_t, false>(keys, vals, vsize, n, s);
        case TC_F64: return desc ? radix_sort_dispatch<double, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<double, false>(keys, vals, vsize, n, s);
        default: set_error("sort: unsupported key type"); return false;
    }
}

}  // namespace trtc_host
