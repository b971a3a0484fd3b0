// launch_sort_32.cu -- radix sort instantiations for the 32 key types.
#include "launch_sort_impl.cuh"
#include "trtc_launch.h"

namespace trtc_host {

bool sort_raw_32(int tc, void* keys, void* vals, size_t vsize, size_t n, bool desc, cudaStream_t s) {
    switch (tc) {
        case TC_U32: return desc ? radix_sort_dispatch<uint32_t, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<uint32_t, false>(keys, vals, vsize, n, s);
        case TC_I32: return desc ? radix_sort_dispatch<int32_t, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<int32_t, false>(keys, vals, vsize, n, s);
        case TC_F32: return desc ? radix_sort_dispatch<float, true>(keys, vals, vsize, n, s)
                          : radix_sort_dispatch<float, false>(keys, vals, vsize, n, s);
        default: set_error("sort: unsupported key type"); return false;
    }
}

bool min_element_raw(int tc, const void* keys, size_t n, cudaStream_t s, unsigned long long* idx) {
    if (n == 0) { *idx = 0; return true; }
    switch (tc) {
        case TC_I8: return min_element_run<int8_t>((const int8_t*)keys, n, s, idx);
        case TC_U8: return min_element_run<uint8_t>((const uint8_t*)keys, n, s, idx);
        case TC_I16: return min_element_run<int16_t>((const int16_t*)keys, n, s, idx);
        case TC_U16: return min_element_run<uint16_t>((const uint16_t*)keys, n, s, idx);
        case TC_I32: return min_element_run<int32_t>((const int32_t*)keys, n, s, idx);
        case TC_U32: return min_element_run<uint32_t>((const uint32_t*)keys, n, s, idx);
        case TC_I64: return min_element_run<int64_t>((const int64_t*)keys, n, s, idx);
        case TC_U64: return min_element_run<uint64_t>((const uint64_t*)keys, n, s, idx);
        case TC_F32: return min_element_run<float>((const float*)keys, n, s, idx);
        case TC_F64: return min_element_run<double>((const double*)keys, n, s, idx);
        default: set_error("min_element: unsupported type"); return false;
    }
}

bool sort_raw(int tc, void* keys, void* vals, size_t vsize, size_t n, bool desc, cudaStream_t s) {
    if (n == 0) { set_error("sort: empty input"); return false; }
    if (n == 1) return true;
    switch (tc) {
        case TC_I8: case TC_U8: case TC_I16: case TC_U16: return sort_raw_narrow(tc, keys, vals, vsize, n, desc, s);
        case TC_I32: case TC_U32: case TC_F32: return sort_raw_32(tc, keys, vals, vsize, n, desc, s);
        case TC_I64: case TC_U64: case TC_F64: return sort_raw_64(tc, keys, vals, vsize, n, desc, s);
        default: set_error("sort: unsupported key type"); return false;
    }
}

}  // namespace trtc_host
