// trtc_search.cuh -- vectorised and single-value binary searches in a sorted view.
//
// The reference searches one value with a multi-round parallel bisection that narrows the
// range on the host (binary_search.cpp:25-240) and many values with one thread per value
// (binary_search.cpp:286-332).  Here both are one launch: a thread per searched value, each
// running d_lower_bound / d_upper_bound / d_binary_search of trtc_builtins.cuh under the
// comparator.  Results match the reference's for views sorted under that comparator.
#pragma once
#include "trtc_builtins.cuh"

namespace trtc {

enum SearchKind : int { SEARCH_LOWER = 0, SEARCH_UPPER = 1, SEARCH_FOUND = 2 };

template <int KIND, class VecV, class Comp>
TRTC_FORCEINLINE size_t search_one(VecV& vec, const typename VecV::value_t& v, Comp& comp) {
    if constexpr (KIND == SEARCH_LOWER) return d_lower_bound(vec, v, comp);
    else if constexpr (KIND == SEARCH_UPPER) return d_upper_bound(vec, v, comp);
    else {
        const size_t i = d_lower_bound(vec, v, comp);
        return (i < vec.size() && !comp(v, vec[i])) ? 1 : 0;
    }
}

// result[i] = search(values[i]) for i < m
template <int KIND, class VecV, class ValV, class OutV, class Comp>
__global__ void search_v_kernel(VecV vec, ValV values, OutV result, size_t m, Comp comp) {
    typedef typename remove_cvref<typename OutV::value_t>::type R;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        const typename VecV::value_t v = (typename VecV::value_t)values[i];
        result[i] = (R)search_one<KIND>(vec, v, comp);
    }
}

// *out = search(value), one thread
template <int KIND, class VecV, class T, class Comp>
__global__ void search_one_kernel(VecV vec, T value, Comp comp, unsigned long long* out) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const typename VecV::value_t v = (typename VecV::value_t)value;
        *out = (unsigned long long)search_one<KIND>(vec, v, comp);
    }
}

}  // namespace trtc
