// trtc_builtins.cuh -- device-side vocabulary shared with user Functor code.
//
// User Functor bodies are written against the names the reference exposes to device code
// (built_in.h:5-458): Pair<>, the built-in operator structs, the *View structs with their
// value_t / ref_t typedefs, _data / _size members, size() and operator[], and the
// d_u32/d_u64 key maps.  This header restates that vocabulary for thrustrtc_b200 so that
// existing Functor strings keep compiling unchanged (same names, member names and byte
// layouts -- the host packs view bytes against these layouts).
#pragma once
#include "trtc_prelude.cuh"

////////// Elements ///////////
template <class T1, class T2>
struct Pair {
    T1 first;
    T2 second;
};

////////// Built-in operators (semantics of built_in.h:14-150) ///////////
struct Identity {
    template <typename T> __device__ inline T operator()(const T& x) const { return x; }
};
struct Maximum {
    template <typename T> __device__ inline T operator()(const T& x, const T& y) const { return x < y ? y : x; }
};
struct Minimum {
    template <typename T> __device__ inline T operator()(const T& x, const T& y) const { return x > y ? y : x; }
};
struct EqualTo {
    template <typename T> __device__ inline bool operator()(const T& x, const T& y) const { return x == y; }
};
struct NotEqualTo {
    template <typename T> __device__ inline bool operator()(const T& x, const T& y) const { return x != y; }
};
struct Greater {
    template <typename T> __device__ inline bool operator()(const T& x, const T& y) const { return x > y; }
};
struct Less {
    template <typename T> __device__ inline bool operator()(const T& x, const T& y) const { return x < y; }
};
struct GreaterEqual {
    template <typename T> __device__ inline bool operator()(const T& x, const T& y) const { return x >= y; }
};
struct LessEqual {
    template <typename T> __device__ inline bool operator()(const T& x, const T& y) const { return x <= y; }
};
struct Plus {
    template <typename T> __device__ inline T operator()(const T& x, const T& y) const { return x + y; }
};
struct Minus {
    template <typename T> __device__ inline T operator()(const T& x, const T& y) const { return x - y; }
};
struct Multiplies {
    template <typename T> __device__ inline T operator()(const T& x, const T& y) const { return x * y; }
};
struct Divides {
    template <typename T> __device__ inline T operator()(const T& x, const T& y) const { return x / y; }
};
struct Modulus {
    template <typename T> __device__ inline T operator()(const T& x, const T& y) const { return x % y; }
};
struct Negate {
    template <typename T> __device__ inline T operator()(const T& x) const { return -x; }
};

////////// Views (byte layouts of the reference's view structs) ///////////
template <class _T>
struct VectorView {
    typedef _T value_t;
    typedef _T& ref_t;
    value_t* _data;
    size_t _size;
    __device__ size_t size() const { return _size; }
    __device__ ref_t operator[](size_t idx) { return _data[idx]; }
};

template <class _TVVALUE>
struct RangeView {
    typedef typename _TVVALUE::value_t value_t;
    typedef typename _TVVALUE::ref_t ref_t;
    _TVVALUE _view_vec_value;
    size_t _begin;
    size_t _end;
    __device__ size_t size() const { return _end - _begin; }
    __device__ ref_t operator[](size_t idx) { return _view_vec_value[idx + _begin]; }
};

template <class _T>
struct ConstantView {
    typedef _T value_t;
    typedef const _T& ref_t;
    size_t _size;
    value_t _value;
    __device__ size_t size() const { return _size; }
    __device__ ref_t operator[](size_t) { return _value; }
};

template <class _T>
struct CounterView {
    typedef _T value_t;
    typedef _T ref_t;
    size_t _size;
    value_t _value_init;
    __device__ size_t size() const { return _size; }
    __device__ ref_t operator[](size_t idx) { return _value_init + (value_t)idx; }
};

template <class _T>
struct _Sink {
    __device__ const _T& operator=(const _T& in) { return in; }
};

template <class _T>
struct DiscardView {
    typedef _T value_t;
    typedef _Sink<_T>& ref_t;
    size_t _size;
    _Sink<_T> _sink;
    __device__ size_t size() const { return _size; }
    __device__ ref_t operator[](size_t) { return _sink; }
};

template <class _TVVALUE, class _TVINDEX>
struct PermutationView {
    typedef typename _TVVALUE::value_t value_t;
    typedef typename _TVVALUE::ref_t ref_t;
    _TVVALUE _view_vec_value;
    _TVINDEX _view_vec_index;
    __device__ size_t size() const { return _view_vec_index.size(); }
    __device__ ref_t operator[](size_t idx) { return _view_vec_value[_view_vec_index[idx]]; }
};

template <class _TVVALUE>
struct ReverseView {
    typedef typename _TVVALUE::value_t value_t;
    typedef typename _TVVALUE::ref_t ref_t;
    _TVVALUE _view_vec_value;
    __device__ size_t size() const { return _view_vec_value.size(); }
    __device__ value_t& operator[](size_t idx) { return _view_vec_value[size() - 1 - idx]; }
};

template <class _T, class _T_VIN, class _T_OP>
struct TransformView {
    typedef _T value_t;
    typedef _T ref_t;
    _T_VIN _view_vec_in;
    _T_OP _view_op;
    __device__ size_t size() const { return _view_vec_in.size(); }
    __device__ ref_t operator[](size_t idx) { return _view_op(_view_vec_in[idx]); }
};

////////// key maps for user code (semantics of built_in.h:430-458) ///////////
template <typename T> __device__ inline uint32_t d_u32(T v) { return (uint32_t)v; }
template <> __device__ inline uint32_t d_u32<float>(float v) {
    uint32_t u = __float_as_uint(v);
    if (u & 0x80000000u) u = 0u - (u & 0x7FFFFFFFu);
    return u;
}
template <typename T> __device__ inline uint64_t d_u64(T v) { return (uint64_t)v; }
// as the reference's d_u64<double> evaluates on the GPU: a negative NaN (quietened) maps to
// 0 - |bits| with bit 63 clear
template <> __device__ inline uint64_t d_u64<double>(double v) {
    uint64_t u = (uint64_t)__double_as_longlong(v);
    if (u & 0x8000000000000000ull) {
        uint64_t mag = u & 0x7FFFFFFFFFFFFFFFull;
        const bool nan = mag > 0x7FF0000000000000ull;
        if (nan) mag |= 0x0008000000000000ull;
        u = 0ull - mag;
        if (nan) u &= 0x7FFFFFFFFFFFFFFFull;
    }
    return u;
}

////////// binary searches over a view (lower/upper bound, comparator slot) ///////////
template <class TVec, class TComp>
__device__ inline size_t d_lower_bound(TVec& vec, const typename TVec::value_t& value, TComp& comp,
                                       size_t begin = 0, size_t end = (size_t)(-1)) {
    if (end == (size_t)(-1)) end = vec.size();
    size_t lo = begin, hi = end;
    while (lo < hi) {
        size_t mid = lo + ((hi - lo) >> 1);
        if (comp(vec[mid], value)) lo = mid + 1; else hi = mid;
    }
    return lo;
}
template <class TVec, class TComp>
__device__ inline size_t d_upper_bound(TVec& vec, const typename TVec::value_t& value, TComp& comp,
                                       size_t begin = 0, size_t end = (size_t)(-1)) {
    if (end == (size_t)(-1)) end = vec.size();
    size_t lo = begin, hi = end;
    while (lo < hi) {
        size_t mid = lo + ((hi - lo) >> 1);
        if (comp(value, vec[mid])) hi = mid; else lo = mid + 1;
    }
    return lo;
}

namespace trtc {
// Contiguity trait: the kernels take a vectorised 16-byte path for VectorView inputs.
template <class V> struct ViewTraits { static constexpr bool contiguous = false; };
template <class T> struct ViewTraits<VectorView<T>> { static constexpr bool contiguous = true; };

// plain pointer view used by the nvcc-built instantiations (same layout as VectorView)
template <class T> __host__ __device__ __forceinline__ VectorView<T> make_view(T* p, size_t n) {
    VectorView<T> v; v._data = p; v._size = n; return v;
}
}  // namespace trtc
