// trtc_prelude.cuh -- shared device-side basics for the thrustrtc_b200 kernels.
//
// Compiled two ways: by nvcc for the built-in (cubin) instantiations, and by NVRTC
// (-arch=sm_100a) when a user Functor or a non-contiguous view has to be slotted into a
// kernel template.  It therefore includes no system header under NVRTC.
#pragma once

#ifdef __CUDACC_RTC__
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef short int16_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
typedef decltype(sizeof(0)) size_t;
#else
#include <cstdint>
#include <cstddef>
#endif

#ifndef TRTC_FORCEINLINE
#define TRTC_FORCEINLINE __device__ __forceinline__
#endif

namespace trtc {

// ------------------------------------------------------------------ small type traits
template <class A, class B> struct is_same { static constexpr bool value = false; };
template <class A> struct is_same<A, A> { static constexpr bool value = true; };
template <bool C, class A, class B> struct conditional { typedef A type; };
template <class A, class B> struct conditional<false, A, B> { typedef B type; };
template <class T> struct remove_cvref { typedef T type; };
template <class T> struct remove_cvref<const T> { typedef T type; };
template <class T> struct remove_cvref<T&> { typedef T type; };
template <class T> struct remove_cvref<const T&> { typedef T type; };

// placeholder for an unused kernel parameter slot (one byte, like an empty struct view)
struct Nothing {
    TRTC_FORCEINLINE Nothing& operator[](size_t) { return *this; }
    template <class T> TRTC_FORCEINLINE Nothing& operator=(const T&) { return *this; }
};

// ------------------------------------------------------------------ memory ordering
// Decoupled look-back publishes a value and then a flag with release semantics; readers
// acquire the flag before they read the value.  Hand-written PTX (sm_70+ memory model).
TRTC_FORCEINLINE uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
TRTC_FORCEINLINE unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
TRTC_FORCEINLINE void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
TRTC_FORCEINLINE void st_release(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Polls use relaxed loads (independent polls may be in flight together; an acquire load
// would order every later load behind it) followed by one fence before the values that the
// flags publish are read.
TRTC_FORCEINLINE uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
TRTC_FORCEINLINE unsigned long long ld_relaxed(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
TRTC_FORCEINLINE void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
// Stores of status words that carry their own value: no ordering with other data needed.
TRTC_FORCEINLINE void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
TRTC_FORCEINLINE void st_relaxed(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

TRTC_FORCEINLINE uint32_t lane_id() { return threadIdx.x & 31u; }
TRTC_FORCEINLINE uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Every spin on another CTA's flag is bounded.  After this many polls the waiting thread
// records an error in the call's status word and gives up (results are then garbage and
// the host reports failure); a GPU is never left spinning.
#ifndef TRTC_SPIN_LIMIT
#define TRTC_SPIN_LIMIT (1u << 22)
#endif
enum : uint32_t { TRTC_ERR_LOOKBACK_TIMEOUT = 1u, TRTC_ERR_BAD_PLAN = 2u, TRTC_ERR_BULK_COPY_TIMEOUT = 4u };

TRTC_FORCEINLINE void report_error(uint32_t* err, uint32_t code) {
    if (err) atomicOr(err, code);
}

TRTC_FORCEINLINE void backoff(uint32_t spins) {
    if (spins > 64) __nanosleep(spins > 4096 ? 256 : 32);
}

// One poll of a bounded wait.  Returns false when the wait must be abandoned: the poll
// budget is spent, or another thread has already reported an error (then every waiter
// gives up quickly instead of each spending its own budget).
// L2 prefetch of elements [first, first + count) of a contiguous array by the tensor memory
// accelerator (cp.async.bulk.prefetch, no multicast: no shared memory, no load/store-pipe
// work), issued only when the whole range lies inside [0, n), starts 16-byte aligned and
// spans a multiple of 16 bytes.  A hint: it changes no result.
template <class E>
TRTC_FORCEINLINE void prefetch_l2_range(const E* base, size_t first, size_t count, size_t n) {
    if (!base || count == 0 || first + count > n) return;
    const E* p = base + first;
    const size_t bytes = count * sizeof(E);
    if ((reinterpret_cast<size_t>(p) & 15u) != 0 || (bytes & 15u) != 0 || bytes >= (1u << 30)) return;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"((uint32_t)bytes) : "memory");
}

TRTC_FORCEINLINE bool spin_continue(uint32_t& spins, const uint32_t* err) {
    ++spins;
    if (spins > TRTC_SPIN_LIMIT) return false;
    if ((spins & 255u) == 0 && err && *(volatile const uint32_t*)err) return false;
    backoff(spins);
    return true;
}

// ------------------------------------------------------------------ L2 eviction hints
// 16-byte global loads/stores with an L2 eviction-priority policy (createpolicy, sm_80+).
TRTC_FORCEINLINE unsigned long long l2_evict_last_policy() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
TRTC_FORCEINLINE unsigned long long l2_evict_first_policy() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
TRTC_FORCEINLINE uint4 ld_l2hint(const uint4* a, unsigned long long pol) {
    uint4 v;
    asm volatile("ld.global.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(a), "l"(pol));
    return v;
}
TRTC_FORCEINLINE void st_l2hint(uint4* a, const uint4& v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v4.u32 [%0], {%1, %2, %3, %4}, %5;"
                 :: "l"(a), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "l"(pol) : "memory");
}

// ------------------------------------------------------------------ radix key maps
// RadixKey<K>::ordered(k) returns an unsigned code whose unsigned order is the order in
// which the reference radix sort places keys (internal/radix_sort.cpp with the key maps of
// built_in.h:430-458): integer types in their natural order; float/double through d_u32 /
// d_u64 (a set sign bit negates the magnitude bits, so -0.0 and +0.0 tie), then the sign
// bit flipped so that the signed order of d becomes the unsigned order of the code.  The
// rotation that a NaN can cause through the reference's Min_Element tree is applied by the
// sort driver, not here.  Narrow types keep their own width so only their bytes are passes.
template <class K> struct RadixKey;
// Keys are moved and ranked as raw bit patterns (B) only.  Floating-point keys are never
// handled as floating-point values inside the sort: arithmetic or selects on a NaN may
// return the canonical NaN and lose its sign and payload bits, which the order depends on.
#define TRTC_RADIX_INT_KEY(K_, B_, DIG_, FLIP_)                                              \
    template <> struct RadixKey<K_> {                                                       \
        typedef B_ B; typedef uint32_t U; enum { DIGITS = DIG_ };                           \
        static TRTC_FORCEINLINE U ordered(B b) { return (U)b ^ (U)(FLIP_); }                \
        static TRTC_FORCEINLINE bool is_nan(B) { return false; }                            \
        static TRTC_FORCEINLINE K_ value(B b) { return (K_)b; }                             \
    };
TRTC_RADIX_INT_KEY(uint8_t, uint8_t, 1, 0u)
TRTC_RADIX_INT_KEY(int8_t, uint8_t, 1, 0x80u)
TRTC_RADIX_INT_KEY(uint16_t, uint16_t, 2, 0u)
TRTC_RADIX_INT_KEY(int16_t, uint16_t, 2, 0x8000u)
TRTC_RADIX_INT_KEY(uint32_t, uint32_t, 4, 0u)
TRTC_RADIX_INT_KEY(int32_t, uint32_t, 4, 0x80000000u)
#undef TRTC_RADIX_INT_KEY
template <> struct RadixKey<uint64_t> {
    typedef unsigned long long B; typedef unsigned long long U; enum { DIGITS = 8 };
    static TRTC_FORCEINLINE U ordered(B b) { return b; }
    static TRTC_FORCEINLINE bool is_nan(B) { return false; }
    static TRTC_FORCEINLINE uint64_t value(B b) { return (uint64_t)b; }
};
template <> struct RadixKey<int64_t> {
    typedef unsigned long long B; typedef unsigned long long U; enum { DIGITS = 8 };
    static TRTC_FORCEINLINE U ordered(B b) { return b ^ 0x8000000000000000ull; }
    static TRTC_FORCEINLINE bool is_nan(B) { return false; }
    static TRTC_FORCEINLINE int64_t value(B b) { return (int64_t)b; }
};
template <> struct RadixKey<float> {
    typedef uint32_t B; typedef uint32_t U; enum { DIGITS = 4 };
    static TRTC_FORCEINLINE U ordered(B u) {
        if (u & 0x80000000u) u = 0u - (u & 0x7FFFFFFFu);
        return u ^ 0x80000000u;
    }
    static TRTC_FORCEINLINE bool is_nan(B u) { return (u & 0x7FFFFFFFu) > 0x7F800000u; }
    static TRTC_FORCEINLINE float value(B b) { return __uint_as_float(b); }
};
// double: d_u64 as the reference computes it on the GPU (built_in.h:450-457, compiled by
// NVRTC): a negative NaN's code is 0 - |bits| with bit 63 clear, after its signalling payload
// is quietened (bit 51 set), which orders it just above +0.0; every other value maps as the
// source reads.
template <> struct RadixKey<double> {
    typedef unsigned long long B; typedef unsigned long long U; enum { DIGITS = 8 };
    static TRTC_FORCEINLINE U ordered(B u) {
        if (u & 0x8000000000000000ull) {
            unsigned long long mag = u & 0x7FFFFFFFFFFFFFFFull;
            const bool nan = mag > 0x7FF0000000000000ull;
            if (nan) mag |= 0x0008000000000000ull;
            u = 0ull - mag;
            if (nan) u &= 0x7FFFFFFFFFFFFFFFull;
        }
        return u ^ 0x8000000000000000ull;
    }
    static TRTC_FORCEINLINE bool is_nan(B u) { return (u & 0x7FFFFFFFFFFFFFFFull) > 0x7FF0000000000000ull; }
    static TRTC_FORCEINLINE double value(B b) { return __longlong_as_double((long long)b); }
};

// ------------------------------------------------------------------ warp helpers
template <class T> TRTC_FORCEINLINE T shfl(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <class T> TRTC_FORCEINLINE T shfl_up(T v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
template <class T> TRTC_FORCEINLINE T shfl_down(T v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

// Generic shuffles for values of any trivially copyable type (user structs, Pair<,>):
// moved as 32-bit words.
template <class T> struct ShflWords { enum { N = (sizeof(T) + 3) / 4 }; };
template <class T> TRTC_FORCEINLINE T shfl_any(const T& v, int src) {
    union U { T t; uint32_t w[ShflWords<T>::N]; TRTC_FORCEINLINE U() {} } a, b;
    a.t = v;
#pragma unroll
    for (int i = 0; i < ShflWords<T>::N; i++) b.w[i] = __shfl_sync(0xffffffffu, a.w[i], src);
    return b.t;
}
template <class T> TRTC_FORCEINLINE T shfl_up_any(const T& v, int d) {
    union U { T t; uint32_t w[ShflWords<T>::N]; TRTC_FORCEINLINE U() {} } a, b;
    a.t = v;
#pragma unroll
    for (int i = 0; i < ShflWords<T>::N; i++) b.w[i] = __shfl_up_sync(0xffffffffu, a.w[i], d);
    return b.t;
}
template <class T> TRTC_FORCEINLINE T shfl_xor_any(const T& v, int m) {
    union U { T t; uint32_t w[ShflWords<T>::N]; TRTC_FORCEINLINE U() {} } a, b;
    a.t = v;
#pragma unroll
    for (int i = 0; i < ShflWords<T>::N; i++) b.w[i] = __shfl_xor_sync(0xffffffffu, a.w[i], m);
    return b.t;
}
template <class T> TRTC_FORCEINLINE T shfl_down_any(const T& v, int d) {
    union U { T t; uint32_t w[ShflWords<T>::N]; TRTC_FORCEINLINE U() {} } a, b;
    a.t = v;
#pragma unroll
    for (int i = 0; i < ShflWords<T>::N; i++) b.w[i] = __shfl_down_sync(0xffffffffu, a.w[i], d);
    return b.t;
}

TRTC_FORCEINLINE size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }

}  // namespace trtc
