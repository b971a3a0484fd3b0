// CPU oracle for the ThrustRTC hot path (sort / scan / scan_by_key / reduce / min_element).
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the host, what the reference library
// (fynv/ThrustRTC) computes on the GPU, so that the CUDA kernels of thrustrtc_b200 can be
// checked against it.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// may load it, and only as the checker or the timed CPU baseline -- never as a product path.
//
// Every function cites the reference file:line whose behaviour it restates.  Type codes:
//   0 int8  1 uint8  2 int16  3 uint16  4 int32  5 uint32  6 int64  7 uint64  8 float  9 double
// Operator codes: 0 Plus, 1 Maximum, 2 Minimum (built_in.h:14-150 semantics).
#include <cstdint>
#include <cstring>
#include <cstddef>
#include <vector>
#include <algorithm>
#include <numeric>
#include <thread>

namespace {

enum { T_I8 = 0, T_U8, T_I16, T_U16, T_I32, T_U32, T_I64, T_U64, T_F32, T_F64 };
enum { OP_PLUS = 0, OP_MAX = 1, OP_MIN = 2 };

// ---- built-in operators, built_in.h:23-39 (Maximum: x<y?y:x, Minimum: x>y?y:x) and :96-103 (Plus)
template <class T> inline T op_apply(int op, T x, T y) {
    switch (op) {
        case OP_PLUS: return (T)(x + y);
        case OP_MAX: return x < y ? y : x;
        default: return x > y ? y : x;
    }
}

// ---- key maps d_u32 / d_u64, built_in.h:430-458.  Integer types are a plain cast
// (sign extending for signed types); float/double: bits, and for a set sign bit the
// two's-complement negation of the magnitude bits (so -0.0 and +0.0 both map to 0).
template <class T> inline uint32_t d_u32(T v) { return (uint32_t)v; }
template <> inline uint32_t d_u32<float>(float v) {
    uint32_t u; std::memcpy(&u, &v, 4);
    if (u & 0x80000000u) u = 0u - (u & 0x7FFFFFFFu);
    return u;
}
template <class T> inline uint64_t d_u64(T v) { return (uint64_t)v; }
// built_in.h:450-457 as the reference runs it on the GPU (NVRTC-compiled; recorded by
// tests/golden/make_ref_fixtures.py in tests/golden/ref_keymap_probe.json): negative
// finite values and -0.0 map to 0 - |bits| as the source reads, but a negative NaN maps to
// (0 - |bits|) with bit 63 clear, its signalling payload first quietened (bit 51 set) -- so
// -NaN orders just above +0.0.  The same source compiled for the CPU keeps bit 63
// (tests/golden/builtin_h_probe.json); the sort follows the GPU.
template <> inline uint64_t d_u64<double>(double v) {
    uint64_t u; std::memcpy(&u, &v, 8);
    if (u & 0x8000000000000000ull) {
        uint64_t mag = u & 0x7FFFFFFFFFFFFFFFull;
        const bool nan = mag > 0x7FF0000000000000ull;
        if (nan) mag |= 0x0008000000000000ull;
        u = 0ull - mag;
        if (nan) u &= 0x7FFFFFFFFFFFFFFFull;
    }
    return u;
}

template <class T> struct KeyW { typedef uint32_t U; static U map(T v) { return d_u32<T>(v); } };
template <> struct KeyW<int64_t> { typedef uint64_t U; static U map(int64_t v) { return d_u64(v); } };
template <> struct KeyW<uint64_t> { typedef uint64_t U; static U map(uint64_t v) { return d_u64(v); } };
template <> struct KeyW<double> { typedef uint64_t U; static U map(double v) { return d_u64<double>(v); } };

// ---- TRTC_Min_Element, extrema.cpp:5-13, evaluated through general_reduce
// (internal/general_reduce.cpp:30-95): round 1 runs blocks of 256 consecutive indices; inside
// a block, for s = 128, 64, ..., 1: if (tid < s && i + s < n) h[tid] = op(h[tid], h[tid+s]);
// block result is h[0].  Later rounds apply the same tree to the block results until one
// remains.  op(i1, i2) = vec[i2] < vec[i1] ? i2 : i1 (a NaN on the left absorbs its subtree).
template <class T> uint64_t min_element_tree(const T* v, uint64_t n) {
    if (n == 0) return 0;
    std::vector<uint64_t> cur(n);
    for (uint64_t i = 0; i < n; i++) cur[i] = i;
    bool first = true;
    while (first || cur.size() > 1) {
        first = false;
        uint64_t m = cur.size();
        uint64_t blocks = (m + 255) / 256;
        std::vector<uint64_t> nxt(blocks);
        for (uint64_t b = 0; b < blocks; b++) {
            uint64_t L = std::min<uint64_t>(256, m - b * 256);
            uint64_t h[256];
            for (uint64_t t = 0; t < L; t++) h[t] = cur[b * 256 + t];
            for (uint64_t s = 128; s > 0; s >>= 1)
                for (uint64_t t = 0; t < s; t++)
                    if (t + s < L) {
                        uint64_t i1 = h[t], i2 = h[t + s];
                        h[t] = v[i2] < v[i1] ? i2 : i1;
                    }
            nxt[b] = h[0];
        }
        cur.swap(nxt);
    }
    return cur[0];
}

// ---- radix sort ordering key, internal/radix_sort.cpp:11-58,165-553: the sort orders by
// key' = (d(x) - d(keys[id_min])) mod 2^w over the bits of mask = OR_i key'_i; ascending
// (Less) splits bit==0 first, descending (Greater) splits bit==1 first, stable, LSD.  A
// stable LSD split over the varying bits is exactly a stable sort by key' (asc) or by key'
// descending, which is what this fast form computes.
template <class T> void sort_perm(const T* v, uint64_t n, int desc, uint64_t* perm) {
    typedef typename KeyW<T>::U U;
    uint64_t m = min_element_tree(v, n);
    U dm = KeyW<T>::map(v[m]);
    std::vector<U> kp(n);
    for (uint64_t i = 0; i < n; i++) kp[i] = (U)(KeyW<T>::map(v[i]) - dm);
    std::vector<uint64_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    if (desc)
        std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) { return kp[a] > kp[b]; });
    else
        std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) { return kp[a] < kp[b]; });
    std::memcpy(perm, idx.data(), n * 8);
}

// Literal restatement of the 1-bit split loop (internal/radix_sort.cpp:184-197 and the
// partition scan/scatter of :47-163), for cross-checking the fast form on small inputs.
template <class T> void sort_perm_bitsplit(const T* v, uint64_t n, int desc, uint64_t* perm) {
    typedef typename KeyW<T>::U U;
    const int W = sizeof(U) * 8;
    uint64_t m = min_element_tree(v, n);
    U dm = KeyW<T>::map(v[m]);
    U mask = 0;
    for (uint64_t i = 0; i < n; i++) mask |= (U)(KeyW<T>::map(v[i]) - dm);
    std::vector<uint64_t> cur(n), nxt(n);
    std::iota(cur.begin(), cur.end(), 0);
    for (int bit = 0; bit < W; bit++) {
        if (!((mask >> bit) & 1)) continue;
        uint64_t w = 0;
        for (int side = 0; side < 2; side++)
            for (uint64_t i = 0; i < n; i++) {
                U kp = (U)(KeyW<T>::map(v[cur[i]]) - dm);
                int b = (int)((kp >> bit) & 1);
                int first = desc ? 1 : 0;
                if ((side == 0) == (b == first)) nxt[w++] = cur[i];
            }
        cur.swap(nxt);
    }
    std::memcpy(perm, cur.data(), n * 8);
}

// ---- scans, scan.cpp:4-39 + internal/general_scan.cpp: inclusive out[i] = in[0] op ... op in[i];
// exclusive out[0] = init, out[i] = init op in[0] op ... op in[i-1].  Sequential left fold in
// the value type (integer Plus wraps); floating point here is the sequential fold, the FP64
// variant below is the tolerance reference.
template <class T> void scan_native(int op, int excl, const T* in, uint64_t n, const T* init, T* out) {
    if (n == 0) return;
    if (excl) {
        T acc = *init;
        for (uint64_t i = 0; i < n; i++) { T x = in[i]; out[i] = acc; acc = op_apply<T>(op, acc, x); }
    } else {
        T acc = in[0];
        out[0] = acc;
        for (uint64_t i = 1; i < n; i++) { acc = op_apply<T>(op, acc, in[i]); out[i] = acc; }
    }
}
template <class T> void scan_f64(int op, int excl, const T* in, uint64_t n, const T* init, double* out) {
    if (n == 0) return;
    if (excl) {
        double acc = (double)*init;
        for (uint64_t i = 0; i < n; i++) { double x = (double)in[i]; out[i] = acc; acc = op_apply<double>(op, acc, x); }
    } else {
        double acc = (double)in[0];
        out[0] = acc;
        for (uint64_t i = 1; i < n; i++) { acc = op_apply<double>(op, acc, (double)in[i]); out[i] = acc; }
    }
}

// ---- scan_by_key, scan_by_key.cpp:4-53 + internal/general_scan_by_key.cpp:8-143.  A segment
// continues at i while key[i-1] == key[i] (EqualTo).  Inclusive: out[i] = head ? v[i] :
// out[i-1] op v[i].  Exclusive: src(i) = continues ? v[i-1] : init, then the same segmented
// inclusive scan of src -- i.e. out[head] = init, out[i] = out[i-1] op v[i-1].
template <class K, class T, class A>
void scan_by_key_gen(int op, int excl, const K* keys, const T* vals, uint64_t n, A init, A* out) {
    if (n == 0) return;
    A acc = 0;
    for (uint64_t i = 0; i < n; i++) {
        bool cont = i > 0 && keys[i - 1] == keys[i];
        if (excl) {
            A src = cont ? (A)vals[i - 1] : init;
            acc = cont ? op_apply<A>(op, acc, src) : src;
        } else {
            A x = (A)vals[i];
            acc = cont ? op_apply<A>(op, acc, x) : x;
        }
        out[i] = acc;
    }
}

// ---- reduce, reduce.cpp:5-31 + internal/general_reduce.cpp.  With init, the reduced
// sequence is (init, v0, v1, ..., v_{n-1}) (init spliced in as element 0 of n+1).
template <class T> T reduce_native(int op, const T* in, uint64_t n, const T* init) {
    T acc;
    uint64_t i = 0;
    if (init) acc = *init;
    else { acc = in[0]; i = 1; }
    for (; i < n; i++) acc = op_apply<T>(op, acc, in[i]);
    return acc;
}
template <class T> double reduce_f64(int op, const T* in, uint64_t n, const T* init) {
    double acc;
    uint64_t i = 0;
    if (init) acc = (double)*init;
    else { acc = (double)in[0]; i = 1; }
    for (; i < n; i++) acc = op_apply<double>(op, acc, (double)in[i]);
    return acc;
}
// The reference's association order: 256-wide strided trees over consecutive blocks,
// applied recursively (internal/general_reduce.cpp:30-95).  Used as an FP diagnostic.
template <class T> T reduce_tree(int op, const T* in, uint64_t n, const T* init) {
    uint64_t N = n + (init ? 1 : 0);
    std::vector<T> cur(N);
    for (uint64_t i = 0; i < N; i++) cur[i] = init ? (i == 0 ? *init : in[i - 1]) : in[i];
    bool first = true;
    while (first || cur.size() > 1) {
        first = false;
        uint64_t m = cur.size(), blocks = (m + 255) / 256;
        std::vector<T> nxt(blocks);
        for (uint64_t b = 0; b < blocks; b++) {
            uint64_t L = std::min<uint64_t>(256, m - b * 256);
            T h[256];
            for (uint64_t t = 0; t < L; t++) h[t] = cur[b * 256 + t];
            for (uint64_t s = 128; s > 0; s >>= 1)
                for (uint64_t t = 0; t < s; t++)
                    if (t + s < L) h[t] = op_apply<T>(op, h[t], h[t + s]);
            nxt[b] = h[0];
        }
        cur.swap(nxt);
    }
    return cur[0];
}

#define DISPATCH_ALL(type, FN)                         \
    switch (type) {                                    \
        case T_I8: FN(int8_t); break;                  \
        case T_U8: FN(uint8_t); break;                 \
        case T_I16: FN(int16_t); break;                \
        case T_U16: FN(uint16_t); break;               \
        case T_I32: FN(int32_t); break;                \
        case T_U32: FN(uint32_t); break;               \
        case T_I64: FN(int64_t); break;                \
        case T_U64: FN(uint64_t); break;               \
        case T_F32: FN(float); break;                  \
        case T_F64: FN(double); break;                 \
        default: return -1;                            \
    }

// ---- the same stable order as sort_perm for 32-bit keys, computed with `threads` host
// threads: (key' << 32 | index) packed in 64-bit words sorts stably with an unstable sort
// (the index breaks ties); chunks are sorted in parallel and merged pairwise.  Used as the
// timed host baseline of a pair sort; the order is that of internal/radix_sort.cpp:328-343.
template <class T> void sort_pairs_packed(const T* keys, const uint32_t* vals, uint64_t n, int desc, int threads,
                                          T* keys_out, uint32_t* vals_out) {
    const uint64_t m = min_element_tree(keys, n);
    const uint32_t dm = KeyW<T>::map(keys[m]);
    std::vector<uint64_t> w(n), tmp(n);
    if (threads < 1) threads = 1;
    auto par = [&](auto&& fn) {
        std::vector<std::thread> th;
        for (int t = 0; t < threads; t++) th.emplace_back(fn, t);
        for (auto& x : th) x.join();
    };
    par([&](int t) {
        const uint64_t a = n * t / threads, b = n * (t + 1) / threads;
        for (uint64_t i = a; i < b; i++) {
            uint32_t k = (uint32_t)(KeyW<T>::map(keys[i]) - dm);
            if (desc) k = ~k;  // descending by key', ties still by index
            w[i] = ((uint64_t)k << 32) | i;
        }
        std::sort(w.begin() + a, w.begin() + b);
    });
    std::vector<uint64_t> bounds(threads + 1);
    for (int t = 0; t <= threads; t++) bounds[t] = n * t / threads;
    while (bounds.size() > 2) {
        std::vector<uint64_t> nb;
        std::vector<std::thread> th;
        for (size_t j = 0; j + 1 < bounds.size(); j += 2) {
            if (j + 2 < bounds.size()) {
                const uint64_t a = bounds[j], mid = bounds[j + 1], b = bounds[j + 2];
                th.emplace_back([&, a, mid, b] { std::merge(w.begin() + a, w.begin() + mid, w.begin() + mid, w.begin() + b, tmp.begin() + a); });
                nb.push_back(a);
            } else {
                const uint64_t a = bounds[j], b = bounds[j + 1];
                th.emplace_back([&, a, b] { std::copy(w.begin() + a, w.begin() + b, tmp.begin() + a); });
                nb.push_back(a);
            }
        }
        for (auto& x : th) x.join();
        nb.push_back(n);
        bounds.swap(nb);
        w.swap(tmp);
    }
    par([&](int t) {
        const uint64_t a = n * t / threads, b = n * (t + 1) / threads;
        for (uint64_t i = a; i < b; i++) {
            const uint64_t src = w[i] & 0xFFFFFFFFull;
            keys_out[i] = keys[src];
            vals_out[i] = vals[src];
        }
    });
}

}  // namespace

extern "C" {

// stable pair sort of 32-bit keys with 32-bit values on `threads` host threads (n < 2^32)
int oracle_sort_pairs32(int type, const void* keys, const void* vals, unsigned long long n, int desc, int threads,
                        void* keys_out, void* vals_out) {
    if (n == 0) return 0;
    if (n >= (1ull << 32)) return -1;
    const uint32_t* v = (const uint32_t*)vals;
    uint32_t* vo = (uint32_t*)vals_out;
    switch (type) {
        case T_I32: sort_pairs_packed<int32_t>((const int32_t*)keys, v, n, desc, threads, (int32_t*)keys_out, vo); break;
        case T_U32: sort_pairs_packed<uint32_t>((const uint32_t*)keys, v, n, desc, threads, (uint32_t*)keys_out, vo); break;
        case T_F32: sort_pairs_packed<float>((const float*)keys, v, n, desc, threads, (float*)keys_out, vo); break;
        default: return -1;
    }
    return 0;
}

unsigned long long oracle_min_element(int type, const void* keys, unsigned long long n) {
    unsigned long long r = 0;
#define FN(T) r = min_element_tree<T>((const T*)keys, n)
    switch (type) {
        case T_I8: FN(int8_t); break;
        case T_U8: FN(uint8_t); break;
        case T_I16: FN(int16_t); break;
        case T_U16: FN(uint16_t); break;
        case T_I32: FN(int32_t); break;
        case T_U32: FN(uint32_t); break;
        case T_I64: FN(int64_t); break;
        case T_U64: FN(uint64_t); break;
        case T_F32: FN(float); break;
        case T_F64: FN(double); break;
        default: return ~0ull;
    }
#undef FN
    return r;
}

int oracle_keymap(int type, const void* keys, unsigned long long n, unsigned long long* out) {
#define FN(T) for (unsigned long long i = 0; i < n; i++) out[i] = KeyW<T>::map(((const T*)keys)[i])
    DISPATCH_ALL(type, FN)
#undef FN
    return 0;
}

int oracle_sort_perm(int type, const void* keys, unsigned long long n, int desc, unsigned long long* perm) {
    if (n == 0) return 0;
#define FN(T) sort_perm<T>((const T*)keys, n, desc, (uint64_t*)perm)
    DISPATCH_ALL(type, FN)
#undef FN
    return 0;
}

int oracle_sort_perm_bitsplit(int type, const void* keys, unsigned long long n, int desc, unsigned long long* perm) {
    if (n == 0) return 0;
#define FN(T) sort_perm_bitsplit<T>((const T*)keys, n, desc, (uint64_t*)perm)
    DISPATCH_ALL(type, FN)
#undef FN
    return 0;
}

int oracle_scan(int type, int op, int excl, const void* in, unsigned long long n, const void* init, void* out) {
#define FN(T) scan_native<T>(op, excl, (const T*)in, n, (const T*)init, (T*)out)
    DISPATCH_ALL(type, FN)
#undef FN
    return 0;
}

int oracle_scan_f64(int type, int op, int excl, const void* in, unsigned long long n, const void* init, double* out) {
#define FN(T) scan_f64<T>(op, excl, (const T*)in, n, (const T*)init, out)
    DISPATCH_ALL(type, FN)
#undef FN
    return 0;
}

// keys int32 or int64 (ktype 4/6), values of any type; native accumulation (out has the
// value type) or FP64 accumulation (out_f64, when non-null).
int oracle_scan_by_key(int ktype, int vtype, int op, int excl, const void* keys, const void* vals,
                       unsigned long long n, const void* init, void* out, double* out_f64) {
#define FNK(K)                                                                                   \
    {                                                                                            \
        const K* kk = (const K*)keys;                                                            \
        switch (vtype) {                                                                         \
            case T_I32: if (out_f64) scan_by_key_gen<K, int32_t, double>(op, excl, kk, (const int32_t*)vals, n, init ? (double)*(const int32_t*)init : 0.0, out_f64); \
                        else scan_by_key_gen<K, int32_t, int32_t>(op, excl, kk, (const int32_t*)vals, n, init ? *(const int32_t*)init : 0, (int32_t*)out); break; \
            case T_U32: if (out_f64) scan_by_key_gen<K, uint32_t, double>(op, excl, kk, (const uint32_t*)vals, n, init ? (double)*(const uint32_t*)init : 0.0, out_f64); \
                        else scan_by_key_gen<K, uint32_t, uint32_t>(op, excl, kk, (const uint32_t*)vals, n, init ? *(const uint32_t*)init : 0u, (uint32_t*)out); break; \
            case T_I64: if (out_f64) scan_by_key_gen<K, int64_t, double>(op, excl, kk, (const int64_t*)vals, n, init ? (double)*(const int64_t*)init : 0.0, out_f64); \
                        else scan_by_key_gen<K, int64_t, int64_t>(op, excl, kk, (const int64_t*)vals, n, init ? *(const int64_t*)init : 0, (int64_t*)out); break; \
            case T_F32: if (out_f64) scan_by_key_gen<K, float, double>(op, excl, kk, (const float*)vals, n, init ? (double)*(const float*)init : 0.0, out_f64); \
                        else scan_by_key_gen<K, float, float>(op, excl, kk, (const float*)vals, n, init ? *(const float*)init : 0.f, (float*)out); break; \
            case T_F64: if (out_f64) scan_by_key_gen<K, double, double>(op, excl, kk, (const double*)vals, n, init ? *(const double*)init : 0.0, out_f64); \
                        else scan_by_key_gen<K, double, double>(op, excl, kk, (const double*)vals, n, init ? *(const double*)init : 0.0, (double*)out); break; \
            default: return -1;                                                                  \
        }                                                                                        \
    }
    switch (ktype) {
        case T_I32: FNK(int32_t); break;
        case T_U32: FNK(uint32_t); break;
        case T_I64: FNK(int64_t); break;
        case T_U64: FNK(uint64_t); break;
        default: return -1;
    }
#undef FNK
    return 0;
}

int oracle_reduce(int type, int op, const void* in, unsigned long long n, const void* init, void* out) {
    if (n == 0 && !init) return -1;  // general_reduce refuses n < 1 (internal/general_reduce.cpp:57)
#define FN(T) *(T*)out = reduce_native<T>(op, (const T*)in, n, (const T*)init)
    DISPATCH_ALL(type, FN)
#undef FN
    return 0;
}

int oracle_reduce_f64(int type, int op, const void* in, unsigned long long n, const void* init, double* out) {
    if (n == 0 && !init) return -1;
#define FN(T) *out = reduce_f64<T>(op, (const T*)in, n, (const T*)init)
    DISPATCH_ALL(type, FN)
#undef FN
    return 0;
}

int oracle_reduce_tree(int type, int op, const void* in, unsigned long long n, const void* init, void* out) {
    if (n == 0 && !init) return -1;
#define FN(T) *(T*)out = reduce_tree<T>(op, (const T*)in, n, (const T*)init)
    DISPATCH_ALL(type, FN)
#undef FN
    return 0;
}

}  // extern "C"
