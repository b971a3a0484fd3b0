// launch_scan.cu -- nvcc instantiations of the scan / reduce / scan_by_key / compaction
// kernels for the built-in element types and operators (Plus, Maximum, Minimum, EqualTo).
#include "trtc_launch.h"
#include "trtc_runtime.h"
#include "../device/trtc_compact.cuh"

namespace trtc_host {

using namespace trtc;

static constexpr int SCAN_BLOCK = 256;
// L2 prefetch distance of the persistent tile kernels, in quarter grids (B200, 2^28 i32 scan
// per launch: 0.3542 / 0.3558 / 0.3569 / 0.3606 / 0.4944 ms at 1/4, 1/2, 3/4, 1 and 2 grids;
// scan_by_key and unique flat within 0.5 % up to one grid; half a grid kept, in the middle
// of the flat range)
#ifndef TRTC_TILE_PF_X4
#define TRTC_TILE_PF_X4 2
#endif

template <class E> static constexpr int scan_nv() { return VecWidth<E>::V >= 16 ? 1 : 16 / VecWidth<E>::V; }

static bool fill_lookback(LookbackState& st, cudaStream_t s, size_t tiles, size_t vsize, bool seg = false) {
    uint32_t e4 = 0;
    LookbackWs* w = lookback_ws(s, tiles, vsize, &e4);
    if (!w) return false;
    st.flags = w->flags;
    st.agg = w->agg;
    st.incl = w->incl;
    st.packed = w->packed;
    st.tile_ctr = w->tile_ctr;
    st.epoch8 = e4;
    st.err = device_error_word();
    st.result = w->result;
    return true;
}

#ifndef TRTC_SCAN2_ITEMS
#define TRTC_SCAN2_ITEMS 32  // elements per thread of a two-phase scan tile (4-byte types)
#endif

template <class T, class Op, int MODE>
static bool scan_t(const T* in, T* out, size_t n, const T* init, cudaStream_t s) {
    T ini = init ? *init : T();
    if constexpr (VecWidth<T>::V > 1) {
        // two-phase tiles: TRTC_SCAN2_ITEMS elements per thread for 4-byte types, the same
        // bytes per thread for other widths
        constexpr int ITEMS = TRTC_SCAN2_ITEMS * 4 / (int)sizeof(T) < VecWidth<T>::V
                                  ? VecWidth<T>::V : TRTC_SCAN2_ITEMS * 4 / (int)sizeof(T);
        constexpr int TILE = SCAN_BLOCK * ITEMS;
        const size_t tiles = (n + TILE - 1) / TILE;
        LookbackState st;
        if (!fill_lookback(st, s, tiles, sizeof(T))) return false;
        // persistent CTAs: as many as fit on the device at once
        auto kernel = scan2_kernel<T, Op, MODE, SCAN_BLOCK, ITEMS, true>;
        static int per_sm = 0;
        if (per_sm == 0 && !TRTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, SCAN_BLOCK, 0)))
            return false;
        size_t grid = (size_t)(per_sm > 0 ? per_sm : 1) * sm_count();
        if (grid > tiles) grid = tiles;
        st.pf_ahead = tile_prefetch_ahead(grid * TRTC_TILE_PF_X4 / 4);
        ktimer_mark("", s);
        kernel<<<(unsigned)grid, SCAN_BLOCK, 0, s>>>(in, out, n, tiles, Op(), ini, st);
        count_launch();
        ktimer_mark("scan_kernel", s);
        return TRTC_CUDA(cudaGetLastError());
    } else {
        constexpr int NV = scan_nv<T>();
        constexpr int TILE = SCAN_BLOCK * NV * VecWidth<T>::V;
        const size_t tiles = (n + TILE - 1) / TILE;
        LookbackState st;
        if (!fill_lookback(st, s, tiles, sizeof(T))) return false;
        VectorView<T> iv = make_view<T>(const_cast<T*>(in), n);
        VectorView<T> ov = make_view<T>(out, n);
        ktimer_mark("", s);
        scan_kernel<VectorView<T>, Nothing, false, VectorView<T>, T, Op, MODE, SCAN_BLOCK, NV>
            <<<(unsigned)tiles, SCAN_BLOCK, 0, s>>>(iv, Nothing(), ov, n, Op(), ini, st);
        count_launch();
        ktimer_mark("scan_kernel", s);
        return TRTC_CUDA(cudaGetLastError());
    }
}

template <class T>
static bool scan_op(int op, int mode, const void* in, void* out, size_t n, const void* init, cudaStream_t s) {
    const T* i = (const T*)in;
    T* o = (T*)out;
    const T* ini = (const T*)init;
    switch (op * 2 + mode) {
        case 0: return scan_t<T, Plus, 0>(i, o, n, ini, s);
        case 1: return scan_t<T, Plus, 1>(i, o, n, ini, s);
        case 2: return scan_t<T, Maximum, 0>(i, o, n, ini, s);
        case 3: return scan_t<T, Maximum, 1>(i, o, n, ini, s);
        case 4: return scan_t<T, Minimum, 0>(i, o, n, ini, s);
        case 5: return scan_t<T, Minimum, 1>(i, o, n, ini, s);
        default: set_error("scan: unsupported operator"); return false;
    }
}

bool scan_raw(int tc, int op, int mode, const void* in, void* out, size_t n, const void* init, cudaStream_t s) {
    if (n == 0) { set_error("scan: empty input"); return false; }
    switch (tc) {
        case TC_I8: return scan_op<int8_t>(op, mode, in, out, n, init, s);
        case TC_U8: return scan_op<uint8_t>(op, mode, in, out, n, init, s);
        case TC_I16: return scan_op<int16_t>(op, mode, in, out, n, init, s);
        case TC_U16: return scan_op<uint16_t>(op, mode, in, out, n, init, s);
        case TC_I32: return scan_op<int32_t>(op, mode, in, out, n, init, s);
        case TC_U32: return scan_op<uint32_t>(op, mode, in, out, n, init, s);
        case TC_I64: return scan_op<int64_t>(op, mode, in, out, n, init, s);
        case TC_U64: return scan_op<uint64_t>(op, mode, in, out, n, init, s);
        case TC_F32: return scan_op<float>(op, mode, in, out, n, init, s);
        case TC_F64: return scan_op<double>(op, mode, in, out, n, init, s);
        default: set_error("scan: unsupported type"); return false;
    }
}

// ---------------------------------------------------------------- reduce
template <class T, class Op>
static bool reduce_t(const T* in, size_t n, const T* init, void** result_dev, cudaStream_t s) {
    constexpr int BLOCK = 256;
    const size_t nvec = n / VecWidth<T>::V;
    size_t grid = (nvec + BLOCK - 1) / BLOCK;
    const size_t cap = (size_t)sm_count() * 8;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    LookbackWs* w = reduce_ws(s, grid, sizeof(T));
    if (!w) return false;
    ktimer_mark("", s);
    reduce_kernel<T, T, Op, Identity, false, BLOCK><<<(unsigned)grid, BLOCK, 0, s>>>(
        in, n, Op(), Identity(), (T*)w->partials, w->partial_has, w->done_ctr, (T*)w->result, init ? 1 : 0,
        init ? *init : T());
    count_launch();
    ktimer_mark("reduce_kernel", s);
    *result_dev = w->result;
    return TRTC_CUDA(cudaGetLastError());
}

template <class T>
static bool reduce_op(int op, const void* in, size_t n, const void* init, void** res, cudaStream_t s) {
    switch (op) {
        case OP_PLUS: return reduce_t<T, Plus>((const T*)in, n, (const T*)init, res, s);
        case OP_MAX: return reduce_t<T, Maximum>((const T*)in, n, (const T*)init, res, s);
        case OP_MIN: return reduce_t<T, Minimum>((const T*)in, n, (const T*)init, res, s);
        default: set_error("reduce: unsupported operator"); return false;
    }
}

bool reduce_raw_async(int tc, int op, const void* in, size_t n, const void* init, void** res, cudaStream_t s) {
    if (n == 0 && !init) { set_error("reduce: empty input without an initial value"); return false; }
    switch (tc) {
        case TC_I8: return reduce_op<int8_t>(op, in, n, init, res, s);
        case TC_U8: return reduce_op<uint8_t>(op, in, n, init, res, s);
        case TC_I16: return reduce_op<int16_t>(op, in, n, init, res, s);
        case TC_U16: return reduce_op<uint16_t>(op, in, n, init, res, s);
        case TC_I32: return reduce_op<int32_t>(op, in, n, init, res, s);
        case TC_U32: return reduce_op<uint32_t>(op, in, n, init, res, s);
        case TC_I64: return reduce_op<int64_t>(op, in, n, init, res, s);
        case TC_U64: return reduce_op<uint64_t>(op, in, n, init, res, s);
        case TC_F32: return reduce_op<float>(op, in, n, init, res, s);
        case TC_F64: return reduce_op<double>(op, in, n, init, res, s);
        default: set_error("reduce: unsupported type"); return false;
    }
}

bool reduce_raw(int tc, int op, const void* in, size_t n, const void* init, void* result_host, cudaStream_t s) {
    void* rd = nullptr;
    if (!reduce_raw_async(tc, op, in, n, init, &rd, s)) return false;
    return TRTC_CUDA(cudaMemcpyAsync(result_host, rd, type_size(tc), cudaMemcpyDeviceToHost, s)) &&
           check_device_errors(s, "reduce");
}

// ---------------------------------------------------------------- scan_by_key
#ifndef TRTC_SBK2
#define TRTC_SBK2 1  // two-phase segmented scan for keys and values of one width
#endif
// B200, 2^28 i32 keys / f32 values in runs of ~32.  Row form: 8 items at 2 / 5 CTAs per SM
// 1.36 / 0.99 ms, 12 items at 4 CTAs 0.93 ms, 16 items at 3 CTAs 1.06 ms.  Blocked form
// (TRTC_SBK2_BLOCKED): 12 items at 4 / 5 / 6 CTAs 0.87 / 0.80 / 0.87 ms, 16 items at 4 CTAs
// 1.14 ms, 8 items at 6 / 8 CTAs 0.98 / 0.93 ms.  Drawing the next ticket during the
// look-back (TRTC_SBK2_AHEAD) gained nothing in either form.
#ifndef TRTC_SBK2_ITEMS
#define TRTC_SBK2_ITEMS 12  // elements per thread of a two-phase segmented-scan tile (4-byte types)
#endif

template <class K, class T, int MODE>
static bool sbk_t(const K* keys, const T* vals, T* out, size_t n, const T* init, cudaStream_t s) {
    const bool out_over_keys = (const void*)out < (const void*)(keys + n) && (const void*)keys < (const void*)(out + n);
    if constexpr (TRTC_SBK2 && sizeof(K) == sizeof(T) && (sizeof(T) == 4 || sizeof(T) == 8)) {
        if (!out_over_keys) {
            constexpr int ITEMS = TRTC_SBK2_ITEMS * 4 / (int)sizeof(T) < VecWidth<T>::V
                                      ? VecWidth<T>::V : TRTC_SBK2_ITEMS * 4 / (int)sizeof(T);
            constexpr int TILE = SCAN_BLOCK * ITEMS;
            const size_t tiles = (n + TILE - 1) / TILE;
            LookbackState st;
            if (!fill_lookback(st, s, tiles, sizeof(T), true)) return false;
            // persistent CTAs: as many as fit on the device at once
            auto kernel = sbk2_kernel<K, T, MODE, SCAN_BLOCK, ITEMS>;
            static int per_sm = 0;
            if (per_sm == 0 && !TRTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, SCAN_BLOCK, 0)))
                return false;
            size_t grid = (size_t)(per_sm > 0 ? per_sm : 1) * sm_count();
            if (grid > tiles) grid = tiles;
            st.pf_ahead = tile_prefetch_ahead(grid * TRTC_TILE_PF_X4 / 4);
            ktimer_mark("", s);
            kernel<<<(unsigned)grid, SCAN_BLOCK, 0, s>>>(keys, vals, out, n, tiles, init ? *init : T(), st);
            count_launch();
            ktimer_mark("scan_by_key_kernel", s);
            return TRTC_CUDA(cudaGetLastError());
        }
    }
    constexpr int VK = VecWidth<K>::V, VT = VecWidth<T>::V;
    constexpr int VEC = VK > VT ? VK : VT;
    constexpr int NV = VEC >= 8 ? 2 : 4;
    constexpr int TILE = SCAN_BLOCK * NV * VEC;
    const size_t tiles = (n + TILE - 1) / TILE;
    LookbackState st;
    if (!fill_lookback(st, s, tiles, sizeof(T), true)) return false;
    VectorView<T> vv = make_view<T>(const_cast<T*>(vals), n);
    VectorView<K> kv = make_view<K>(const_cast<K*>(keys), n);
    VectorView<T> ov = make_view<T>(out, n);
    ktimer_mark("", s);
    scan_by_key_kernel<VectorView<K>, VectorView<T>, VectorView<T>, T, EqualTo, Plus, MODE, SCAN_BLOCK, NV>
        <<<(unsigned)tiles, SCAN_BLOCK, 0, s>>>(kv, vv, ov, n, EqualTo(), Plus(), init ? *init : T(), st);
    count_launch();
    ktimer_mark("scan_by_key_kernel", s);
    return TRTC_CUDA(cudaGetLastError());
}

template <class K>
static bool sbk_k(int vtc, int mode, const void* keys, const void* vals, void* out, size_t n, const void* init,
                  cudaStream_t s) {
    const K* k = (const K*)keys;
#define TRTC_SBK(T) return mode ? sbk_t<K, T, 1>(k, (const T*)vals, (T*)out, n, (const T*)init, s) \
                                : sbk_t<K, T, 0>(k, (const T*)vals, (T*)out, n, (const T*)init, s)
    switch (vtc) {
        case TC_I32: TRTC_SBK(int32_t);
        case TC_U32: TRTC_SBK(uint32_t);
        case TC_I64: TRTC_SBK(int64_t);
        case TC_F32: TRTC_SBK(float);
        case TC_F64: TRTC_SBK(double);
        default: set_error("scan_by_key: unsupported value type"); return false;
    }
#undef TRTC_SBK
}

bool scan_by_key_raw(int ktc, int vtc, int mode, const void* keys, const void* vals, void* out, size_t n,
                     const void* init, cudaStream_t s) {
    if (n == 0) { set_error("scan_by_key: empty input"); return false; }
    switch (ktc) {
        case TC_I32: return sbk_k<int32_t>(vtc, mode, keys, vals, out, n, init, s);
        case TC_U32: return sbk_k<uint32_t>(vtc, mode, keys, vals, out, n, init, s);
        case TC_I64: return sbk_k<int64_t>(vtc, mode, keys, vals, out, n, init, s);
        default: set_error("scan_by_key: unsupported key type"); return false;
    }
}

// ---------------------------------------------------------------- compaction (built-in selectors)
// B200, remove from 2^28 i32 (half kept): 32 items at 4 CTAs per SM 0.400 ms (64 registers,
// ~320 B of spills); 24 items at 4 / 5 CTAs 0.471 / 0.423 ms; 16 items at 4 / 6 CTAs
// 0.597 / 0.463 ms; 12 items at 6 CTAs 0.560 ms; 8 items at 8 CTAs 0.647 ms
#ifndef TRTC_COMPACT2_ITEMS
#define TRTC_COMPACT2_ITEMS 32  // elements per thread of a two-phase compaction tile
#endif
#ifndef TRTC_COMPACT2_GENERIC_ITEMS
#define TRTC_COMPACT2_GENERIC_ITEMS 16  // the same for the forms outside the 16-byte vector path
#endif

template <class T, int MODE, class CT>
static bool compact_t(const T* in, T* out, size_t n, const T* value, cudaStream_t s, unsigned long long* count) {
    const char* ib = (const char*)in;
    const char* ob = (const char*)out;
    const bool disjoint = ob + n * sizeof(T) <= ib || ib + n * sizeof(T) <= ob;
    if (!disjoint) {
        // in place: the two-phase kernel into a pool temporary, then the kept elements copied
        // back (2^28 i32, half kept: 0.42 + 0.17 ms against 1.06 ms for the one-pass kernel);
        // the one-pass kernel remains for when no temporary can be had
        T* tmp = (T*)tmp_alloc(n * sizeof(T), s);
        if (tmp) {
            unsigned long long c = 0;
            bool ok = compact_t<T, MODE, CT>(in, tmp, n, value, s, &c);
            if (ok && c > 0)
                ok = TRTC_CUDA(cudaMemcpyAsync(out, tmp, (size_t)c * sizeof(T), cudaMemcpyDeviceToDevice, s));
            tmp_free(tmp, s);
            *count = c;
            return ok;
        }
        (void)cudaGetLastError();  // the failed allocation must not fail the launch check below
    }
    // the vector path (4-byte elements: remove's element-wise test, unique's neighbour test)
    // takes TRTC_COMPACT2_ITEMS; other widths take TRTC_COMPACT2_GENERIC_ITEMS
    constexpr bool VEC = sizeof(T) == 4 && (MODE == CM_NOT_EQUAL || MODE == CM_UNIQUE);
    constexpr int ITEMS1 = 16, ITEMS2 = VEC ? TRTC_COMPACT2_ITEMS : TRTC_COMPACT2_GENERIC_ITEMS;
    const int ITEMS = disjoint ? ITEMS2 : ITEMS1;
    const size_t TILE = (size_t)SCAN_BLOCK * ITEMS;
    const size_t tiles = (n + TILE - 1) / TILE;
    LookbackState st;
    if (!fill_lookback(st, s, tiles, 8)) return false;
    VectorView<T> iv = make_view<T>(const_cast<T*>(in), n);
    VectorView<T> ov = make_view<T>(out, n);
    ktimer_mark("", s);
    if (disjoint) {
        // out-of-place: persistent two-phase tiles (the input is read twice, the second time
        // normally from L2)
        auto kernel = compact2_kernel<MODE, false, false, VectorView<T>, Nothing, EqualTo, T, VectorView<T>, Nothing,
                                      Nothing, Nothing, SCAN_BLOCK, ITEMS2, CT>;
        static int per_sm = 0;
        if (per_sm == 0 && !TRTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, SCAN_BLOCK, 0)))
            return false;
        size_t grid = (size_t)(per_sm > 0 ? per_sm : 1) * sm_count();
        if (grid > tiles) grid = tiles;
        st.pf_ahead = tile_prefetch_ahead(grid * TRTC_TILE_PF_X4 / 4);
        kernel<<<(unsigned)grid, SCAN_BLOCK, 0, s>>>(iv, Nothing(), EqualTo(), value ? *value : T(), ov, Nothing(),
                                                      Nothing(), Nothing(), n, tiles, st);
    } else {
        compact_kernel<MODE, false, false, VectorView<T>, Nothing, EqualTo, T, VectorView<T>, Nothing, Nothing,
                       Nothing, SCAN_BLOCK, ITEMS1, CT><<<(unsigned)tiles, SCAN_BLOCK, 0, s>>>(
            iv, Nothing(), EqualTo(), value ? *value : T(), ov, Nothing(), Nothing(), Nothing(), n, st);
    }
    count_launch();
    ktimer_mark("compact_kernel", s);
    if (!TRTC_CUDA(cudaGetLastError())) return false;
    return TRTC_CUDA(cudaMemcpyAsync(count, st.result, 8, cudaMemcpyDeviceToHost, s)) &&
           check_device_errors(s, "compaction");
}

template <class T>
static bool compact_m(int mode, const void* in, void* out, size_t n, const void* value, cudaStream_t s,
                      unsigned long long* count) {
    // 32-bit counts below 2^32 elements (packed look-back words)
    const bool c32 = n < (1ull << 32);
    if (mode == CM_NOT_EQUAL)
        return c32 ? compact_t<T, CM_NOT_EQUAL, uint32_t>((const T*)in, (T*)out, n, (const T*)value, s, count)
                   : compact_t<T, CM_NOT_EQUAL, unsigned long long>((const T*)in, (T*)out, n, (const T*)value, s, count);
    if (mode == CM_UNIQUE)
        return c32 ? compact_t<T, CM_UNIQUE, uint32_t>((const T*)in, (T*)out, n, nullptr, s, count)
                   : compact_t<T, CM_UNIQUE, unsigned long long>((const T*)in, (T*)out, n, nullptr, s, count);
    set_error("compaction: unsupported built-in mode");
    return false;
}

bool compact_raw(int tc, int mode, const void* in, void* out, size_t n, const void* value, cudaStream_t s,
                 unsigned long long* count) {
    if (n == 0) { set_error("compaction: empty input"); return false; }
    switch (tc) {
        case TC_I8: return compact_m<int8_t>(mode, in, out, n, value, s, count);
        case TC_U8: return compact_m<uint8_t>(mode, in, out, n, value, s, count);
        case TC_I16: return compact_m<int16_t>(mode, in, out, n, value, s, count);
        case TC_U16: return compact_m<uint16_t>(mode, in, out, n, value, s, count);
        case TC_I32: return compact_m<int32_t>(mode, in, out, n, value, s, count);
        case TC_U32: return compact_m<uint32_t>(mode, in, out, n, value, s, count);
        case TC_I64: return compact_m<int64_t>(mode, in, out, n, value, s, count);
        case TC_U64: return compact_m<uint64_t>(mode, in, out, n, value, s, count);
        case TC_F32: return compact_m<float>(mode, in, out, n, value, s, count);
        case TC_F64: return compact_m<double>(mode, in, out, n, value, s, count);
        default: set_error("compaction: unsupported type"); return false;
    }
}

}  // namespace trtc_host
