// trtc_algorithms.cpp -- the TRTC_* hot-path algorithms (sort.h, scan.h, transform_scan.h,
// reduce.h, transform_reduce.h, extrema.h, copy.h, remove.h, unique.h, partition.h).
//
// Dispatch: contiguous vectors (DVVector, DVVectorAdaptor, ranges of them) of built-in
// element types with built-in operators run the nvcc-built kernels; anything involving a
// user Functor, a computed view (counter, constant, permutation, ...) or a non-arithmetic
// element type instantiates the same kernel templates through NVRTC.  All work is issued on
// the legacy default stream, like the reference, and calls that return a host value
// (counts, reductions) synchronise as the reference's blocking copies do.
#include "thrustrtc_cpp.h"
#include "trtc_jit.h"
#include "trtc_launch.h"
#include "trtc_runtime.h"
#include "../device/trtc_abi.h"

#include <cstdio>
#include <memory>

using namespace trtc_host;

namespace {

cudaStream_t S() { return (cudaStream_t)0; }

const char* k_nothing = "trtc::Nothing";

ViewBuf nothing_bytes() { return ViewBuf(1, 0); }

template <class T>
ViewBuf pod_bytes(const T& v) {
    ViewBuf b(sizeof(T));
    memcpy(b.data(), &v, sizeof(T));
    return b;
}

int builtin_op_code(const Functor& f) {
    if (!f.is_built_in()) return -1;
    const std::string& n = f.name_view_cls();
    if (n == "Plus") return OP_PLUS;
    if (n == "Maximum") return OP_MAX;
    if (n == "Minimum") return OP_MIN;
    return -1;
}

bool is_builtin(const Functor& f, const char* name) { return f.is_built_in() && f.name_view_cls() == name; }

bool is_vector_view(const DeviceViewable& v) { return v.name_view_cls().compare(0, 11, "VectorView<") == 0; }

int vec_width(size_t esize) {
    return (esize == 1 || esize == 2 || esize == 4 || esize == 8 || esize == 16) ? (int)(16 / esize) : 1;
}

std::string num(long long v) { return std::to_string(v); }

// A DVVectorLike as a kernel view parameter: contiguous vectors pass as VectorView of their
// first element (a DVRange over a DVVector becomes a plain VectorView), others as themselves.
struct ViewArg {
    std::string type;
    ViewBuf bytes;
    bool contiguous = false;
};
ViewArg view_arg(const DVVectorLike& v) {
    ViewArg a;
    void* p = v.contiguous_data();
    if (p) {
        a.type = "VectorView<" + v.name_elem_cls() + ">";
        a.bytes.resize(16);
        unsigned long long s = v.size();
        memcpy(a.bytes.data(), &p, 8);
        memcpy(a.bytes.data() + 8, &s, 8);
        a.contiguous = true;
    } else {
        a.type = v.name_view_cls();
        a.bytes = v.view();
    }
    return a;
}
ViewArg raw_view(void* p, size_t n, const std::string& elem) {
    ViewArg a;
    a.type = "VectorView<" + elem + ">";
    a.bytes.resize(16);
    unsigned long long s = n;
    memcpy(a.bytes.data(), &p, 8);
    memcpy(a.bytes.data() + 8, &s, 8);
    a.contiguous = true;
    return a;
}

// value of a scalar DeviceViewable converted to the named built-in type (host conversion,
// the same C++ conversion the reference's generated code applies on the device)
bool convert_scalar(const DeviceViewable& dv, const std::string& to, ViewBuf& out) {
    if (dv.name_view_cls() == to) { out = dv.view(); return true; }
    const int ft = type_code_of(dv.name_view_cls()), tt = type_code_of(to);
    const bool fb = dv.name_view_cls() == "bool";
    if ((ft < 0 && !fb) || tt < 0) return false;
    const ViewBuf in = dv.view();
    double d = 0;
    long long i = 0;
    unsigned long long u = 0;
    bool is_f = false, is_u = false;
    switch (fb ? -2 : ft) {
        case -2: i = *(const bool*)in.data(); break;
        case TC_I8: i = *(const int8_t*)in.data(); break;
        case TC_U8: u = *(const uint8_t*)in.data(); is_u = true; break;
        case TC_I16: i = *(const int16_t*)in.data(); break;
        case TC_U16: u = *(const uint16_t*)in.data(); is_u = true; break;
        case TC_I32: i = *(const int32_t*)in.data(); break;
        case TC_U32: u = *(const uint32_t*)in.data(); is_u = true; break;
        case TC_I64: i = *(const int64_t*)in.data(); break;
        case TC_U64: u = *(const uint64_t*)in.data(); is_u = true; break;
        case TC_F32: d = *(const float*)in.data(); is_f = true; break;
        case TC_F64: d = *(const double*)in.data(); is_f = true; break;
    }
#define TRTC_CONV(T) { T v = is_f ? (T)d : (is_u ? (T)u : (T)i); out = pod_bytes<T>(v); return true; }
    switch (tt) {
        case TC_I8: TRTC_CONV(int8_t)
        case TC_U8: TRTC_CONV(uint8_t)
        case TC_I16: TRTC_CONV(int16_t)
        case TC_U16: TRTC_CONV(uint16_t)
        case TC_I32: TRTC_CONV(int32_t)
        case TC_U32: TRTC_CONV(uint32_t)
        case TC_I64: TRTC_CONV(int64_t)
        case TC_U64: TRTC_CONV(uint64_t)
        case TC_F32: TRTC_CONV(float)
        case TC_F64: TRTC_CONV(double)
    }
#undef TRTC_CONV
    return false;
}

ViewBuf zero_of(const std::string& type) {
    Layout l;
    if (!layout_of(type, l)) l.size = 8;
    return ViewBuf(l.size, 0);
}

bool lookback_param(size_t tiles, size_t vsize, ViewBuf& out, trtc::LookbackState* st_out = nullptr) {
    uint32_t e8 = 0;
    LookbackWs* w = lookback_ws(S(), tiles, vsize, &e8);
    if (!w) return false;
    trtc::LookbackState st;
    st.flags = w->flags;
    st.packed = w->packed;
    st.agg = w->agg;
    st.incl = w->incl;
    st.tile_ctr = w->tile_ctr;
    st.epoch8 = e8;
    st.err = device_error_word();
    st.result = w->result;
    out = pod_bytes(st);
    if (st_out) *st_out = st;
    return true;
}

unsigned grid_for(size_t n, unsigned block) {
    size_t g = (n + block - 1) / block;
    const size_t cap = (size_t)sm_count() * 16;
    if (g > cap) g = cap;
    return (unsigned)(g < 1 ? 1 : g);
}

// ------------------------------------------------------------------ JIT launch helpers
bool jit_run(const std::vector<std::string>& headers, const std::string& kernel_expr, unsigned grid, unsigned block,
             const std::vector<ViewBuf>& params, unsigned smem = 0) {
    JitFunction f;
    if (!jit_get_kernel(headers, "", kernel_expr, "", f)) return false;
    ktimer_mark("", S());
    const bool ok = jit_launch(f, dim_type{grid, 1, 1}, dim_type{block, 1, 1}, smem, S(), params);
    ktimer_mark(("jit:" + kernel_expr.substr(0, kernel_expr.find('<'))).c_str(), S());
    return ok;
}

// generic copy out[out_off + i] = in[in_off + i]
bool jit_copy(const ViewArg& in, const ViewArg& out, size_t n, size_t in_off = 0, size_t out_off = 0,
              const unsigned long long* tail = nullptr) {
    if (n == 0) return true;
    const std::string k = "trtc::copy_view_kernel<" + in.type + ", " + out.type + ">";
    return jit_run({"trtc_merge.cuh"}, k, grid_for(n, 256), 256,
                   {in.bytes, out.bytes, pod_bytes<size_t>(n), pod_bytes<size_t>(in_off), pod_bytes<size_t>(out_off),
                    pod_bytes<const unsigned long long*>(tail)});
}

// Scan-family kernel through NVRTC.  mode: 0 inclusive, 1 exclusive (init), 2 reduce,
// 3 reduce with init; reductions leave their result in *result_dev.
bool jit_scan(const DVVectorLike& in, const Functor* uop, const DVVectorLike* out, const std::string& T,
              const Functor& op, int mode, const ViewBuf& init, void** result_dev, const char* extra_header = nullptr) {
    const size_t n = in.size();
    const ViewArg iv = view_arg(in);
    const int vec = iv.contiguous ? vec_width(in.elem_size()) : 1;
    const int nv = iv.contiguous ? (vec >= 16 ? 1 : 16 / vec) : 16;
    const size_t tile = (size_t)256 * nv * vec;
    const size_t tiles = (n + tile - 1) / tile;
    Layout tl;
    if (!layout_of(T, tl)) { set_error("scan: unknown value type " + T); return false; }
    ViewBuf st;
    trtc::LookbackState lst;
    if (!lookback_param(tiles, tl.size, st, &lst)) return false;
    void* res = nullptr;
    if (mode >= 2) {
        if (tl.size > 16) {
            res = tmp_alloc(tl.size, S());
            lst.result = res;
            st = pod_bytes(lst);
        } else {
            res = lst.result;
        }
    }
    ViewArg ov;
    if (out) ov = view_arg(*out);
    else { ov.type = k_nothing; ov.bytes = nothing_bytes(); }
    const std::string k = "trtc::scan_kernel<" + iv.type + ", " + (uop ? uop->name_view_cls() : k_nothing) + ", " +
                          (uop ? "true" : "false") + ", " + ov.type + ", " + T + ", " + op.name_view_cls() + ", " +
                          num(mode) + ", 256, " + num(nv) + ">";
    std::vector<std::string> headers{"trtc_scan.cuh"};
    if (extra_header) headers.push_back(extra_header);
    const bool ok = jit_run(headers, k, (unsigned)tiles, 256,
                            {iv.bytes, uop ? uop->view() : nothing_bytes(), ov.bytes, pod_bytes<size_t>(n), op.view(),
                             init.size() == tl.size ? init : zero_of(T), st});
    if (result_dev) *result_dev = res;
    return ok;
}

// copies the reduction result of type T from the device into a host ViewBuf (blocking)
bool fetch_result(void* dev, size_t bytes, ViewBuf& ret, bool free_it) {
    ret.resize(bytes);
    bool ok = TRTC_CUDA(cudaMemcpyAsync(ret.data(), dev, bytes, cudaMemcpyDeviceToHost, S())) &&
              check_device_errors(S(), "reduce");
    if (free_it) tmp_free(dev, S());
    return ok;
}

}  // namespace

// ====================================================================== scans
static bool scan_dispatch(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& op, bool exclusive,
                          const DeviceViewable* init) {
    const size_t n = vec_in.size();
    if (n == 0) { set_error("scan: empty input"); return false; }  // general_scan launches no block
    if (!ensure_device()) return false;
    const std::string T = vec_out.name_elem_cls();
    ViewBuf ini;
    if (exclusive) {
        if (init) {
            // (decltype(vec_in)::value_t)init, then the out type (scan.cpp:28)
            ViewBuf as_in;
            if (convert_scalar(*init, vec_in.name_elem_cls(), as_in)) {
                SomeDeviceViewable in_typed(vec_in.name_elem_cls().c_str(), as_in.data(), as_in.size());
                if (!convert_scalar(in_typed, T, ini)) ini = as_in;
            } else {
                ini = init->view();
            }
        } else {
            ini = zero_of(T);
        }
    }
    const int oc = builtin_op_code(op);
    const int tc = type_code_of(T);
    void* ip = vec_in.contiguous_data();
    void* op_ = vec_out.contiguous_data();
    if (oc >= 0 && tc >= 0 && ip && op_ && vec_in.name_elem_cls() == T && vec_out.size() >= n) {
        if (!scan_raw(tc, oc, exclusive ? 1 : 0, ip, op_, n, exclusive ? ini.data() : nullptr, S())) return false;
        return true;
    }
    return jit_scan(vec_in, nullptr, &vec_out, T, op, exclusive ? 1 : 0, ini, nullptr);
}

bool TRTC_Inclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& binary_op) {
    return scan_dispatch(vec_in, vec_out, binary_op, false, nullptr);
}
bool TRTC_Inclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out) {
    Functor plus("Plus");
    return TRTC_Inclusive_Scan(vec_in, vec_out, plus);
}
bool TRTC_Exclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out) {
    Functor plus("Plus");
    return scan_dispatch(vec_in, vec_out, plus, true, nullptr);
}
bool TRTC_Exclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out, const DeviceViewable& init,
                         const Functor& binary_op) {
    return scan_dispatch(vec_in, vec_out, binary_op, true, &init);
}
bool TRTC_Exclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out, const DeviceViewable& init) {
    Functor plus("Plus");
    return TRTC_Exclusive_Scan(vec_in, vec_out, init, plus);
}

// transform scans: element i is (out_t)unary_op(vec_in[i]) (transform_scan.cpp:4-16)
bool TRTC_Transform_Inclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& unary_op,
                                   const Functor& binary_op) {
    if (vec_in.size() == 0) { set_error("transform scan: empty input"); return false; }
    if (!ensure_device()) return false;
    return jit_scan(vec_in, &unary_op, &vec_out, vec_out.name_elem_cls(), binary_op, 0, ViewBuf(), nullptr);
}
bool TRTC_Transform_Exclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& unary_op,
                                   const DeviceViewable& init, const Functor& binary_op) {
    if (vec_in.size() == 0) { set_error("transform scan: empty input"); return false; }
    if (!ensure_device()) return false;
    ViewBuf ini;
    if (!convert_scalar(init, vec_out.name_elem_cls(), ini)) ini = init.view();
    return jit_scan(vec_in, &unary_op, &vec_out, vec_out.name_elem_cls(), binary_op, 1, ini, nullptr);
}

// ====================================================================== scan_by_key
static bool scan_by_key_dispatch(const DVVectorLike& keys, const DVVectorLike& vals, DVVectorLike& out,
                                 const Functor& pred, const Functor& op, bool exclusive, const DeviceViewable* init) {
    const size_t n = keys.size();
    if (n == 0) { set_error("scan_by_key: empty input"); return false; }
    if (vals.size() < n) { set_error("scan_by_key: fewer values than keys"); return false; }
    if (!ensure_device()) return false;
    const std::string T = out.name_elem_cls();
    ViewBuf ini;
    if (exclusive) {
        if (!init) ini = zero_of(T);
        else if (!convert_scalar(*init, T, ini)) ini = init->view();
    }
    const int ktc = type_code_of(keys.name_elem_cls()), vtc = type_code_of(T);
    void* kp = keys.contiguous_data();
    void* vp = vals.contiguous_data();
    void* op_ = out.contiguous_data();
    const bool fast_types = (ktc == TC_I32 || ktc == TC_U32 || ktc == TC_I64) &&
                            (vtc == TC_I32 || vtc == TC_U32 || vtc == TC_I64 || vtc == TC_F32 || vtc == TC_F64);
    if (is_builtin(pred, "EqualTo") && is_builtin(op, "Plus") && fast_types && kp && vp && op_ &&
        vals.name_elem_cls() == T && out.size() >= n)
        return scan_by_key_raw(ktc, vtc, exclusive ? 1 : 0, kp, vp, op_, n, exclusive ? ini.data() : nullptr, S());
    // NVRTC instantiation
    const ViewArg kv = view_arg(keys), vv = view_arg(vals), ov = view_arg(out);
    const bool contig = kv.contiguous && vv.contiguous && vec_width(keys.elem_size()) > 1 && vec_width(vals.elem_size()) > 1;
    int vec = 1, nv = 16;
    if (contig) {
        vec = std::max(vec_width(keys.elem_size()), vec_width(vals.elem_size()));
        nv = vec >= 8 ? 2 : 4;
    }
    const size_t tile = (size_t)256 * nv * vec;
    const size_t tiles = (n + tile - 1) / tile;
    Layout tl;
    if (!layout_of(T, tl)) return false;
    ViewBuf st;
    if (!lookback_param(tiles, tl.size, st)) return false;
    const std::string k = "trtc::scan_by_key_kernel<" + kv.type + ", " + vv.type + ", " + ov.type + ", " + T + ", " +
                          pred.name_view_cls() + ", " + op.name_view_cls() + ", " + num(exclusive ? 1 : 0) +
                          ", 256, " + num(nv) + ">";
    return jit_run({"trtc_scan.cuh"}, k, (unsigned)tiles, 256,
                   {kv.bytes, vv.bytes, ov.bytes, pod_bytes<size_t>(n), pred.view(), op.view(),
                    exclusive ? ini : zero_of(T), st});
}

bool TRTC_Inclusive_Scan_By_Key(const DVVectorLike& k, const DVVectorLike& v, DVVectorLike& o, const Functor& pred,
                                const Functor& op) {
    return scan_by_key_dispatch(k, v, o, pred, op, false, nullptr);
}
bool TRTC_Inclusive_Scan_By_Key(const DVVectorLike& k, const DVVectorLike& v, DVVectorLike& o, const Functor& pred) {
    Functor plus("Plus");
    return scan_by_key_dispatch(k, v, o, pred, plus, false, nullptr);
}
bool TRTC_Inclusive_Scan_By_Key(const DVVectorLike& k, const DVVectorLike& v, DVVectorLike& o) {
    Functor eq("EqualTo"), plus("Plus");
    return scan_by_key_dispatch(k, v, o, eq, plus, false, nullptr);
}
bool TRTC_Exclusive_Scan_By_Key(const DVVectorLike& k, const DVVectorLike& v, DVVectorLike& o) {
    Functor eq("EqualTo"), plus("Plus");
    return scan_by_key_dispatch(k, v, o, eq, plus, true, nullptr);
}
bool TRTC_Exclusive_Scan_By_Key(const DVVectorLike& k, const DVVectorLike& v, DVVectorLike& o,
                                const DeviceViewable& init) {
    Functor eq("EqualTo"), plus("Plus");
    return scan_by_key_dispatch(k, v, o, eq, plus, true, &init);
}
bool TRTC_Exclusive_Scan_By_Key(const DVVectorLike& k, const DVVectorLike& v, DVVectorLike& o,
                                const DeviceViewable& init, const Functor& pred) {
    Functor plus("Plus");
    return scan_by_key_dispatch(k, v, o, pred, plus, true, &init);
}
bool TRTC_Exclusive_Scan_By_Key(const DVVectorLike& k, const DVVectorLike& v, DVVectorLike& o,
                                const DeviceViewable& init, const Functor& pred, const Functor& op) {
    return scan_by_key_dispatch(k, v, o, pred, op, true, &init);
}

// ====================================================================== reduce
// TRTC_Reduce: fold of the vector (with init: init is element 0 of n+1, reduce.cpp:16-24).
static bool reduce_dispatch(const DVVectorLike& vec, const DeviceViewable* init, const Functor& op, ViewBuf& ret) {
    const size_t n = vec.size();
    if (n == 0 && !init) { set_error("reduce: empty input without an initial value"); return false; }
    if (!ensure_device()) return false;
    const std::string T = vec.name_elem_cls();
    ViewBuf ini;
    if (init && !convert_scalar(*init, T, ini)) ini = init->view();
    if (n == 0) { ret = ini; return true; }
    const int oc = builtin_op_code(op), tc = type_code_of(T);
    void* p = vec.contiguous_data();
    if (oc >= 0 && tc >= 0 && p) {
        ret.resize(type_size(tc));
        return reduce_raw(tc, oc, p, n, init ? ini.data() : nullptr, ret.data(), S());
    }
    void* res = nullptr;
    Layout tl;
    if (!layout_of(T, tl)) return false;
    if (!jit_scan(vec, nullptr, nullptr, T, op, init ? 3 : 2, ini, &res)) return false;
    return fetch_result(res, tl.size, ret, tl.size > 16);
}

bool TRTC_Reduce(const DVVectorLike& vec, ViewBuf& ret) {
    Functor plus("Plus");
    return reduce_dispatch(vec, nullptr, plus, ret);
}
bool TRTC_Reduce(const DVVectorLike& vec, const DeviceViewable& init, const Functor& binary_op, ViewBuf& ret) {
    return reduce_dispatch(vec, &init, binary_op, ret);
}
bool TRTC_Reduce(const DVVectorLike& vec, const DeviceViewable& init, ViewBuf& ret) {
    Functor plus("Plus");
    return reduce_dispatch(vec, &init, plus, ret);
}

// init, unary_op(v0), ..., folded in the init's type (transform_reduce.cpp:5-14)
bool TRTC_Transform_Reduce(const DVVectorLike& vec, const Functor& unary_op, const DeviceViewable& init,
                           const Functor& binary_op, ViewBuf& ret) {
    if (!ensure_device()) return false;
    const std::string T = init.name_view_cls();
    if (vec.size() == 0) { ret = init.view(); return true; }
    void* res = nullptr;
    Layout tl;
    if (!layout_of(T, tl)) return false;
    if (!jit_scan(vec, &unary_op, nullptr, T, binary_op, 3, init.view(), &res)) return false;
    return fetch_result(res, tl.size, ret, tl.size > 16);
}

bool TRTC_Min_Element(const DVVectorLike& vec, size_t& id_min) {
    if (vec.size() < 1) return true;  // extrema.cpp:8: nothing to do, id_min untouched
    if (!ensure_device()) return false;
    const int tc = type_code_of(vec.name_elem_cls());
    void* p = vec.contiguous_data();
    std::unique_ptr<DVVector> tmp;
    if (tc < 0) { set_error("min_element: unsupported element type"); return false; }
    if (!p) {
        tmp.reset(new DVVector(vec.name_elem_cls().c_str(), vec.size()));
        if (!jit_copy(view_arg(vec), view_arg(*tmp), vec.size())) return false;
        p = tmp->data();
    }
    unsigned long long idx = 0;
    if (!min_element_raw(tc, p, vec.size(), S(), &idx)) return false;
    id_min = (size_t)idx;
    return true;
}

// ====================================================================== copy
bool TRTC_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_out) {
    const size_t n = vec_in.size();
    if (n == 0) return true;
    if (!ensure_device()) return false;
    void* ip = vec_in.contiguous_data();
    void* op = vec_out.contiguous_data();
    if (ip && op && vec_in.name_elem_cls() == vec_out.name_elem_cls())
        return TRTC_CUDA(cudaMemcpyAsync(op, ip, n * vec_in.elem_size(), cudaMemcpyDeviceToDevice, S()));
    return jit_copy(view_arg(vec_in), view_arg(vec_out), n);
}

// ====================================================================== compaction family
#ifndef TRTC_COMPACT2_GENERIC_ITEMS
#define TRTC_COMPACT2_GENERIC_ITEMS 16  // 2^28 int32 unique outside the vector path: 16 items 0.69 ms, 32 0.77-0.99
#endif
namespace {
enum { CM_PRED = 0, CM_PRED_STENCIL = 1, CM_NOT_EQUAL = 2, CM_NOT_PRED = 3, CM_NOT_PRED_STENCIL = 4, CM_UNIQUE = 5,
       CM_UNIQUE_PRED = 6, CM_TAIL = 7 };

struct CompactSpec {
    int mode = CM_PRED;
    const DVVectorLike* in = nullptr;
    const DVVectorLike* stencil = nullptr;
    const Functor* pred = nullptr;
    const DeviceViewable* value = nullptr;
    ViewArg out, out_false, in2, out2;
    bool partition = false, two = false;
    std::vector<const DVVectorLike*> written, read;  // for the overlap test
    void set_out(const DVVectorLike& v) { out = view_arg(v); written.push_back(&v); }
    void set_false(const DVVectorLike& v) { out_false = view_arg(v); written.push_back(&v); }
    void set_out2(const DVVectorLike& v) { out2 = view_arg(v); written.push_back(&v); }
    void set_in2(const DVVectorLike& v) { in2 = view_arg(v); read.push_back(&v); }
    // true when no written vector can share memory with a read one (both contiguous and
    // their byte ranges disjoint)
    bool disjoint() const {
        std::vector<const DVVectorLike*> r(read);
        r.push_back(in);
        if (stencil) r.push_back(stencil);
        for (const DVVectorLike* w : written) {
            const char* wp = (const char*)w->contiguous_data();
            if (!wp) return false;
            const size_t wb = w->size() * w->elem_size();
            for (const DVVectorLike* x : r) {
                const char* xp = (const char*)x->contiguous_data();
                if (!xp) return false;
                const size_t xb = x->size() * x->elem_size();
                if (!(wp + wb <= xp || xp + xb <= wp)) return false;
            }
        }
        return true;
    }
};

const unsigned long long kFail = ~0ull;

// one single-pass compaction launch; returns the number of selected elements
unsigned long long run_compact(CompactSpec& c) {
    const size_t n = c.in->size();
    if (n == 0) { set_error("compaction: empty input"); return kFail; }
    if (!ensure_device()) return kFail;
    const ViewArg iv = view_arg(*c.in);
    ViewArg sv;
    if (c.stencil) sv = view_arg(*c.stencil);
    else { sv.type = k_nothing; sv.bytes = nothing_bytes(); }
    auto nothing_arg = [](ViewArg& a) {
        if (a.type.empty()) { a.type = k_nothing; a.bytes = nothing_bytes(); }
    };
    nothing_arg(c.out_false);
    nothing_arg(c.in2);
    nothing_arg(c.out2);
    std::string vtype = k_nothing;
    ViewBuf vbytes = nothing_bytes();
    if (c.value) {
        vtype = c.in->name_elem_cls();
        if (!convert_scalar(*c.value, vtype, vbytes)) { vtype = c.value->name_view_cls(); vbytes = c.value->view(); }
    }
    const std::string ptype = c.pred ? c.pred->name_view_cls() : "EqualTo";
    const ViewBuf pbytes = c.pred ? c.pred->view() : nothing_bytes();
    const bool two_phase = c.disjoint();
    if (!two_phase && !c.partition && !c.two && c.written.size() == 1 && c.written[0]->contiguous_data() &&
        c.in->contiguous_data() && (!c.stencil || c.stencil->contiguous_data())) {
        // in place (one contiguous output overlapping the input): the two-phase kernel into a
        // pool temporary, then the kept elements copied back; the one-pass kernel remains for
        // views and multi-output forms, or when no temporary can be had
        const DVVectorLike* o = c.written[0];
        void* tmp = tmp_alloc(n * o->elem_size(), S());
        if (tmp) {
            CompactSpec t = c;
            t.out = raw_view(tmp, n, o->name_elem_cls());
            t.written.clear();
            const unsigned long long cnt = run_compact(t);
            bool ok = cnt != kFail;
            const size_t keep = cnt == kFail ? 0 : (size_t)std::min<unsigned long long>(cnt, o->size());
            if (ok && keep > 0)
                ok = TRTC_CUDA(cudaMemcpyAsync(o->contiguous_data(), tmp, keep * o->elem_size(), cudaMemcpyDeviceToDevice,
                                               S()));
            tmp_free(tmp, S());
            return ok ? cnt : kFail;
        }
        (void)cudaGetLastError();  // the failed allocation must not fail a later launch check
    }
    // the 16-byte vector path (contiguous 4-byte input and output: element-wise tests of one
    // array, or neighbour tests with an optional second array) takes 32 items per thread; the
    // other two-phase forms (views, other widths, stencils, partitions) hold their rows in
    // registers and take TRTC_COMPACT2_GENERIC_ITEMS
    const bool neigh = c.mode == CM_UNIQUE || c.mode == CM_UNIQUE_PRED || c.mode == CM_TAIL;
    const bool vec_mode = !c.partition && c.in->elem_size() == 4 && c.in->contiguous_data() && !c.written.empty() &&
                          c.written[0]->contiguous_data() &&
                          ((!c.two && (c.mode == CM_PRED || c.mode == CM_NOT_EQUAL || c.mode == CM_NOT_PRED)) || neigh);
    // (two-array vector forms hold their second array's rows in registers too: 16 items)
    const int items2 = vec_mode ? (c.two ? 16 : 32) : TRTC_COMPACT2_GENERIC_ITEMS;
    const size_t tile = 256 * (two_phase ? (size_t)items2 : 16);
    const size_t tiles = (n + tile - 1) / tile;
    ViewBuf st;
    trtc::LookbackState lst;
    const bool c32 = n < (1ull << 32);  // 32-bit counts: flag and count in one look-back word
    if (!lookback_param(tiles, c32 ? 4 : 8, st, &lst)) return kFail;
    const std::string k = std::string(two_phase ? "trtc::compact2_kernel<" : "trtc::compact_kernel<") + num(c.mode) +
                          ", " + (c.partition ? "true" : "false") + ", " + (c.two ? "true" : "false") + ", " +
                          iv.type + ", " + sv.type + ", " + ptype + ", " + vtype + ", " + c.out.type + ", " +
                          c.out_false.type + ", " + c.in2.type + ", " + c.out2.type + ", 256, " +
                          (two_phase ? std::to_string(items2) + ", " : std::string("16, ")) +
                          (c32 ? "unsigned int" : "unsigned long long") + ">";
    std::vector<ViewBuf> params{iv.bytes, sv.bytes, pbytes, vbytes, c.out.bytes, c.out_false.bytes, c.in2.bytes,
                                c.out2.bytes, pod_bytes<size_t>(n)};
    unsigned grid = (unsigned)tiles;
    if (two_phase) {
        // persistent CTAs: 4 per SM (the kernel's register budget allows it for 4-byte elements)
        const size_t g = (size_t)sm_count() * 4;
        grid = (unsigned)(g < tiles ? g : tiles);
        params.push_back(pod_bytes<size_t>(tiles));
        lst.pf_ahead = tile_prefetch_ahead(grid / 2);  // half a grid ahead, as the built-in launches
        st = pod_bytes(lst);
    }
    params.push_back(st);
    if (!jit_run({"trtc_compact.cuh"}, k, grid, 256, params)) return kFail;
    unsigned long long cnt = 0;
    if (!TRTC_CUDA(cudaMemcpyAsync(&cnt, lst.result, 8, cudaMemcpyDeviceToHost, S())) ||
        !check_device_errors(S(), "compaction"))
        return kFail;
    return cnt;
}

uint32_t to_u32(unsigned long long c) { return c == kFail ? (uint32_t)(-1) : (uint32_t)c; }

// built-in fast path for Remove/Unique on contiguous vectors of arithmetic types
bool fast_compact(int mode, const DVVectorLike& in, DVVectorLike& out, const DeviceViewable* value,
                  unsigned long long& cnt) {
    const int tc = type_code_of(in.name_elem_cls());
    void* ip = in.contiguous_data();
    void* op = out.contiguous_data();
    if (tc < 0 || !ip || !op || in.name_elem_cls() != out.name_elem_cls() || out.size() < in.size()) return false;
    ViewBuf vb;
    if (value && !convert_scalar(*value, in.name_elem_cls(), vb)) return false;
    if (in.size() == 0) return false;
    if (!compact_raw(tc, mode, ip, op, in.size(), value ? vb.data() : nullptr, S(), &cnt)) cnt = kFail;
    return true;
}
}  // namespace

uint32_t TRTC_Copy_If(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& pred) {
    CompactSpec c;
    c.mode = CM_PRED; c.in = &vec_in; c.pred = &pred; c.set_out(vec_out);
    return to_u32(run_compact(c));
}
uint32_t TRTC_Copy_If_Stencil(const DVVectorLike& vec_in, const DVVectorLike& vec_stencil, DVVectorLike& vec_out,
                              const Functor& pred) {
    CompactSpec c;
    c.mode = CM_PRED_STENCIL; c.in = &vec_in; c.stencil = &vec_stencil; c.pred = &pred; c.set_out(vec_out);
    return to_u32(run_compact(c));
}
uint32_t TRTC_Remove_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_out, const DeviceViewable& value) {
    unsigned long long cnt = 0;
    if (fast_compact(CM_NOT_EQUAL, vec_in, vec_out, &value, cnt)) return to_u32(cnt);
    CompactSpec c;
    c.mode = CM_NOT_EQUAL; c.in = &vec_in; c.value = &value; c.set_out(vec_out);
    return to_u32(run_compact(c));
}
// in place: a tile reads its input before anything is published, and selected elements only
// move to lower positions, so no copy of the input is needed (the reference copies first)
uint32_t TRTC_Remove(DVVectorLike& vec, const DeviceViewable& value) { return TRTC_Remove_Copy(vec, vec, value); }
uint32_t TRTC_Remove_Copy_If(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& pred) {
    CompactSpec c;
    c.mode = CM_NOT_PRED; c.in = &vec_in; c.pred = &pred; c.set_out(vec_out);
    return to_u32(run_compact(c));
}
uint32_t TRTC_Remove_If(DVVectorLike& vec, const Functor& pred) { return TRTC_Remove_Copy_If(vec, vec, pred); }
uint32_t TRTC_Remove_Copy_If_Stencil(const DVVectorLike& vec_in, const DVVectorLike& stencil, DVVectorLike& vec_out,
                                     const Functor& pred) {
    CompactSpec c;
    c.mode = CM_NOT_PRED_STENCIL; c.in = &vec_in; c.stencil = &stencil; c.pred = &pred; c.set_out(vec_out);
    return to_u32(run_compact(c));
}
uint32_t TRTC_Remove_If_Stencil(DVVectorLike& vec, const DVVectorLike& stencil, const Functor& pred) {
    return TRTC_Remove_Copy_If_Stencil(vec, stencil, vec, pred);
}
uint32_t TRTC_Unique_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_out) {
    unsigned long long cnt = 0;
    if (fast_compact(CM_UNIQUE, vec_in, vec_out, nullptr, cnt)) return to_u32(cnt);
    CompactSpec c;
    c.mode = CM_UNIQUE; c.in = &vec_in; c.set_out(vec_out);
    return to_u32(run_compact(c));
}
uint32_t TRTC_Unique_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& binary_pred) {
    if (is_builtin(binary_pred, "EqualTo")) return TRTC_Unique_Copy(vec_in, vec_out);
    CompactSpec c;
    c.mode = CM_UNIQUE_PRED; c.in = &vec_in; c.pred = &binary_pred; c.set_out(vec_out);
    return to_u32(run_compact(c));
}
uint32_t TRTC_Unique(DVVectorLike& vec) { return TRTC_Unique_Copy(vec, vec); }
uint32_t TRTC_Unique(DVVectorLike& vec, const Functor& binary_pred) { return TRTC_Unique_Copy(vec, vec, binary_pred); }
uint32_t TRTC_Unique_By_Key_Copy(const DVVectorLike& keys_in, const DVVectorLike& values_in, DVVectorLike& keys_out,
                                 DVVectorLike& values_out, const Functor& binary_pred) {
    CompactSpec c;
    c.mode = is_builtin(binary_pred, "EqualTo") ? CM_UNIQUE : CM_UNIQUE_PRED;
    c.in = &keys_in; c.pred = &binary_pred; c.set_out(keys_out);
    c.two = true; c.set_in2(values_in); c.set_out2(values_out);
    return to_u32(run_compact(c));
}
uint32_t TRTC_Unique_By_Key_Copy(const DVVectorLike& keys_in, const DVVectorLike& values_in, DVVectorLike& keys_out,
                                 DVVectorLike& values_out) {
    Functor eq("EqualTo");
    return TRTC_Unique_By_Key_Copy(keys_in, values_in, keys_out, values_out, eq);
}
uint32_t TRTC_Unique_By_Key(DVVectorLike& keys, DVVectorLike& values) {
    return TRTC_Unique_By_Key_Copy(keys, values, keys, values);
}
uint32_t TRTC_Unique_By_Key(DVVectorLike& keys, DVVectorLike& values, const Functor& binary_pred) {
    return TRTC_Unique_By_Key_Copy(keys, values, keys, values, binary_pred);
}

uint32_t TRTC_Partition_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_true, DVVectorLike& vec_false,
                             const Functor& pred) {
    CompactSpec c;
    c.mode = CM_PRED; c.in = &vec_in; c.pred = &pred; c.partition = true;
    c.set_out(vec_true); c.set_false(vec_false);
    return to_u32(run_compact(c));
}
uint32_t TRTC_Partition_Copy_Stencil(const DVVectorLike& vec_in, const DVVectorLike& stencil, DVVectorLike& vec_true,
                                     DVVectorLike& vec_false, const Functor& pred) {
    CompactSpec c;
    c.mode = CM_PRED_STENCIL; c.in = &vec_in; c.stencil = &stencil; c.pred = &pred; c.partition = true;
    c.set_out(vec_true); c.set_false(vec_false);
    return to_u32(run_compact(c));
}
// in place: selected elements are compacted in place, rejected ones into a temporary that is
// then appended behind them (partition.cpp:29-53 copies the whole input first instead)
static uint32_t partition_in_place(DVVectorLike& vec, const DVVectorLike* stencil, const Functor& pred) {
    const size_t n = vec.size();
    if (n == 0) { set_error("partition: empty input"); return (uint32_t)(-1); }
    if (!ensure_device()) return (uint32_t)(-1);
    void* tmp = tmp_alloc(n * vec.elem_size(), S());
    if (!tmp) return (uint32_t)(-1);
    const ViewArg tv = raw_view(tmp, n, vec.name_elem_cls());
    CompactSpec c;
    c.mode = stencil ? CM_PRED_STENCIL : CM_PRED; c.in = &vec; c.stencil = stencil; c.pred = &pred;
    c.partition = true; c.set_out(vec); c.out_false = tv;
    const unsigned long long cnt = run_compact(c);
    bool ok = cnt != kFail;
    if (ok && cnt < n) {
        // the count is already on the host: copy the n - cnt rejected elements behind it
        ok = jit_copy(tv, view_arg(vec), n - cnt, 0, cnt) && check_device_errors(S(), "partition");
    }
    tmp_free(tmp, S());
    return ok ? (uint32_t)cnt : (uint32_t)(-1);
}
uint32_t TRTC_Partition(DVVectorLike& vec, const Functor& pred) { return partition_in_place(vec, nullptr, pred); }
uint32_t TRTC_Partition_Stencil(DVVectorLike& vec, const DVVectorLike& stencil, const Functor& pred) {
    return partition_in_place(vec, &stencil, pred);
}

// reduce_by_key: segmented inclusive scan, then compaction of segment tails
// (reduce.cpp:36-62); the tails are selected from the keys with the same predicate.
static uint32_t reduce_by_key_impl(const DVVectorLike& key_in, const DVVectorLike& value_in, DVVectorLike& key_out,
                                   DVVectorLike& value_out, const Functor& pred, const Functor& op) {
    const size_t n = key_in.size();
    if (n == 0) { set_error("reduce_by_key: empty input"); return (uint32_t)(-1); }
    DVVector scanned(value_out.name_elem_cls().c_str(), n);
    if (!scan_by_key_dispatch(key_in, value_in, scanned, pred, op, false, nullptr)) return (uint32_t)(-1);
    CompactSpec c;
    c.mode = CM_TAIL; c.in = &key_in; c.pred = &pred; c.set_out(key_out);
    c.two = true; c.set_in2(scanned); c.set_out2(value_out);
    return to_u32(run_compact(c));
}
uint32_t TRTC_Reduce_By_Key(const DVVectorLike& key_in, const DVVectorLike& value_in, DVVectorLike& key_out,
                            DVVectorLike& value_out) {
    Functor eq("EqualTo"), plus("Plus");
    return reduce_by_key_impl(key_in, value_in, key_out, value_out, eq, plus);
}
uint32_t TRTC_Reduce_By_Key(const DVVectorLike& key_in, const DVVectorLike& value_in, DVVectorLike& key_out,
                            DVVectorLike& value_out, const Functor& binary_pred) {
    Functor plus("Plus");
    return reduce_by_key_impl(key_in, value_in, key_out, value_out, binary_pred, plus);
}
uint32_t TRTC_Reduce_By_Key(const DVVectorLike& key_in, const DVVectorLike& value_in, DVVectorLike& key_out,
                            DVVectorLike& value_out, const Functor& binary_pred, const Functor& binary_op) {
    return reduce_by_key_impl(key_in, value_in, key_out, value_out, binary_pred, binary_op);
}

// ====================================================================== sort
// Radix sort for Less/Greater on the built-in key types (sort.cpp:7-65 routes the same
// set); everything else is a stable merge sort with the comparator in a template slot.
static bool radix_key_type(const std::string& e) {
    const int tc = type_code_of(e);
    return tc >= 0;
}

static bool merge_sort_impl(DVVectorLike& keys, DVVectorLike* values, const Functor& comp) {
    const size_t n = keys.size();
    if (n <= 1) return true;
    const std::string K = keys.name_elem_cls();
    const std::string V = values ? values->name_elem_cls() : std::string(k_nothing);
    const size_t ks = keys.elem_size(), vs = values ? values->elem_size() : 1;
    void* k0 = tmp_alloc(n * ks, S());
    void* k1 = tmp_alloc(n * ks, S());
    void* v0 = values ? tmp_alloc(n * vs, S()) : nullptr;
    void* v1 = values ? tmp_alloc(n * vs, S()) : nullptr;
    bool ok = k0 && k1 && (!values || (v0 && v1));
    const ViewArg kv = view_arg(keys);
    ViewArg vv;
    if (values) vv = view_arg(*values);
    else { vv.type = k_nothing; vv.bytes = nothing_bytes(); }
    const std::string hv = values ? "true" : "false";
    if (ok) {
        const unsigned blocks = (unsigned)((n + 511) / 512);
        ok = jit_run({"trtc_merge.cuh"}, "trtc::merge_block_sort_kernel<" + kv.type + ", " + vv.type + ", " +
                                             comp.name_view_cls() + ", " + hv + ", 256>",
                     blocks, 256, {kv.bytes, vv.bytes, comp.view(), pod_bytes<size_t>(n), pod_bytes<void*>(k0),
                                   pod_bytes<void*>(v0)});
    }
    int cur = 0;
    void* kb[2] = {k0, k1};
    void* vb[2] = {v0, v1};
    for (size_t w = 512; ok && w < n; w *= 2) {
        ok = jit_run({"trtc_merge.cuh"}, "trtc::merge_level_kernel<" + K + ", " + V + ", " + comp.name_view_cls() + ", " +
                                             hv + ">",
                     grid_for(n, 256), 256,
                     {pod_bytes<void*>(kb[cur]), pod_bytes<void*>(vb[cur]), pod_bytes<void*>(kb[cur ^ 1]),
                      pod_bytes<void*>(vb[cur ^ 1]), pod_bytes<size_t>(n), pod_bytes<size_t>(w), comp.view()});
        cur ^= 1;
    }
    if (ok) ok = jit_copy(raw_view(kb[cur], n, K), kv, n);
    if (ok && values) ok = jit_copy(raw_view(vb[cur], n, V), vv, n);
    tmp_free(k0, S()); tmp_free(k1, S()); tmp_free(v0, S()); tmp_free(v1, S());
    return ok;
}

static bool sort_impl(DVVectorLike& keys, DVVectorLike* values, const Functor& comp) {
    const size_t n = keys.size();
    // the reference fails on an empty vector (the Min_Element reduction refuses n < 1)
    if (n == 0) { set_error("sort: empty input"); return false; }
    if (!ensure_device()) return false;
    if (values && values->size() < n) { set_error("sort_by_key: fewer values than keys"); return false; }
    const bool less = is_builtin(comp, "Less"), greater = is_builtin(comp, "Greater");
    if (!(less || greater) || !radix_key_type(keys.name_elem_cls())) return merge_sort_impl(keys, values, comp);
    if (n == 1) return true;
    const int tc = type_code_of(keys.name_elem_cls());
    // radix kernels work on plain arrays; computed views are staged through temporaries
    std::unique_ptr<DVVector> tk, tv;
    void* kp = keys.contiguous_data();
    void* vp = values ? values->contiguous_data() : nullptr;
    if (!kp) {
        tk.reset(new DVVector(keys.name_elem_cls().c_str(), n));
        if (!jit_copy(view_arg(keys), view_arg(*tk), n)) return false;
        kp = tk->data();
    }
    if (values && !vp) {
        tv.reset(new DVVector(values->name_elem_cls().c_str(), n));
        if (!jit_copy(view_arg(*values), view_arg(*tv), n)) return false;
        vp = tv->data();
    }
    if (!sort_raw(tc, kp, values ? vp : nullptr, values ? values->elem_size() : 0, n, greater, S())) return false;
    if (tk && !jit_copy(view_arg(*tk), view_arg(keys), n)) return false;
    if (tv && !jit_copy(view_arg(*tv), view_arg(*values), n)) return false;
    return check_device_errors(S(), "sort");
}

bool TRTC_Sort(DVVectorLike& vec, const Functor& comp) { return sort_impl(vec, nullptr, comp); }
bool TRTC_Sort(DVVectorLike& vec) {
    Functor less("Less");
    return sort_impl(vec, nullptr, less);
}
bool TRTC_Sort_By_Key(DVVectorLike& keys, DVVectorLike& values, const Functor& comp) {
    return sort_impl(keys, &values, comp);
}
bool TRTC_Sort_By_Key(DVVectorLike& keys, DVVectorLike& values) {
    Functor less("Less");
    return sort_impl(keys, &values, less);
}

// ====================================================================== searches
// binary_search.h: single values return through the host (one blocking copy, like the
// reference's), vectorised searches write `result` (one thread per value).
static bool search_value(int kind, const DVVectorLike& vec, const DeviceViewable& value, const Functor& comp,
                         unsigned long long& out) {
    if (vec.size() == 0) { out = 0; return true; }  // binary_search.cpp:27-31
    if (!ensure_device()) return false;
    const ViewArg vv = view_arg(vec);
    ViewBuf vb;
    std::string vt = vec.name_elem_cls();
    if (!convert_scalar(value, vt, vb)) { vt = value.name_view_cls(); vb = value.view(); }
    unsigned long long* d = (unsigned long long*)tmp_alloc(8, S());
    if (!d) return false;
    const std::string k = "trtc::search_one_kernel<" + num(kind) + ", " + vv.type + ", " + vt + ", " +
                          comp.name_view_cls() + ">";
    bool ok = jit_run({"trtc_search.cuh"}, k, 1, 32, {vv.bytes, vb, comp.view(), pod_bytes<unsigned long long*>(d)}) &&
              TRTC_CUDA(cudaMemcpyAsync(&out, d, 8, cudaMemcpyDeviceToHost, S())) &&
              check_device_errors(S(), "search");
    tmp_free(d, S());
    return ok;
}

static bool search_vector(int kind, const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result,
                          const Functor& comp) {
    const size_t m = values.size();
    if (m == 0) return true;
    if (!ensure_device()) return false;
    const ViewArg vv = view_arg(vec), qv = view_arg(values), rv = view_arg(result);
    const std::string k = "trtc::search_v_kernel<" + num(kind) + ", " + vv.type + ", " + qv.type + ", " + rv.type +
                          ", " + comp.name_view_cls() + ">";
    return jit_run({"trtc_search.cuh"}, k, grid_for(m, 256), 256,
                   {vv.bytes, qv.bytes, rv.bytes, pod_bytes<size_t>(m), comp.view()});
}

bool TRTC_Lower_Bound(const DVVectorLike& vec, const DeviceViewable& value, const Functor& comp, size_t& result) {
    unsigned long long r = 0;
    if (!search_value(0, vec, value, comp, r)) return false;
    result = (size_t)r;
    return true;
}
bool TRTC_Lower_Bound(const DVVectorLike& vec, const DeviceViewable& value, size_t& result) {
    return TRTC_Lower_Bound(vec, value, Functor("Less"), result);
}
bool TRTC_Upper_Bound(const DVVectorLike& vec, const DeviceViewable& value, const Functor& comp, size_t& result) {
    unsigned long long r = 0;
    if (!search_value(1, vec, value, comp, r)) return false;
    result = (size_t)r;
    return true;
}
bool TRTC_Upper_Bound(const DVVectorLike& vec, const DeviceViewable& value, size_t& result) {
    return TRTC_Upper_Bound(vec, value, Functor("Less"), result);
}
bool TRTC_Binary_Search(const DVVectorLike& vec, const DeviceViewable& value, const Functor& comp, bool& result) {
    unsigned long long r = 0;
    if (vec.size() == 0) { result = false; return true; }
    if (!search_value(2, vec, value, comp, r)) return false;
    result = r != 0;
    return true;
}
bool TRTC_Binary_Search(const DVVectorLike& vec, const DeviceViewable& value, bool& result) {
    return TRTC_Binary_Search(vec, value, Functor("Less"), result);
}
bool TRTC_Lower_Bound_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result,
                        const Functor& comp) {
    return search_vector(0, vec, values, result, comp);
}
bool TRTC_Lower_Bound_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result) {
    return search_vector(0, vec, values, result, Functor("Less"));
}
bool TRTC_Upper_Bound_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result,
                        const Functor& comp) {
    return search_vector(1, vec, values, result, comp);
}
bool TRTC_Upper_Bound_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result) {
    return search_vector(1, vec, values, result, Functor("Less"));
}
bool TRTC_Binary_Search_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result,
                          const Functor& comp) {
    return search_vector(2, vec, values, result, comp);
}
bool TRTC_Binary_Search_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result) {
    return search_vector(2, vec, values, result, Functor("Less"));
}

// ====================================================================== remaining algorithms
// fill.h, sequence.h, tabulate.h, transform.h, replace.h, for_each.h, adjacent_difference.h,
// gather.h, scatter.h, swap.h, count.h, find.h, mismatch.h, equal.h, logical.h, extrema.h,
// inner_product.h, partition.h (point, is_partitioned), sort.h (is_sorted*), merge.h: one
// NVRTC-instantiated kernel of trtc_misc.cuh each, over any views and user functors.
namespace {

ViewArg nothing_arg() {
    ViewArg a;
    a.type = k_nothing;
    a.bytes = nothing_bytes();
    return a;
}
ViewArg functor_arg(const Functor& f) {
    ViewArg a;
    a.type = f.name_view_cls();
    a.bytes = f.view();
    return a;
}
// a DeviceViewable (scalar, tuple, ...) as a kernel argument of its own view type
ViewArg dv_arg(const DeviceViewable& d) {
    ViewArg a;
    a.type = d.name_view_cls();
    a.bytes = d.view();
    return a;
}

std::string targs(const std::vector<std::string>& parts) {
    std::string s = "<";
    for (size_t i = 0; i < parts.size(); i++) s += parts[i] + (i + 1 < parts.size() ? ", " : "");
    return s + ">";
}

// one grid-stride launch of trtc::<kernel> over n items; params in the kernel's order
bool misc_run(const std::string& kernel, const std::vector<ViewArg>& args, size_t n, std::vector<ViewBuf> tail) {
    if (n == 0) return true;
    if (!ensure_device()) return false;
    std::vector<std::string> types;
    std::vector<ViewBuf> params;
    for (const ViewArg& a : args) {
        types.push_back(a.type);
        params.push_back(a.bytes);
    }
    for (auto& t : tail) params.push_back(t);
    return jit_run({"trtc_misc.cuh"}, "trtc::" + kernel + targs(types), grid_for(n, 256), 256, params);
}
// same, with leading non-type template arguments
bool misc_run_t(const std::string& kernel, const std::vector<std::string>& lead, const std::vector<ViewArg>& args,
                size_t n, std::vector<ViewBuf> tail) {
    if (n == 0) return true;
    if (!ensure_device()) return false;
    std::vector<std::string> types = lead;
    std::vector<ViewBuf> params;
    for (const ViewArg& a : args) {
        types.push_back(a.type);
        params.push_back(a.bytes);
    }
    for (auto& t : tail) params.push_back(t);
    return jit_run({"trtc_misc.cuh"}, "trtc::" + kernel + targs(types), grid_for(n, 256), 256, params);
}

// the value as the vector's element type when it converts on the host, else as itself
ViewArg value_as_elem(const DeviceViewable& value, const DVVectorLike& vec) {
    ViewArg a;
    a.type = vec.name_elem_cls();
    if (!convert_scalar(value, a.type, a.bytes)) a = dv_arg(value);
    return a;
}

// first index in [begin, n) with the property of `mode` (FindMode of trtc_misc.cuh); n if none
bool find_first(int mode, const ViewArg& v, const ViewArg& w, const ViewArg& value, const ViewArg& pred, size_t begin,
                size_t n, size_t& result) {
    result = n;
    if (begin >= n) return true;
    if (!ensure_device()) return false;
    unsigned long long* d = (unsigned long long*)tmp_alloc(8, S());
    if (!d) return false;
    const unsigned long long init = n;
    bool ok = TRTC_CUDA(cudaMemcpyAsync(d, &init, 8, cudaMemcpyHostToDevice, S()));
    const std::string k = "trtc::find_first_kernel" + targs({num(mode), v.type, w.type, value.type, pred.type});
    ok = ok && jit_run({"trtc_misc.cuh"}, k, grid_for(n - begin, 256), 256,
                       {v.bytes, w.bytes, value.bytes, pred.bytes, pod_bytes<size_t>(begin), pod_bytes<size_t>(n),
                        pod_bytes<unsigned long long*>(d)});
    unsigned long long r = n;
    ok = ok && TRTC_CUDA(cudaMemcpyAsync(&r, d, 8, cudaMemcpyDeviceToHost, S())) && check_device_errors(S(), "find");
    tmp_free(d, S());
    result = (size_t)r;
    return ok;
}
// general_find's convention (internal/general_find.cpp): (size_t)-1 when nothing is found
bool find_or_none(int mode, const ViewArg& v, const ViewArg& w, const ViewArg& value, const ViewArg& pred, size_t n,
                  size_t& result) {
    size_t r = 0;
    if (!find_first(mode, v, w, value, pred, 0, n, r)) return false;
    result = r >= n ? (size_t)(-1) : r;
    return true;
}

bool count_run(int mode, const DVVectorLike& vec, const ViewArg& value, const ViewArg& pred, size_t& result) {
    result = 0;
    const size_t n = vec.size();
    if (n == 0) return true;
    if (!ensure_device()) return false;
    unsigned long long* d = (unsigned long long*)tmp_alloc(8, S());
    if (!d) return false;
    bool ok = TRTC_CUDA(cudaMemsetAsync(d, 0, 8, S()));
    const ViewArg v = view_arg(vec);
    ok = ok && jit_run({"trtc_misc.cuh"}, "trtc::count_kernel" + targs({num(mode), v.type, value.type, pred.type}),
                       grid_for(n, 256), 256,
                       {v.bytes, value.bytes, pred.bytes, pod_bytes<size_t>(n), pod_bytes<unsigned long long*>(d)});
    unsigned long long r = 0;
    ok = ok && TRTC_CUDA(cudaMemcpyAsync(&r, d, 8, cudaMemcpyDeviceToHost, S())) && check_device_errors(S(), "count");
    tmp_free(d, S());
    result = (size_t)r;
    return ok;
}

// the reference's element-index reduction (MAX, or min, under comp); empty leaves result as is
bool index_tree(bool max, const DVVectorLike& vec, const Functor& comp, size_t& result) {
    const size_t n = vec.size();
    if (n == 0) return true;  // extrema.cpp:8
    if (!ensure_device()) return false;
    const ViewArg v = view_arg(vec);
    const size_t nb1 = (n + 255) / 256;
    unsigned long long* t[2] = {(unsigned long long*)tmp_alloc(nb1 * 8, S()),
                                (unsigned long long*)tmp_alloc(nb1 * 8, S())};
    bool ok = t[0] && t[1];
    size_t m = n;
    int cur = 0;  // buffer holding the latest round's results
    for (bool first = true; ok && (first || m > 1); first = false) {
        const size_t nb = (m + 255) / 256;
        const size_t cap = (size_t)sm_count() * 8;
        const unsigned grid = (unsigned)(nb < cap ? nb : cap);
        const int dst = first ? 0 : cur ^ 1;
        const std::string k = "trtc::index_tree_kernel" +
                              targs({max ? "true" : "false", first ? "true" : "false", v.type, comp.name_view_cls()});
        ok = jit_run({"trtc_misc.cuh"}, k, grid, 256,
                     {v.bytes, comp.view(), pod_bytes<const unsigned long long*>(first ? nullptr : t[cur]),
                      pod_bytes<size_t>(m), pod_bytes<unsigned long long*>(t[dst])});
        cur = dst;
        m = nb;
    }
    unsigned long long r = 0;
    ok = ok && TRTC_CUDA(cudaMemcpyAsync(&r, t[cur], 8, cudaMemcpyDeviceToHost, S())) &&
         check_device_errors(S(), "extrema");
    if (t[0]) tmp_free(t[0], S());
    if (t[1]) tmp_free(t[1], S());
    if (ok) result = (size_t)r;
    return ok;
}

// does [p, p + n*es) overlap [q, q + m*es2)?
bool overlaps(const void* p, size_t bytes_p, const void* q, size_t bytes_q) {
    const char* a = (const char*)p;
    const char* b = (const char*)q;
    return a < b + bytes_q && b < a + bytes_p;
}

}  // namespace

// ---------------------------------------------------------------- transformations
bool TRTC_Fill(DVVectorLike& vec, const DeviceViewable& value) {
    return misc_run("fill_kernel", {view_arg(vec), dv_arg(value)}, vec.size(), {pod_bytes<size_t>(vec.size())});
}
bool TRTC_Sequence(DVVectorLike& vec, const DeviceViewable& value_init, const DeviceViewable& value_step) {
    return misc_run("sequence_kernel", {view_arg(vec), dv_arg(value_init), dv_arg(value_step)}, vec.size(),
                    {pod_bytes<size_t>(vec.size())});
}
bool TRTC_Sequence(DVVectorLike& vec, const DeviceViewable& value_init) {
    return TRTC_Sequence(vec, value_init, DVInt32(1));
}
bool TRTC_Sequence(DVVectorLike& vec) { return TRTC_Sequence(vec, DVInt32(0), DVInt32(1)); }
bool TRTC_Tabulate(DVVectorLike& vec, const Functor& op) {
    return misc_run("tabulate_kernel", {view_arg(vec), functor_arg(op)}, vec.size(), {pod_bytes<size_t>(vec.size())});
}
bool TRTC_For_Each(DVVectorLike& vec, const Functor& f) {
    return misc_run("for_each_kernel", {view_arg(vec), functor_arg(f)}, vec.size(), {pod_bytes<size_t>(vec.size())});
}
static bool transform_any(int mode, const DVVectorLike& in, const DVVectorLike* st, DVVectorLike& out,
                          const Functor& op, const Functor* pred) {
    return misc_run_t("transform_kernel", {num(mode)},
                      {view_arg(in), st ? view_arg(*st) : nothing_arg(), view_arg(out), functor_arg(op),
                       pred ? functor_arg(*pred) : nothing_arg()},
                      in.size(), {pod_bytes<size_t>(in.size())});
}
bool TRTC_Transform(const DVVectorLike& in, DVVectorLike& out, const Functor& op) {
    return transform_any(0, in, nullptr, out, op, nullptr);
}
bool TRTC_Transform_If(const DVVectorLike& in, DVVectorLike& out, const Functor& op, const Functor& pred) {
    return transform_any(1, in, nullptr, out, op, &pred);
}
bool TRTC_Transform_If_Stencil(const DVVectorLike& in, const DVVectorLike& stencil, DVVectorLike& out,
                               const Functor& op, const Functor& pred) {
    return transform_any(2, in, &stencil, out, op, &pred);
}
static bool transform_binary_any(bool stencil, const DVVectorLike& in1, const DVVectorLike& in2,
                                 const DVVectorLike* st, DVVectorLike& out, const Functor& op, const Functor* pred) {
    return misc_run_t("transform_binary_kernel", {stencil ? "true" : "false"},
                      {view_arg(in1), view_arg(in2), st ? view_arg(*st) : nothing_arg(), view_arg(out),
                       functor_arg(op), pred ? functor_arg(*pred) : nothing_arg()},
                      in1.size(), {pod_bytes<size_t>(in1.size())});
}
bool TRTC_Transform_Binary(const DVVectorLike& in1, const DVVectorLike& in2, DVVectorLike& out, const Functor& op) {
    return transform_binary_any(false, in1, in2, nullptr, out, op, nullptr);
}
bool TRTC_Transform_Binary_If_Stencil(const DVVectorLike& in1, const DVVectorLike& in2, const DVVectorLike& stencil,
                                      DVVectorLike& out, const Functor& op, const Functor& pred) {
    return transform_binary_any(true, in1, in2, &stencil, out, op, &pred);
}
// replace.cpp: both values are converted to the input's element type before use
static bool replace_any(bool use_pred, const DVVectorLike& in, DVVectorLike& out, const DeviceViewable* old_value,
                        const Functor* pred, const DeviceViewable& new_value) {
    const ViewArg nv = value_as_elem(new_value, in);
    const ViewArg ov = old_value ? value_as_elem(*old_value, in) : nv;
    if (ov.type != nv.type) {
        set_error("replace: old and new values must convert to the element type");
        return false;
    }
    return misc_run_t("replace_kernel", {use_pred ? "true" : "false"},
                      {view_arg(in), view_arg(out), ov, pred ? functor_arg(*pred) : nothing_arg(), nv}, in.size(),
                      {pod_bytes<size_t>(in.size())});
}
bool TRTC_Replace(DVVectorLike& vec, const DeviceViewable& old_value, const DeviceViewable& new_value) {
    return replace_any(false, vec, vec, &old_value, nullptr, new_value);
}
bool TRTC_Replace_If(DVVectorLike& vec, const Functor& pred, const DeviceViewable& new_value) {
    return replace_any(true, vec, vec, nullptr, &pred, new_value);
}
bool TRTC_Replace_Copy(const DVVectorLike& in, DVVectorLike& out, const DeviceViewable& old_value,
                       const DeviceViewable& new_value) {
    return replace_any(false, in, out, &old_value, nullptr, new_value);
}
bool TRTC_Replace_Copy_If(const DVVectorLike& in, DVVectorLike& out, const Functor& pred,
                          const DeviceViewable& new_value) {
    return replace_any(true, in, out, nullptr, &pred, new_value);
}
// out[0] = in[0], out[i] = op(in[i], in[i-1]) (adjacent_difference.cpp:3-25).  An output that
// may share memory with the input reads from a copy of it, so in-place calls are well defined.
bool TRTC_Adjacent_Difference(const DVVectorLike& in, DVVectorLike& out, const Functor& op) {
    const size_t n = in.size();
    if (n == 0) return true;
    if (!ensure_device()) return false;
    std::unique_ptr<DVVector> tmp;
    const DVVectorLike* src = &in;
    const void* ip = in.contiguous_data();
    const void* opp = out.contiguous_data();
    if (!ip || !opp || overlaps(ip, n * in.elem_size(), opp, out.size() * out.elem_size())) {
        tmp.reset(new DVVector(in.name_elem_cls().c_str(), n));
        if (!jit_copy(view_arg(in), view_arg(*tmp), n)) return false;
        src = tmp.get();
    }
    return misc_run("adjacent_difference_kernel", {view_arg(*src), view_arg(out), functor_arg(op)}, n,
                    {pod_bytes<size_t>(n)});
}
bool TRTC_Adjacent_Difference(const DVVectorLike& in, DVVectorLike& out) {
    return TRTC_Adjacent_Difference(in, out, Functor("Minus"));
}

// ---------------------------------------------------------------- copying
static bool gather_any(int sel, const DVVectorLike& map, const DVVectorLike* st, const DVVectorLike& in,
                       DVVectorLike& out, const Functor* pred) {
    return misc_run_t("gather_kernel", {num(sel)},
                      {view_arg(map), st ? view_arg(*st) : nothing_arg(), view_arg(in), view_arg(out),
                       pred ? functor_arg(*pred) : nothing_arg()},
                      map.size(), {pod_bytes<size_t>(map.size())});
}
bool TRTC_Gather(const DVVectorLike& map, const DVVectorLike& in, DVVectorLike& out) {
    return gather_any(0, map, nullptr, in, out, nullptr);
}
bool TRTC_Gather_If(const DVVectorLike& map, const DVVectorLike& stencil, const DVVectorLike& in, DVVectorLike& out) {
    return gather_any(1, map, &stencil, in, out, nullptr);
}
bool TRTC_Gather_If(const DVVectorLike& map, const DVVectorLike& stencil, const DVVectorLike& in, DVVectorLike& out,
                    const Functor& pred) {
    return gather_any(2, map, &stencil, in, out, &pred);
}
static bool scatter_any(int sel, const DVVectorLike& in, const DVVectorLike& map, const DVVectorLike* st,
                        DVVectorLike& out, const Functor* pred) {
    return misc_run_t("scatter_kernel", {num(sel)},
                      {view_arg(in), view_arg(map), st ? view_arg(*st) : nothing_arg(), view_arg(out),
                       pred ? functor_arg(*pred) : nothing_arg()},
                      in.size(), {pod_bytes<size_t>(in.size())});
}
bool TRTC_Scatter(const DVVectorLike& in, const DVVectorLike& map, DVVectorLike& out) {
    return scatter_any(0, in, map, nullptr, out, nullptr);
}
bool TRTC_Scatter_If(const DVVectorLike& in, const DVVectorLike& map, const DVVectorLike& stencil,
                     DVVectorLike& out) {
    return scatter_any(1, in, map, &stencil, out, nullptr);
}
bool TRTC_Scatter_If(const DVVectorLike& in, const DVVectorLike& map, const DVVectorLike& stencil,
                     DVVectorLike& out, const Functor& pred) {
    return scatter_any(2, in, map, &stencil, out, &pred);
}
bool TRTC_Swap(DVVectorLike& a, DVVectorLike& b) {
    return misc_run("swap_kernel", {view_arg(a), view_arg(b)}, a.size(), {pod_bytes<size_t>(a.size())});
}

// ---------------------------------------------------------------- reductions
// count.cpp: the value is converted to the element type (vec[i] == (value_t)value)
bool TRTC_Count(const DVVectorLike& vec, const DeviceViewable& value, size_t& result) {
    return count_run(0, vec, value_as_elem(value, vec), nothing_arg(), result);
}
bool TRTC_Count_If(const DVVectorLike& vec, const Functor& pred, size_t& result) {
    return count_run(1, vec, nothing_arg(), functor_arg(pred), result);
}
bool TRTC_Equal(const DVVectorLike& vec1, const DVVectorLike& vec2, bool& result) {
    size_t r = 0;
    if (!find_first(5, view_arg(vec1), view_arg(vec2), nothing_arg(), nothing_arg(), 0, vec1.size(), r)) return false;
    result = r >= vec1.size();
    return true;
}
bool TRTC_Equal(const DVVectorLike& vec1, const DVVectorLike& vec2, const Functor& pred, bool& result) {
    size_t r = 0;
    if (!find_first(3, view_arg(vec1), view_arg(vec2), nothing_arg(), functor_arg(pred), 0, vec1.size(), r))
        return false;
    result = r >= vec1.size();
    return true;
}
// logical.cpp: an empty range gives all_of false, any_of false, none_of true
bool TRTC_All_Of(const DVVectorLike& vec, const Functor& pred, bool& result) {
    result = false;
    if (vec.size() < 1) return true;
    size_t r = 0;
    if (!find_first(2, view_arg(vec), nothing_arg(), nothing_arg(), functor_arg(pred), 0, vec.size(), r))
        return false;
    result = r >= vec.size();
    return true;
}
bool TRTC_Any_Of(const DVVectorLike& vec, const Functor& pred, bool& result) {
    result = false;
    if (vec.size() < 1) return true;
    size_t r = 0;
    if (!find_first(1, view_arg(vec), nothing_arg(), nothing_arg(), functor_arg(pred), 0, vec.size(), r))
        return false;
    result = r < vec.size();
    return true;
}
bool TRTC_None_Of(const DVVectorLike& vec, const Functor& pred, bool& result) {
    result = true;
    if (vec.size() < 1) return true;
    bool any = false;
    if (!TRTC_Any_Of(vec, pred, any)) return false;
    result = !any;
    return true;
}
bool TRTC_Min_Element(const DVVectorLike& vec, const Functor& comp, size_t& id_min) {
    return index_tree(false, vec, comp, id_min);
}
bool TRTC_Max_Element(const DVVectorLike& vec, const Functor& comp, size_t& id_max) {
    return index_tree(true, vec, comp, id_max);
}
bool TRTC_Max_Element(const DVVectorLike& vec, size_t& id_max) { return index_tree(true, vec, Functor("Less"), id_max); }
// both indices of the reference's Pair reduction: the same tree shape for each half
bool TRTC_MinMax_Element(const DVVectorLike& vec, const Functor& comp, size_t& id_min, size_t& id_max) {
    return index_tree(false, vec, comp, id_min) && index_tree(true, vec, comp, id_max);
}
bool TRTC_MinMax_Element(const DVVectorLike& vec, size_t& id_min, size_t& id_max) {
    return TRTC_MinMax_Element(vec, Functor("Less"), id_min, id_max);
}

namespace {
// BinaryTransformView<T, A, B, Op> { A _a; B _b; Op _op; }: element i = op(a[i], b[i]) in T
class DVBinaryTransform : public DVVectorLike {
public:
    DVBinaryTransform(const std::string& T, const DVVectorLike& a, const DVVectorLike& b, const Functor& op)
        : DVVectorLike(T.c_str(), T.c_str(), a.size()) {
        const ViewArg x = view_arg(a), y = view_arg(b);
        m_name_view_cls = "trtc::BinaryTransformView<" + T + ", " + x.type + ", " + y.type + ", " +
                          op.name_view_cls() + ">";
        StructLayout sl;
        const Layout lx = x.contiguous ? Layout{16, 8} : Layout{a.view_size(), a.view_align()};
        const Layout ly = y.contiguous ? Layout{16, 8} : Layout{b.view_size(), b.view_align()};
        const size_t o0 = sl.add(lx), o1 = sl.add(ly), o2 = sl.add(Layout{op.view_size(), op.view_align()});
        const Layout l = sl.finish();
        m_buf.assign(l.size, 0);
        const ViewBuf fv = op.view();
        memcpy(m_buf.data() + o0, x.bytes.data(), x.bytes.size());
        memcpy(m_buf.data() + o1, y.bytes.data(), y.bytes.size());
        memcpy(m_buf.data() + o2, fv.data(), fv.size());
        m_view_size = l.size;
        m_view_align = l.align;
        layout_register(m_name_view_cls, l);
    }
    ViewBuf view() const override { return m_buf; }

private:
    ViewBuf m_buf;
};
}  // namespace

// init op1 op2(a0, b0) op1 op2(a1, b1) ... in the init's type (inner_product.cpp:4-30)
bool TRTC_Inner_Product(const DVVectorLike& vec1, const DVVectorLike& vec2, const DeviceViewable& init, ViewBuf& ret,
                        const Functor& op1, const Functor& op2) {
    const std::string T = init.name_view_cls();
    if (vec1.size() == 0) { ret = init.view(); return true; }
    if (!ensure_device()) return false;
    Layout tl;
    if (!layout_of(T, tl)) { set_error("inner_product: unknown value type " + T); return false; }
    DVBinaryTransform terms(T, vec1, vec2, op2);
    void* res = nullptr;
    if (!jit_scan(terms, nullptr, nullptr, T, op1, 3, init.view(), &res, "trtc_misc.cuh")) return false;
    return fetch_result(res, tl.size, ret, tl.size > 16);
}
bool TRTC_Inner_Product(const DVVectorLike& vec1, const DVVectorLike& vec2, const DeviceViewable& init,
                        ViewBuf& ret) {
    return TRTC_Inner_Product(vec1, vec2, init, ret, Functor("Plus"), Functor("trtc::ProductOf"));
}

// ---------------------------------------------------------------- searching
// find.cpp / mismatch.cpp: (size_t)-1 when there is no such index
bool TRTC_Find(const DVVectorLike& vec, const DeviceViewable& value, size_t& result) {
    return find_or_none(0, view_arg(vec), nothing_arg(), dv_arg(value), nothing_arg(), vec.size(), result);
}
bool TRTC_Find_If(const DVVectorLike& vec, const Functor& pred, size_t& result) {
    return find_or_none(1, view_arg(vec), nothing_arg(), nothing_arg(), functor_arg(pred), vec.size(), result);
}
bool TRTC_Find_If_Not(const DVVectorLike& vec, const Functor& pred, size_t& result) {
    return find_or_none(2, view_arg(vec), nothing_arg(), nothing_arg(), functor_arg(pred), vec.size(), result);
}
bool TRTC_Mismatch(const DVVectorLike& vec1, const DVVectorLike& vec2, size_t& result) {
    return find_or_none(4, view_arg(vec1), view_arg(vec2), nothing_arg(), nothing_arg(), vec1.size(), result);
}
bool TRTC_Mismatch(const DVVectorLike& vec1, const DVVectorLike& vec2, const Functor& pred, size_t& result) {
    return find_or_none(3, view_arg(vec1), view_arg(vec2), nothing_arg(), functor_arg(pred), vec1.size(), result);
}
// sort.cpp:93-103: first i with comp(v[i], v[i-1]), else the size
bool TRTC_Is_Sorted_Until(const DVVectorLike& vec, const Functor& comp, size_t& result) {
    return find_first(6, view_arg(vec), nothing_arg(), nothing_arg(), functor_arg(comp), 1, vec.size(), result);
}
bool TRTC_Is_Sorted_Until(const DVVectorLike& vec, size_t& result) {
    return TRTC_Is_Sorted_Until(vec, Functor("Less"), result);
}
bool TRTC_Is_Sorted(const DVVectorLike& vec, const Functor& comp, bool& result) {
    size_t r = 0;
    if (!TRTC_Is_Sorted_Until(vec, comp, r)) return false;
    result = r >= vec.size();
    return true;
}
bool TRTC_Is_Sorted(const DVVectorLike& vec, bool& result) { return TRTC_Is_Sorted(vec, Functor("Less"), result); }
// partition.cpp:127-197: fails on an empty range; for a partitioned range the first index
// whose element fails pred (the size when all pass)
bool TRTC_Partition_Point(const DVVectorLike& vec, const Functor& pred, size_t& result) {
    if (vec.size() == 0) return false;
    return find_first(2, view_arg(vec), nothing_arg(), nothing_arg(), functor_arg(pred), 0, vec.size(), result);
}
// partition.cpp:199-214: no element satisfying pred right after one that does not
bool TRTC_Is_Partitioned(const DVVectorLike& vec, const Functor& pred, bool& result) {
    result = true;
    if (vec.size() == 0) return true;
    size_t r = 0;
    if (!find_first(7, view_arg(vec), nothing_arg(), nothing_arg(), functor_arg(pred), 1, vec.size(), r)) return false;
    result = r >= vec.size();
    return true;
}

// ---------------------------------------------------------------- merging
bool TRTC_Merge(const DVVectorLike& a, const DVVectorLike& b, DVVectorLike& out, const Functor& comp) {
    const size_t n = a.size() > b.size() ? a.size() : b.size();
    return misc_run_t("merge_kernel", {"false"},
                      {view_arg(a), view_arg(b), view_arg(out), nothing_arg(), nothing_arg(), nothing_arg(),
                       functor_arg(comp)},
                      n, {pod_bytes<size_t>(a.size()), pod_bytes<size_t>(b.size())});
}
bool TRTC_Merge(const DVVectorLike& a, const DVVectorLike& b, DVVectorLike& out) {
    return TRTC_Merge(a, b, out, Functor("Less"));
}
bool TRTC_Merge_By_Key(const DVVectorLike& keys1, const DVVectorLike& keys2, const DVVectorLike& values1,
                       const DVVectorLike& values2, DVVectorLike& keys_out, DVVectorLike& values_out,
                       const Functor& comp) {
    const size_t n = keys1.size() > keys2.size() ? keys1.size() : keys2.size();
    return misc_run_t("merge_kernel", {"true"},
                      {view_arg(keys1), view_arg(keys2), view_arg(keys_out), view_arg(values1), view_arg(values2),
                       view_arg(values_out), functor_arg(comp)},
                      n, {pod_bytes<size_t>(keys1.size()), pod_bytes<size_t>(keys2.size())});
}
bool TRTC_Merge_By_Key(const DVVectorLike& keys1, const DVVectorLike& keys2, const DVVectorLike& values1,
                       const DVVectorLike& values2, DVVectorLike& keys_out, DVVectorLike& values_out) {
    return TRTC_Merge_By_Key(keys1, keys2, values1, values2, keys_out, values_out, Functor("Less"));
}
