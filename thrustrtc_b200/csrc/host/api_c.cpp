// api_c.cpp -- the drop-in C ABI (include/thrustrtc_b200.h; python/api.h of the reference).
// Handles are heap objects of the C++ object model; NULL functor / init arguments select
// the default overloads exactly as python/api_*.cpp do.
#include "thrustrtc_b200.h"
#include "thrustrtc_cpp.h"
#include "trtc_runtime.h"

#include <string>
#include <vector>

typedef std::vector<std::string> StrArray;
typedef std::vector<const DeviceViewable*> PtrArray;

#define TRTC_EXPORT extern "C" __attribute__((visibility("default")))

// ------------------------------------------------------------------ utils
TRTC_EXPORT void* n_string_array_create(unsigned long long size, const char* const* strs) {
    StrArray* a = new StrArray(size);
    for (size_t i = 0; i < size; i++) (*a)[i] = strs[i];
    return a;
}
TRTC_EXPORT void n_string_array_destroy(void* p) { delete (StrArray*)p; }
TRTC_EXPORT void* n_pointer_array_create(unsigned long long size, const void* const* ptrs) {
    PtrArray* a = new PtrArray(size);
    for (size_t i = 0; i < size; i++) (*a)[i] = (const DeviceViewable*)ptrs[i];
    return a;
}
TRTC_EXPORT void n_pointer_array_destroy(void* p) { delete (PtrArray*)p; }
TRTC_EXPORT void* n_dim3_create(unsigned x, unsigned y, unsigned z) { return new dim_type{x, y, z}; }
TRTC_EXPORT void n_dim3_destroy(void* p) { delete (dim_type*)p; }

// ------------------------------------------------------------------ context
TRTC_EXPORT void n_set_libnvrtc_path(const char* path) { set_libnvrtc_path(path); }
TRTC_EXPORT int n_trtc_try_init() { return TRTC_Try_Init() ? 0 : -100; }
TRTC_EXPORT int n_get_ptx_arch() { return TRTC_Get_PTX_Arch(); }
TRTC_EXPORT void n_set_verbose(unsigned v) { TRTC_Set_Verbose(v != 0); }
TRTC_EXPORT void n_set_kernel_debug(unsigned v) { TRTC_Set_Kernel_Debug(v != 0); }
TRTC_EXPORT void n_add_include_dir(const char* dir) { TRTC_Add_Include_Dir(dir); }
TRTC_EXPORT void n_add_built_in_header(const char* fn, const char* content) { TRTC_Add_Built_In_Header(fn, content); }
TRTC_EXPORT void n_add_inlcude_filename(const char* fn) { TRTC_Add_Inlcude_Filename(fn); }
TRTC_EXPORT void n_add_code_block(const char* line) { TRTC_Add_Code_Block(line); }
TRTC_EXPORT void n_add_constant_object(const char* name, void* cptr) {
    TRTC_Add_Constant_Object(name, *(const DeviceViewable*)cptr);
}
TRTC_EXPORT void n_wait() { TRTC_Wait(); }

// ------------------------------------------------------------------ JIT launchers
static std::vector<const char*> c_strs(const StrArray& a) {
    std::vector<const char*> r;
    for (auto& s : a) r.push_back(s.c_str());
    return r;
}
TRTC_EXPORT void* n_kernel_create(void* ptr_param_list, const char* body) {
    return new TRTC_Kernel(c_strs(*(StrArray*)ptr_param_list), body);
}
TRTC_EXPORT void n_kernel_destroy(void* p) { delete (TRTC_Kernel*)p; }
TRTC_EXPORT int n_kernel_num_params(void* p) { return (int)((TRTC_Kernel*)p)->num_params(); }
TRTC_EXPORT int n_kernel_calc_optimal_block_size(void* pk, void* pargs, unsigned smem) {
    TRTC_Kernel* k = (TRTC_Kernel*)pk;
    PtrArray* a = (PtrArray*)pargs;
    if (a->size() != k->num_params()) return -2;
    int bs;
    return k->calc_optimal_block_size(a->data(), bs, smem) ? bs : -1;
}
TRTC_EXPORT int n_kernel_calc_number_blocks(void* pk, void* pargs, int sizeBlock, unsigned smem) {
    TRTC_Kernel* k = (TRTC_Kernel*)pk;
    PtrArray* a = (PtrArray*)pargs;
    if (a->size() != k->num_params()) return -2;
    int nb;
    return k->calc_number_blocks(a->data(), sizeBlock, nb, smem) ? nb : -1;
}
TRTC_EXPORT int n_kernel_launch(void* pk, void* pgrid, void* pblock, void* pargs, int smem) {
    TRTC_Kernel* k = (TRTC_Kernel*)pk;
    PtrArray* a = (PtrArray*)pargs;
    if (a->size() != k->num_params()) return -2;
    return k->launch(*(dim_type*)pgrid, *(dim_type*)pblock, a->data(), (unsigned)smem) ? 0 : -1;
}
TRTC_EXPORT void* n_for_create(void* ptr_param_list, const char* name_iter, const char* body) {
    return new TRTC_For(c_strs(*(StrArray*)ptr_param_list), name_iter, body);
}
TRTC_EXPORT void n_for_destroy(void* p) { delete (TRTC_For*)p; }
TRTC_EXPORT int n_for_num_params(void* p) { return (int)((TRTC_For*)p)->num_params(); }
TRTC_EXPORT int n_for_launch(void* p, int begin, int end, void* pargs) {
    TRTC_For* f = (TRTC_For*)p;
    PtrArray* a = (PtrArray*)pargs;
    if (a->size() != f->num_params()) return -2;
    return f->launch((size_t)begin, (size_t)end, a->data()) ? 0 : -1;
}
TRTC_EXPORT int n_for_launch_n(void* p, int n, void* pargs) {
    TRTC_For* f = (TRTC_For*)p;
    PtrArray* a = (PtrArray*)pargs;
    if (a->size() != f->num_params()) return -2;
    return f->launch_n((size_t)n, a->data()) ? 0 : -1;
}

// ------------------------------------------------------------------ device viewables
TRTC_EXPORT const char* n_dv_name_view_cls(void* p) { return ((DeviceViewable*)p)->name_view_cls().c_str(); }
TRTC_EXPORT void n_dv_destroy(void* p) { delete (DeviceViewable*)p; }

#define TRTC_DV_SCALAR(lower, Cls, ctype, argt, rett)                                              \
    TRTC_EXPORT void* n_dv##lower##_create(argt v) { return new Cls((ctype)v); }                   \
    TRTC_EXPORT rett n_dv##lower##_value(void* p) {                                               \
        ViewBuf b = ((DeviceViewable*)p)->view();                                                  \
        return (rett)(*(const ctype*)b.data());                                                    \
    }
TRTC_DV_SCALAR(int8, DVInt8, int8_t, int, int)
TRTC_DV_SCALAR(uint8, DVUInt8, uint8_t, unsigned, unsigned)
TRTC_DV_SCALAR(int16, DVInt16, int16_t, int, int)
TRTC_DV_SCALAR(uint16, DVUInt16, uint16_t, unsigned, unsigned)
TRTC_DV_SCALAR(int32, DVInt32, int32_t, int, int)
TRTC_DV_SCALAR(uint32, DVUInt32, uint32_t, unsigned, unsigned)
TRTC_DV_SCALAR(int64, DVInt64, int64_t, long long, long long)
TRTC_DV_SCALAR(uint64, DVUInt64, uint64_t, unsigned long long, unsigned long long)
TRTC_DV_SCALAR(float, DVFloat, float, float, float)
TRTC_DV_SCALAR(double, DVDouble, double, double, double)
#undef TRTC_DV_SCALAR
TRTC_EXPORT void* n_dvbool_create(int v) { return new DVBool(v != 0); }
TRTC_EXPORT int n_dvbool_value(void* p) {
    ViewBuf b = ((DeviceViewable*)p)->view();
    return *(const bool*)b.data() ? 1 : 0;
}
TRTC_EXPORT void* n_dvcomplex64_create(float re, float im) { return new DVComplex64(re, im); }
TRTC_EXPORT float n_dvcomplex64_real(void* p) {
    ViewBuf b = ((DeviceViewable*)p)->view();
    return ((const float*)b.data())[0];
}
TRTC_EXPORT float n_dvcomplex64_imag(void* p) {
    ViewBuf b = ((DeviceViewable*)p)->view();
    return ((const float*)b.data())[1];
}
TRTC_EXPORT void* n_dvcomplex128_create(double re, double im) { return new DVComplex128(re, im); }
TRTC_EXPORT double n_dvcomplex128_real(void* p) {
    ViewBuf b = ((DeviceViewable*)p)->view();
    return ((const double*)b.data())[0];
}
TRTC_EXPORT double n_dvcomplex128_imag(void* p) {
    ViewBuf b = ((DeviceViewable*)p)->view();
    return ((const double*)b.data())[1];
}

// ------------------------------------------------------------------ vectors
TRTC_EXPORT const char* n_dvvectorlike_name_elem_cls(void* p) { return ((DVVectorLike*)p)->name_elem_cls().c_str(); }
TRTC_EXPORT unsigned long long n_dvvectorlike_size(void* p) { return ((DVVectorLike*)p)->size(); }
TRTC_EXPORT void* n_dvvector_create(const char* elem_cls, unsigned long long size, void* hdata) {
    if (!TRTC_Try_Init()) return nullptr;
    DVVector* v = new DVVector(elem_cls, (size_t)size, hdata);
    if (size > 0 && !v->data()) { delete v; return nullptr; }
    return v;
}
TRTC_EXPORT void n_dvvector_to_host(void* p, void* hdata, unsigned long long begin, unsigned long long end) {
    ((DVVector*)p)->to_host(hdata, (size_t)begin, (size_t)end);
}
TRTC_EXPORT void* n_dvvector_from_dvs(void* ptr_dvs) {
    PtrArray* dvs = (PtrArray*)ptr_dvs;
    if (dvs->empty()) return nullptr;
    const std::string cls = (*dvs)[0]->name_view_cls();
    for (auto d : *dvs)
        if (d->name_view_cls() != cls) return nullptr;
    const size_t es = (*dvs)[0]->view_size();
    std::vector<char> buf(es * dvs->size());
    for (size_t i = 0; i < dvs->size(); i++) {
        ViewBuf b = (*dvs)[i]->view();
        memcpy(buf.data() + es * i, b.data(), es);
    }
    return new DVVector(cls.c_str(), dvs->size(), buf.data());
}
TRTC_EXPORT void* n_dvvectoradaptor_create(const char* elem_cls, unsigned long long size, void* data) {
    return new DVVectorAdaptor(elem_cls, (size_t)size, data);
}
// a range over a plain vector is itself a plain vector (python/api_DVVector.cpp:58-75)
TRTC_EXPORT void* n_dvrange_create(void* ptr_in, unsigned long long begin, unsigned long long end) {
    DVVectorLike* v = (DVVectorLike*)ptr_in;
    if (DVVector* pv = dynamic_cast<DVVector*>(v)) return new DVVectorAdaptor(*pv, (size_t)begin, (size_t)end);
    if (DVVectorAdaptor* pa = dynamic_cast<DVVectorAdaptor*>(v)) return new DVVectorAdaptor(*pa, (size_t)begin, (size_t)end);
    return new DVRange(*v, (size_t)begin, (size_t)end);
}

TRTC_EXPORT void* n_dvconstant_create(void* cptr, unsigned long long size) {
    return new DVConstant(*(DeviceViewable*)cptr, (size_t)size);
}
TRTC_EXPORT void* n_dvcounter_create(void* cptr, unsigned long long size) {
    return new DVCounter(*(DeviceViewable*)cptr, (size_t)size);
}
TRTC_EXPORT void* n_dvdiscard_create(const char* elem_cls, unsigned long long size) {
    return new DVDiscard(elem_cls, (size_t)size);
}
TRTC_EXPORT void* n_dvpermutation_create(void* pv, void* pi) {
    return new DVPermutation(*(DVVectorLike*)pv, *(DVVectorLike*)pi);
}
TRTC_EXPORT void* n_dvreverse_create(void* pv) { return new DVReverse(*(DVVectorLike*)pv); }
TRTC_EXPORT void* n_dvtransform_create(void* pin, const char* elem_cls, void* pop) {
    return new DVTransform(*(DVVectorLike*)pin, elem_cls, *(Functor*)pop);
}

// DVTuple / DVZipped / DVCustomVector -- python/api_DVTuple.cpp:8-20, api_FakeVectors.cpp:52-81
static std::vector<CapturedDeviceViewable> captured(void* ptr_dvs, void* ptr_names) {
    PtrArray* dvs = (PtrArray*)ptr_dvs;
    StrArray* names = (StrArray*)ptr_names;
    std::vector<CapturedDeviceViewable> m(dvs->size());
    for (size_t i = 0; i < dvs->size(); i++) {
        m[i].obj_name = (*names)[i].c_str();
        m[i].obj = (*dvs)[i];
    }
    return m;
}
TRTC_EXPORT void* n_dvtuple_create(void* ptr_dvs, void* ptr_names) {
    if (((PtrArray*)ptr_dvs)->size() != ((StrArray*)ptr_names)->size()) {
        trtc_host::set_error("dvtuple: number of objects and names differ");
        return nullptr;
    }
    return new DVTuple(captured(ptr_dvs, ptr_names));
}
TRTC_EXPORT void* n_dvzipped_create(void* ptr_vecs, void* ptr_elem_names) {
    PtrArray* a = (PtrArray*)ptr_vecs;
    StrArray* names = (StrArray*)ptr_elem_names;
    if (a->empty() || a->size() != names->size()) {
        trtc_host::set_error("dvzipped: number of vectors and element names differ");
        return nullptr;
    }
    std::vector<DVVectorLike*> vecs(a->size());
    for (size_t i = 0; i < a->size(); i++) vecs[i] = (DVVectorLike*)(*a)[i];
    return new DVZipped(vecs, c_strs(*names));
}
TRTC_EXPORT void* n_dvcustomvector_create(void* ptr_dvs, void* ptr_names, const char* name_idx, const char* body,
                                          const char* elem_cls, unsigned long long size, unsigned read_only) {
    return new DVCustomVector(captured(ptr_dvs, ptr_names), name_idx, body, elem_cls, (size_t)size, read_only != 0);
}

// ------------------------------------------------------------------ functors
TRTC_EXPORT void* n_functor_create(void* ptr_dvs, void* ptr_names, void* ptr_functor_params, const char* code_body) {
    PtrArray* dvs = (PtrArray*)ptr_dvs;
    StrArray* names = (StrArray*)ptr_names;
    std::vector<CapturedDeviceViewable> arg_map(dvs->size());
    for (size_t i = 0; i < dvs->size(); i++) {
        arg_map[i].obj_name = (*names)[i].c_str();
        arg_map[i].obj = (*dvs)[i];
    }
    return new Functor(arg_map, c_strs(*(StrArray*)ptr_functor_params), code_body);
}
TRTC_EXPORT void* n_built_in_functor_create(const char* name) { return new Functor(name); }

// ------------------------------------------------------------------ algorithms
#define V(p) (*(DVVectorLike*)(p))
#define F(p) (*(Functor*)(p))
#define D(p) (*(DeviceViewable*)(p))

TRTC_EXPORT int n_copy(void* in, void* out) { return TRTC_Copy(V(in), V(out)) ? 0 : -1; }

TRTC_EXPORT void* n_reduce(void* vec, void* init, void* op) {
    ViewBuf ret;
    bool ok;
    if (!init) ok = TRTC_Reduce(V(vec), ret);
    else if (!op) ok = TRTC_Reduce(V(vec), D(init), ret);
    else ok = TRTC_Reduce(V(vec), D(init), F(op), ret);
    return ok ? dv_from_viewbuf(ret, V(vec).name_elem_cls().c_str()) : nullptr;
}
TRTC_EXPORT unsigned n_reduce_by_key(void* ki, void* vi, void* ko, void* vo, void* pred, void* op) {
    if (!pred) return TRTC_Reduce_By_Key(V(ki), V(vi), V(ko), V(vo));
    if (!op) return TRTC_Reduce_By_Key(V(ki), V(vi), V(ko), V(vo), F(pred));
    return TRTC_Reduce_By_Key(V(ki), V(vi), V(ko), V(vo), F(pred), F(op));
}
TRTC_EXPORT unsigned long long n_min_element(void* vec, void* comp) {
    size_t id = 0;
    const bool ok = comp ? TRTC_Min_Element(V(vec), F(comp), id) : TRTC_Min_Element(V(vec), id);
    return ok ? (unsigned long long)id : ~0ull;
}
// searches -- python/api_Searching.cpp:110-245 (NULL comparator = Less)
TRTC_EXPORT unsigned long long n_lower_bound(void* vec, void* value, void* comp) {
    size_t r = 0;
    const bool ok = comp ? TRTC_Lower_Bound(V(vec), D(value), F(comp), r) : TRTC_Lower_Bound(V(vec), D(value), r);
    return ok ? (unsigned long long)r : ~0ull;
}
TRTC_EXPORT unsigned long long n_upper_bound(void* vec, void* value, void* comp) {
    size_t r = 0;
    const bool ok = comp ? TRTC_Upper_Bound(V(vec), D(value), F(comp), r) : TRTC_Upper_Bound(V(vec), D(value), r);
    return ok ? (unsigned long long)r : ~0ull;
}
TRTC_EXPORT int n_binary_search(void* vec, void* value, void* comp) {
    bool r = false;
    const bool ok = comp ? TRTC_Binary_Search(V(vec), D(value), F(comp), r) : TRTC_Binary_Search(V(vec), D(value), r);
    return ok ? (r ? 1 : 0) : -1;
}
TRTC_EXPORT int n_lower_bound_v(void* vec, void* values, void* result, void* comp) {
    return (comp ? TRTC_Lower_Bound_V(V(vec), V(values), V(result), F(comp))
                 : TRTC_Lower_Bound_V(V(vec), V(values), V(result))) ? 0 : -1;
}
TRTC_EXPORT int n_upper_bound_v(void* vec, void* values, void* result, void* comp) {
    return (comp ? TRTC_Upper_Bound_V(V(vec), V(values), V(result), F(comp))
                 : TRTC_Upper_Bound_V(V(vec), V(values), V(result))) ? 0 : -1;
}
TRTC_EXPORT int n_binary_search_v(void* vec, void* values, void* result, void* comp) {
    return (comp ? TRTC_Binary_Search_V(V(vec), V(values), V(result), F(comp))
                 : TRTC_Binary_Search_V(V(vec), V(values), V(result))) ? 0 : -1;
}
TRTC_EXPORT void* n_transform_reduce(void* vec, void* uop, void* init, void* bop) {
    ViewBuf ret;
    if (!TRTC_Transform_Reduce(V(vec), F(uop), D(init), F(bop), ret)) return nullptr;
    return dv_from_viewbuf(ret, D(init).name_view_cls().c_str());
}

TRTC_EXPORT int n_inclusive_scan(void* in, void* out, void* op) {
    bool ok = op ? TRTC_Inclusive_Scan(V(in), V(out), F(op)) : TRTC_Inclusive_Scan(V(in), V(out));
    return ok ? 0 : -1;
}
TRTC_EXPORT int n_exclusive_scan(void* in, void* out, void* init, void* op) {
    bool ok;
    if (!init) ok = TRTC_Exclusive_Scan(V(in), V(out));
    else if (!op) ok = TRTC_Exclusive_Scan(V(in), V(out), D(init));
    else ok = TRTC_Exclusive_Scan(V(in), V(out), D(init), F(op));
    return ok ? 0 : -1;
}
TRTC_EXPORT int n_inclusive_scan_by_key(void* k, void* v, void* out, void* pred, void* op) {
    bool ok;
    if (!pred) ok = TRTC_Inclusive_Scan_By_Key(V(k), V(v), V(out));
    else if (!op) ok = TRTC_Inclusive_Scan_By_Key(V(k), V(v), V(out), F(pred));
    else ok = TRTC_Inclusive_Scan_By_Key(V(k), V(v), V(out), F(pred), F(op));
    return ok ? 0 : -1;
}
TRTC_EXPORT int n_exclusive_scan_by_key(void* k, void* v, void* out, void* init, void* pred, void* op) {
    bool ok;
    if (!init) ok = TRTC_Exclusive_Scan_By_Key(V(k), V(v), V(out));
    else if (!pred) ok = TRTC_Exclusive_Scan_By_Key(V(k), V(v), V(out), D(init));
    else if (!op) ok = TRTC_Exclusive_Scan_By_Key(V(k), V(v), V(out), D(init), F(pred));
    else ok = TRTC_Exclusive_Scan_By_Key(V(k), V(v), V(out), D(init), F(pred), F(op));
    return ok ? 0 : -1;
}
TRTC_EXPORT int n_transform_inclusive_scan(void* in, void* out, void* uop, void* bop) {
    return TRTC_Transform_Inclusive_Scan(V(in), V(out), F(uop), F(bop)) ? 0 : -1;
}
// the reference returns 1 here on failure (python/api_PrefixSums.cpp:112), which its Python
// layer does not treat as an error; this build reports -1 like every other int entry point
TRTC_EXPORT int n_transform_exclusive_scan(void* in, void* out, void* uop, void* init, void* bop) {
    return TRTC_Transform_Exclusive_Scan(V(in), V(out), F(uop), D(init), F(bop)) ? 0 : -1;
}

TRTC_EXPORT unsigned n_copy_if(void* in, void* out, void* pred) { return TRTC_Copy_If(V(in), V(out), F(pred)); }
TRTC_EXPORT unsigned n_copy_if_stencil(void* in, void* st, void* out, void* pred) {
    return TRTC_Copy_If_Stencil(V(in), V(st), V(out), F(pred));
}
TRTC_EXPORT unsigned n_remove(void* vec, void* value) { return TRTC_Remove(V(vec), D(value)); }
TRTC_EXPORT unsigned n_remove_copy(void* in, void* out, void* value) { return TRTC_Remove_Copy(V(in), V(out), D(value)); }
TRTC_EXPORT unsigned n_remove_if(void* vec, void* pred) { return TRTC_Remove_If(V(vec), F(pred)); }
TRTC_EXPORT unsigned n_remove_copy_if(void* in, void* out, void* pred) {
    return TRTC_Remove_Copy_If(V(in), V(out), F(pred));
}
TRTC_EXPORT unsigned n_remove_if_stencil(void* vec, void* st, void* pred) {
    return TRTC_Remove_If_Stencil(V(vec), V(st), F(pred));
}
TRTC_EXPORT unsigned n_remove_copy_if_stencil(void* in, void* st, void* out, void* pred) {
    return TRTC_Remove_Copy_If_Stencil(V(in), V(st), V(out), F(pred));
}
TRTC_EXPORT unsigned n_unique(void* vec, void* pred) {
    return pred ? TRTC_Unique(V(vec), F(pred)) : TRTC_Unique(V(vec));
}
TRTC_EXPORT unsigned n_unique_copy(void* in, void* out, void* pred) {
    return pred ? TRTC_Unique_Copy(V(in), V(out), F(pred)) : TRTC_Unique_Copy(V(in), V(out));
}
TRTC_EXPORT unsigned n_unique_by_key(void* k, void* v, void* pred) {
    return pred ? TRTC_Unique_By_Key(V(k), V(v), F(pred)) : TRTC_Unique_By_Key(V(k), V(v));
}
TRTC_EXPORT unsigned n_unique_by_key_copy(void* ki, void* vi, void* ko, void* vo, void* pred) {
    return pred ? TRTC_Unique_By_Key_Copy(V(ki), V(vi), V(ko), V(vo), F(pred))
                : TRTC_Unique_By_Key_Copy(V(ki), V(vi), V(ko), V(vo));
}
TRTC_EXPORT unsigned n_partition(void* vec, void* pred) { return TRTC_Partition(V(vec), F(pred)); }
TRTC_EXPORT unsigned n_partition_stencil(void* vec, void* st, void* pred) {
    return TRTC_Partition_Stencil(V(vec), V(st), F(pred));
}
TRTC_EXPORT unsigned n_partition_copy(void* in, void* t, void* f, void* pred) {
    return TRTC_Partition_Copy(V(in), V(t), V(f), F(pred));
}
TRTC_EXPORT unsigned n_partition_copy_stencil(void* in, void* st, void* t, void* f, void* pred) {
    return TRTC_Partition_Copy_Stencil(V(in), V(st), V(t), V(f), F(pred));
}

TRTC_EXPORT int n_sort(void* vec, void* comp) {
    return (comp ? TRTC_Sort(V(vec), F(comp)) : TRTC_Sort(V(vec))) ? 0 : -1;
}
TRTC_EXPORT int n_sort_by_key(void* keys, void* values, void* comp) {
    return (comp ? TRTC_Sort_By_Key(V(keys), V(values), F(comp)) : TRTC_Sort_By_Key(V(keys), V(values))) ? 0 : -1;
}

// ---- the remaining entry points (python/api.h:104-186); return conventions of the
// reference's python/api_*.cpp: 0 / -1 for int status, 1 / 0 / -1 for booleans,
// (unsigned long long)-1 for failed counts and indices, NULL for failed value results.
// transformations -- python/api_Transformations.cpp
TRTC_EXPORT int n_fill(void* vec, void* value) { return TRTC_Fill(V(vec), D(value)) ? 0 : -1; }
TRTC_EXPORT int n_replace(void* vec, void* old_value, void* new_value) {
    return TRTC_Replace(V(vec), D(old_value), D(new_value)) ? 0 : -1;
}
TRTC_EXPORT int n_replace_if(void* vec, void* pred, void* new_value) {
    return TRTC_Replace_If(V(vec), F(pred), D(new_value)) ? 0 : -1;
}
TRTC_EXPORT int n_replace_copy(void* in, void* out, void* old_value, void* new_value) {
    return TRTC_Replace_Copy(V(in), V(out), D(old_value), D(new_value)) ? 0 : -1;
}
TRTC_EXPORT int n_replace_copy_if(void* in, void* out, void* pred, void* new_value) {
    return TRTC_Replace_Copy_If(V(in), V(out), F(pred), D(new_value)) ? 0 : -1;
}
TRTC_EXPORT int n_for_each(void* vec, void* f) { return TRTC_For_Each(V(vec), F(f)) ? 0 : -1; }
TRTC_EXPORT int n_adjacent_difference(void* in, void* out, void* op) {
    return (op ? TRTC_Adjacent_Difference(V(in), V(out), F(op)) : TRTC_Adjacent_Difference(V(in), V(out))) ? 0 : -1;
}
TRTC_EXPORT int n_sequence(void* vec, void* init, void* step) {
    bool ok;
    if (!init) ok = TRTC_Sequence(V(vec));
    else if (!step) ok = TRTC_Sequence(V(vec), D(init));
    else ok = TRTC_Sequence(V(vec), D(init), D(step));
    return ok ? 0 : -1;
}
TRTC_EXPORT int n_tabulate(void* vec, void* op) { return TRTC_Tabulate(V(vec), F(op)) ? 0 : -1; }
TRTC_EXPORT int n_transform(void* in, void* out, void* op) { return TRTC_Transform(V(in), V(out), F(op)) ? 0 : -1; }
TRTC_EXPORT int n_transform_binary(void* in1, void* in2, void* out, void* op) {
    return TRTC_Transform_Binary(V(in1), V(in2), V(out), F(op)) ? 0 : -1;
}
TRTC_EXPORT int n_transform_if(void* in, void* out, void* op, void* pred) {
    return TRTC_Transform_If(V(in), V(out), F(op), F(pred)) ? 0 : -1;
}
TRTC_EXPORT int n_transform_if_stencil(void* in, void* st, void* out, void* op, void* pred) {
    return TRTC_Transform_If_Stencil(V(in), V(st), V(out), F(op), F(pred)) ? 0 : -1;
}
TRTC_EXPORT int n_transform_binary_if_stencil(void* in1, void* in2, void* st, void* out, void* op, void* pred) {
    return TRTC_Transform_Binary_If_Stencil(V(in1), V(in2), V(st), V(out), F(op), F(pred)) ? 0 : -1;
}
// copying -- python/api_Copying.cpp
TRTC_EXPORT int n_gather(void* map, void* in, void* out) { return TRTC_Gather(V(map), V(in), V(out)) ? 0 : -1; }
TRTC_EXPORT int n_gather_if(void* map, void* st, void* in, void* out, void* pred) {
    return (pred ? TRTC_Gather_If(V(map), V(st), V(in), V(out), F(pred)) : TRTC_Gather_If(V(map), V(st), V(in), V(out)))
               ? 0 : -1;
}
TRTC_EXPORT int n_scatter(void* in, void* map, void* out) { return TRTC_Scatter(V(in), V(map), V(out)) ? 0 : -1; }
TRTC_EXPORT int n_scatter_if(void* in, void* map, void* st, void* out, void* pred) {
    return (pred ? TRTC_Scatter_If(V(in), V(map), V(st), V(out), F(pred))
                 : TRTC_Scatter_If(V(in), V(map), V(st), V(out))) ? 0 : -1;
}
TRTC_EXPORT int n_swap(void* vec1, void* vec2) { return TRTC_Swap(V(vec1), V(vec2)) ? 0 : -1; }
// reductions -- python/api_Reductions.cpp
TRTC_EXPORT unsigned long long n_count(void* vec, void* value) {
    size_t r = 0;
    return TRTC_Count(V(vec), D(value), r) ? (unsigned long long)r : ~0ull;
}
TRTC_EXPORT unsigned long long n_count_if(void* vec, void* pred) {
    size_t r = 0;
    return TRTC_Count_If(V(vec), F(pred), r) ? (unsigned long long)r : ~0ull;
}
TRTC_EXPORT int n_equal(void* vec1, void* vec2, void* pred) {
    bool r = false;
    const bool ok = pred ? TRTC_Equal(V(vec1), V(vec2), F(pred), r) : TRTC_Equal(V(vec1), V(vec2), r);
    return ok ? (r ? 1 : 0) : -1;
}
TRTC_EXPORT unsigned long long n_max_element(void* vec, void* comp) {
    size_t id = 0;
    const bool ok = comp ? TRTC_Max_Element(V(vec), F(comp), id) : TRTC_Max_Element(V(vec), id);
    return ok ? (unsigned long long)id : ~0ull;
}
TRTC_EXPORT int n_minmax_element(void* vec, void* comp, unsigned long long* ret) {
    size_t lo = 0, hi = 0;
    const bool ok = comp ? TRTC_MinMax_Element(V(vec), F(comp), lo, hi) : TRTC_MinMax_Element(V(vec), lo, hi);
    if (!ok) return -1;
    ret[0] = lo;
    ret[1] = hi;
    return 0;
}
TRTC_EXPORT void* n_inner_product(void* vec1, void* vec2, void* init, void* op1, void* op2) {
    ViewBuf ret;
    const bool ok = (op1 && op2) ? TRTC_Inner_Product(V(vec1), V(vec2), D(init), ret, F(op1), F(op2))
                                 : TRTC_Inner_Product(V(vec1), V(vec2), D(init), ret);
    return ok ? dv_from_viewbuf(ret, D(init).name_view_cls().c_str()) : nullptr;
}
#define TRTC_BOOL_EXPORT(name, fn)                        \
    TRTC_EXPORT int name(void* vec, void* pred) {         \
        bool r = false;                                   \
        return fn(V(vec), F(pred), r) ? (r ? 1 : 0) : -1; \
    }
TRTC_BOOL_EXPORT(n_all_of, TRTC_All_Of)
TRTC_BOOL_EXPORT(n_any_of, TRTC_Any_Of)
TRTC_BOOL_EXPORT(n_none_of, TRTC_None_Of)
TRTC_BOOL_EXPORT(n_is_partitioned, TRTC_Is_Partitioned)
#undef TRTC_BOOL_EXPORT
TRTC_EXPORT int n_is_sorted(void* vec, void* comp) {
    bool r = false;
    const bool ok = comp ? TRTC_Is_Sorted(V(vec), F(comp), r) : TRTC_Is_Sorted(V(vec), r);
    return ok ? (r ? 1 : 0) : -1;
}
// searching -- python/api_Searching.cpp: a missing index reads as the size
static long long index_or_size(bool ok, size_t r, size_t size) {
    if (!ok) return -1;
    return r == (size_t)(-1) ? (long long)size : (long long)r;
}
TRTC_EXPORT long long n_find(void* vec, void* value) {
    size_t r = 0;
    const bool ok = TRTC_Find(V(vec), D(value), r);
    return index_or_size(ok, r, V(vec).size());
}
TRTC_EXPORT long long n_find_if(void* vec, void* pred) {
    size_t r = 0;
    const bool ok = TRTC_Find_If(V(vec), F(pred), r);
    return index_or_size(ok, r, V(vec).size());
}
TRTC_EXPORT long long n_find_if_not(void* vec, void* pred) {
    size_t r = 0;
    const bool ok = TRTC_Find_If_Not(V(vec), F(pred), r);
    return index_or_size(ok, r, V(vec).size());
}
TRTC_EXPORT long long n_mismatch(void* vec1, void* vec2, void* pred) {
    size_t r = 0;
    const bool ok = pred ? TRTC_Mismatch(V(vec1), V(vec2), F(pred), r) : TRTC_Mismatch(V(vec1), V(vec2), r);
    return index_or_size(ok, r, V(vec1).size());
}
TRTC_EXPORT unsigned long long n_partition_point(void* vec, void* pred) {
    size_t r = 0;
    if (!TRTC_Partition_Point(V(vec), F(pred), r)) return ~0ull;
    return r == (size_t)(-1) ? (unsigned long long)V(vec).size() : (unsigned long long)r;
}
TRTC_EXPORT unsigned long long n_is_sorted_until(void* vec, void* comp) {
    size_t r = 0;
    const bool ok = comp ? TRTC_Is_Sorted_Until(V(vec), F(comp), r) : TRTC_Is_Sorted_Until(V(vec), r);
    return ok ? (unsigned long long)r : ~0ull;
}
// merging -- python/api_Merging.cpp
TRTC_EXPORT int n_merge(void* vec1, void* vec2, void* out, void* comp) {
    return (comp ? TRTC_Merge(V(vec1), V(vec2), V(out), F(comp)) : TRTC_Merge(V(vec1), V(vec2), V(out))) ? 0 : -1;
}
TRTC_EXPORT int n_merge_by_key(void* k1, void* k2, void* v1, void* v2, void* ko, void* vo, void* comp) {
    return (comp ? TRTC_Merge_By_Key(V(k1), V(k2), V(v1), V(v2), V(ko), V(vo), F(comp))
                 : TRTC_Merge_By_Key(V(k1), V(k2), V(v1), V(v2), V(ko), V(vo))) ? 0 : -1;
}
