// trtc_objects.cpp -- device-viewable object model (DeviceViewable.h:9-157, DVVector.h:8-60,
// functor.h:6-17, fake_vectors/*).  Each object knows the name, byte size and alignment of
// its device view struct; composite views (ranges, counters, functors with captured
// objects) are laid out on the host with C++ struct rules, so no reflection compile is needed
// for them.  Only user-named types of unknown layout go through the NVRTC probe.
#include "thrustrtc_cpp.h"
#include "trtc_jit.h"
#include "trtc_runtime.h"

#include <cstdio>

using namespace trtc_host;

static Layout layout_or_die(const std::string& name, size_t fallback_size) {
    Layout l;
    if (layout_of(name, l)) return l;
    // unknown layout without a GPU to probe: assume the natural alignment of its size
    l.size = fallback_size ? fallback_size : 1;
    l.align = 1;
    while (l.align < 16 && l.size % (l.align * 2) == 0) l.align *= 2;
    return l;
}

static void set_view_layout(DeviceViewable* dv, const std::string& name, const Layout& l, size_t* size_out,
                            size_t* align_out) {
    layout_register(name, l);
    *size_out = l.size;
    *align_out = l.align;
    (void)dv;
}

// ------------------------------------------------------------------ scalars
SomeDeviceViewable::SomeDeviceViewable(const char* name_view_cls, const void* data_view, size_t size_view) {
    m_name_view_cls = name_view_cls;
    m_view_buf.resize(size_view);
    memcpy(m_view_buf.data(), data_view, size_view);
    Layout l = layout_or_die(m_name_view_cls, size_view);
    m_view_size = size_view;
    m_view_align = l.align;
}

DVComplex64::DVComplex64(float real, float imag) {
    m_name_view_cls = "cuFloatComplex";
    m_v[0] = real;
    m_v[1] = imag;
    m_view_size = 8;
    m_view_align = 8;
}
ViewBuf DVComplex64::view() const {
    ViewBuf b(8);
    memcpy(b.data(), m_v, 8);
    return b;
}
DVComplex128::DVComplex128(double real, double imag) {
    m_name_view_cls = "cuDoubleComplex";
    m_v[0] = real;
    m_v[1] = imag;
    m_view_size = 16;
    m_view_align = 16;
}
ViewBuf DVComplex128::view() const {
    ViewBuf b(16);
    memcpy(b.data(), m_v, 16);
    return b;
}

DeviceViewable* dv_from_viewbuf(const ViewBuf& buf, const char* type) {
    const std::string t = type;
    if (t == "int8_t") return new DVInt8(*(const int8_t*)buf.data());
    if (t == "uint8_t") return new DVUInt8(*(const uint8_t*)buf.data());
    if (t == "int16_t") return new DVInt16(*(const int16_t*)buf.data());
    if (t == "uint16_t") return new DVUInt16(*(const uint16_t*)buf.data());
    if (t == "int32_t") return new DVInt32(*(const int32_t*)buf.data());
    if (t == "uint32_t") return new DVUInt32(*(const uint32_t*)buf.data());
    if (t == "int64_t") return new DVInt64(*(const int64_t*)buf.data());
    if (t == "uint64_t") return new DVUInt64(*(const uint64_t*)buf.data());
    if (t == "float") return new DVFloat(*(const float*)buf.data());
    if (t == "double") return new DVDouble(*(const double*)buf.data());
    if (t == "bool") return new DVBool(*(const bool*)buf.data());
    return new SomeDeviceViewable(type, buf.data(), buf.size());
}

// ------------------------------------------------------------------ vectors
DVVectorLike::DVVectorLike(const char* elem_cls, const char* ref_type, size_t size) {
    m_elem_cls = elem_cls;
    m_ref_type = ref_type;
    m_elem_size = layout_or_die(m_elem_cls, 0).size;
    m_size = size;
}

static void vector_view_layout(const std::string& elem, std::string& name, size_t& vs, size_t& va) {
    name = "VectorView<" + elem + ">";
    layout_register(name, Layout{16, 8});
    vs = 16;
    va = 8;
}

DVVector::DVVector(const char* elem_cls, size_t size, void* hdata)
    : DVVectorLike(elem_cls, (std::string(elem_cls) + "&").c_str(), size) {
    vector_view_layout(m_elem_cls, m_name_view_cls, m_view_size, m_view_align);
    if (!ensure_device()) return;
    const size_t bytes = m_elem_size * m_size;
    if (bytes == 0) return;
    if (!(m_data = vector_alloc(bytes))) return;
    if (hdata) TRTC_CUDA(cudaMemcpy(m_data, hdata, bytes, cudaMemcpyHostToDevice));
    else TRTC_CUDA(cudaMemset(m_data, 0, bytes));
}

DVVector::~DVVector() {
    vector_free(m_data);
}

void DVVector::to_host(void* hdata, size_t begin, size_t end) const {
    if (end == (size_t)(-1) || end > m_size) end = m_size;
    if (begin >= end || !m_data) return;
    TRTC_CUDA(cudaMemcpy(hdata, (char*)m_data + begin * m_elem_size, (end - begin) * m_elem_size, cudaMemcpyDeviceToHost));
}

ViewBuf DVVector::view() const {
    ViewBuf b(16);
    void* p = m_data;
    unsigned long long s = m_size;
    memcpy(b.data(), &p, 8);
    memcpy(b.data() + 8, &s, 8);
    return b;
}

DVVectorAdaptor::DVVectorAdaptor(const char* elem_cls, size_t size, void* ddata)
    : DVVectorLike(elem_cls, (std::string(elem_cls) + "&").c_str(), size), m_data(ddata) {
    vector_view_layout(m_elem_cls, m_name_view_cls, m_view_size, m_view_align);
}
DVVectorAdaptor::DVVectorAdaptor(const DVVector& vec, size_t begin, size_t end)
    : DVVectorLike(vec.name_elem_cls().c_str(), vec.name_ref_type().c_str(),
                   (end == (size_t)(-1) ? vec.size() : end) - begin) {
    m_data = (char*)vec.data() + begin * vec.elem_size();
    vector_view_layout(m_elem_cls, m_name_view_cls, m_view_size, m_view_align);
}
DVVectorAdaptor::DVVectorAdaptor(const DVVectorAdaptor& vec, size_t begin, size_t end)
    : DVVectorLike(vec.name_elem_cls().c_str(), vec.name_ref_type().c_str(),
                   (end == (size_t)(-1) ? vec.size() : end) - begin) {
    m_data = (char*)vec.data() + begin * vec.elem_size();
    vector_view_layout(m_elem_cls, m_name_view_cls, m_view_size, m_view_align);
}
ViewBuf DVVectorAdaptor::view() const {
    ViewBuf b(16);
    void* p = m_data;
    unsigned long long s = m_size;
    memcpy(b.data(), &p, 8);
    memcpy(b.data() + 8, &s, 8);
    return b;
}

// RangeView<V> { V _view_vec_value; size_t _begin; size_t _end; }  (fake_vectors/DVRange.cpp)
DVRange::DVRange(const DVVectorLike& vec_value, size_t begin, size_t end)
    : DVVectorLike(vec_value.name_elem_cls().c_str(), vec_value.name_ref_type().c_str(),
                   (end == (size_t)(-1) ? vec_value.size() : end) - begin) {
    if (end == (size_t)(-1)) end = vec_value.size();
    m_readable = vec_value.is_readable();
    m_writable = vec_value.is_writable();
    m_view_value = vec_value.view();
    m_begin = begin;
    m_end = end;
    void* base = vec_value.contiguous_data();
    m_base_data = base ? (char*)base + begin * vec_value.elem_size() : nullptr;
    m_name_view_cls = "RangeView<" + vec_value.name_view_cls() + ">";
    StructLayout sl;
    m_off[0] = sl.add(Layout{vec_value.view_size(), vec_value.view_align()});
    m_off[1] = sl.add(Layout{8, 8});
    m_off[2] = sl.add(Layout{8, 8});
    set_view_layout(this, m_name_view_cls, sl.finish(), &m_view_size, &m_view_align);
}
ViewBuf DVRange::view() const {
    ViewBuf b(m_view_size, 0);
    memcpy(b.data() + m_off[0], m_view_value.data(), m_view_value.size());
    memcpy(b.data() + m_off[1], &m_begin, 8);
    memcpy(b.data() + m_off[2], &m_end, 8);
    return b;
}
void* DVRange::contiguous_data() const { return m_base_data; }

// ConstantView<T> { size_t _size; T _value; }
DVConstant::DVConstant(const DeviceViewable& dvobj, size_t size)
    : DVVectorLike(dvobj.name_view_cls().c_str(), ("const " + dvobj.name_view_cls() + "&").c_str(), size) {
    m_value = dvobj.view();
    m_name_view_cls = "ConstantView<" + m_elem_cls + ">";
    StructLayout sl;
    m_off[0] = sl.add(Layout{8, 8});
    m_off[1] = sl.add(Layout{dvobj.view_size(), dvobj.view_align()});
    set_view_layout(this, m_name_view_cls, sl.finish(), &m_view_size, &m_view_align);
}
ViewBuf DVConstant::view() const {
    ViewBuf b(m_view_size, 0);
    memcpy(b.data() + m_off[0], &m_size, 8);
    memcpy(b.data() + m_off[1], m_value.data(), m_value.size());
    return b;
}

// CounterView<T> { size_t _size; T _value_init; }
DVCounter::DVCounter(const DeviceViewable& dvobj_init, size_t size)
    : DVVectorLike(dvobj_init.name_view_cls().c_str(), dvobj_init.name_view_cls().c_str(), size) {
    m_value_init = dvobj_init.view();
    m_name_view_cls = "CounterView<" + m_elem_cls + ">";
    StructLayout sl;
    m_off[0] = sl.add(Layout{8, 8});
    m_off[1] = sl.add(Layout{dvobj_init.view_size(), dvobj_init.view_align()});
    set_view_layout(this, m_name_view_cls, sl.finish(), &m_view_size, &m_view_align);
}
ViewBuf DVCounter::view() const {
    ViewBuf b(m_view_size, 0);
    memcpy(b.data() + m_off[0], &m_size, 8);
    memcpy(b.data() + m_off[1], m_value_init.data(), m_value_init.size());
    return b;
}

// DiscardView<T> { size_t _size; _Sink<T> _sink; }
DVDiscard::DVDiscard(const char* elem_cls, size_t size)
    : DVVectorLike(elem_cls, ("_Sink<" + std::string(elem_cls) + ">&").c_str(), size) {
    m_name_view_cls = "DiscardView<" + m_elem_cls + ">";
    set_view_layout(this, m_name_view_cls, Layout{16, 8}, &m_view_size, &m_view_align);
}
ViewBuf DVDiscard::view() const {
    ViewBuf b(16, 0);
    memcpy(b.data(), &m_size, 8);
    return b;
}

// ReverseView<V> { V _view_vec_value; }
DVReverse::DVReverse(const DVVectorLike& vec_value)
    : DVVectorLike(vec_value.name_elem_cls().c_str(), vec_value.name_ref_type().c_str(), vec_value.size()) {
    m_readable = vec_value.is_readable();
    m_writable = vec_value.is_writable();
    m_view_value = vec_value.view();
    m_name_view_cls = "ReverseView<" + vec_value.name_view_cls() + ">";
    set_view_layout(this, m_name_view_cls, Layout{vec_value.view_size(), vec_value.view_align()}, &m_view_size,
                    &m_view_align);
}

// PermutationView<V, I> { V _view_vec_value; I _view_vec_index; }
DVPermutation::DVPermutation(const DVVectorLike& vec_value, const DVVectorLike& vec_index)
    : DVVectorLike(vec_value.name_elem_cls().c_str(), vec_value.name_ref_type().c_str(), vec_index.size()) {
    m_readable = vec_value.is_readable();
    m_writable = vec_value.is_writable();
    m_view_value = vec_value.view();
    m_view_index = vec_index.view();
    m_name_view_cls = "PermutationView<" + vec_value.name_view_cls() + ", " + vec_index.name_view_cls() + ">";
    StructLayout sl;
    m_off[0] = sl.add(Layout{vec_value.view_size(), vec_value.view_align()});
    m_off[1] = sl.add(Layout{vec_index.view_size(), vec_index.view_align()});
    set_view_layout(this, m_name_view_cls, sl.finish(), &m_view_size, &m_view_align);
}
ViewBuf DVPermutation::view() const {
    ViewBuf b(m_view_size, 0);
    memcpy(b.data() + m_off[0], m_view_value.data(), m_view_value.size());
    memcpy(b.data() + m_off[1], m_view_index.data(), m_view_index.size());
    return b;
}

// TransformView<T, VIN, OP> { VIN _view_vec_in; OP _view_op; }
DVTransform::DVTransform(const DVVectorLike& vec_in, const char* elem_cls, const Functor& op)
    : DVVectorLike(elem_cls, elem_cls, vec_in.size()) {
    m_view_in = vec_in.view();
    m_view_op = op.view();
    m_name_view_cls = "TransformView<" + m_elem_cls + ", " + vec_in.name_view_cls() + ", " + op.name_view_cls() + ">";
    StructLayout sl;
    m_off[0] = sl.add(Layout{vec_in.view_size(), vec_in.view_align()});
    m_off[1] = sl.add(Layout{op.view_size(), op.view_align()});
    set_view_layout(this, m_name_view_cls, sl.finish(), &m_view_size, &m_view_align);
}
ViewBuf DVTransform::view() const {
    ViewBuf b(m_view_size, 0);
    memcpy(b.data() + m_off[0], m_view_in.data(), m_view_in.size());
    memcpy(b.data() + m_off[1], m_view_op.data(), m_view_op.size());
    return b;
}

// ------------------------------------------------------------------ Functor
// User functor: a struct with the captured objects' views as members and a templated
// device operator() whose body is the user's code (functor.cpp:4-45 builds the same shape).
Functor::Functor(const std::vector<CapturedDeviceViewable>& arg_map, const std::vector<const char*>& functor_params,
                 const char* code_body) {
    std::string body;
    StructLayout sl;
    m_view_args.resize(arg_map.size());
    for (size_t i = 0; i < arg_map.size(); i++) {
        body += std::string("    ") + arg_map[i].obj->name_view_cls() + " " + arg_map[i].obj_name + ";\n";
        m_view_args[i] = arg_map[i].obj->view();
        sl.add(Layout{arg_map[i].obj->view_size(), arg_map[i].obj->view_align()});
    }
    if (!functor_params.empty()) {
        body += "    template<";
        for (size_t i = 0; i < functor_params.size(); i++) {
            char tn[32];
            snprintf(tn, sizeof(tn), "class _T%d", (int)i);
            body += tn;
            if (i + 1 < functor_params.size()) body += ",";
        }
        body += ">\n";
    }
    body += "    __device__ inline auto operator()(";
    for (size_t i = 0; i < functor_params.size(); i++) {
        char p[96];
        snprintf(p, sizeof(p), "const _T%d& %s", (int)i, functor_params[i]);
        body += p;
        if (i + 1 < functor_params.size()) body += ",";
    }
    body += ")\n    {\n";
    body += code_body;
    body += "\n    }\n";
    m_name_view_cls = jit_add_struct(body);
    m_offsets = sl.offsets;
    const Layout l = sl.finish();
    m_offsets.push_back(l.size);
    m_view_size = l.size;
    m_view_align = l.align;
    layout_register(m_name_view_cls, l);
}

Functor::Functor(const char* name_built_in_view_cls) {
    m_name_view_cls = name_built_in_view_cls;
    m_built_in = true;
    m_offsets.assign(1, 1);
    m_view_size = 1;
    m_view_align = 1;
    layout_register(m_name_view_cls, Layout{1, 1});
}

ViewBuf Functor::view() const {
    ViewBuf ret(m_offsets.back(), 0);
    for (size_t i = 0; i < m_view_args.size(); i++)
        memcpy(ret.data() + m_offsets[i], m_view_args[i].data(), m_view_args[i].size());
    return ret;
}

// ------------------------------------------------------------------ DVTuple
// struct { V0 name0; V1 name1; ... } of the objects' views (DVTuple.cpp:4-19)
DVTuple::DVTuple(const std::vector<CapturedDeviceViewable>& elem_map) {
    std::string body;
    StructLayout sl;
    m_view_elems.resize(elem_map.size());
    for (size_t i = 0; i < elem_map.size(); i++) {
        body += std::string("    ") + elem_map[i].obj->name_view_cls() + " " + elem_map[i].obj_name + ";\n";
        m_view_elems[i] = elem_map[i].obj->view();
        sl.add(Layout{elem_map[i].obj->view_size(), elem_map[i].obj->view_align()});
    }
    m_name_view_cls = jit_add_struct(body);
    m_offsets = sl.offsets;
    const Layout l = sl.finish();
    m_offsets.push_back(l.size);
    m_view_size = l.size;
    m_view_align = l.align;
    layout_register(m_name_view_cls, l);
}
ViewBuf DVTuple::view() const {
    ViewBuf ret(m_offsets.back(), 0);
    for (size_t i = 0; i < m_view_elems.size(); i++)
        memcpy(ret.data() + m_offsets[i], m_view_elems[i].data(), m_view_elems[i].size());
    return ret;
}

// ------------------------------------------------------------------ DVZipped
// The element struct has the same body text as a DVTuple of scalars with the same member
// names and types, so both name the same struct (a DVConstant of such a tuple assigns to a
// zipped vector, as in the reference).
static std::string zipped_elem_struct(const std::vector<DVVectorLike*>& vecs, const std::vector<const char*>& names) {
    std::string body;
    StructLayout sl;
    for (size_t i = 0; i < vecs.size(); i++) {
        body += std::string("    ") + vecs[i]->name_elem_cls() + " " + names[i] + ";\n";
        Layout l;
        if (!layout_of(vecs[i]->name_elem_cls(), l)) l = Layout{vecs[i]->elem_size(), vecs[i]->elem_size()};
        sl.add(l);
    }
    const std::string name = jit_add_struct(body);
    layout_register(name, sl.finish());
    return name;
}

// reference struct: members are the vectors' reference types; converts to the element
// struct when all are readable, assigns from it when all are writable
static std::string zipped_ref_struct(const std::vector<DVVectorLike*>& vecs, const std::vector<const char*>& names,
                                     const std::string& elem_cls, bool& readable, bool& writable) {
    readable = writable = true;
    for (auto* v : vecs) {
        readable = readable && v->is_readable();
        writable = writable && v->is_writable();
    }
    std::string body;
    for (size_t i = 0; i < vecs.size(); i++)
        body += std::string("    ") + vecs[i]->name_ref_type() + " " + names[i] + ";\n";
    if (readable) {
        body += "    __device__ operator " + elem_cls + "()\n    {\n        return {";
        for (size_t i = 0; i < vecs.size(); i++) body += std::string(names[i]) + (i + 1 < vecs.size() ? ", " : "");
        body += "};\n    }\n";
    }
    if (writable) {
        body += "    __device__ CurType& operator = (const " + elem_cls + "& in)\n    {\n";
        for (size_t i = 0; i < vecs.size(); i++)
            body += std::string("        this->") + names[i] + " = in." + names[i] + ";\n";
        body += "        return *this;\n    }\n";
    }
    return jit_add_struct(body);
}

static std::string zipped_elem_cls_for(const std::vector<DVVectorLike*>& vecs, const std::vector<const char*>& names) {
    return vecs.empty() ? std::string("char") : zipped_elem_struct(vecs, names);
}

DVZipped::DVZipped(const std::vector<DVVectorLike*>& vecs, const std::vector<const char*>& elem_names)
    : DVVectorLike(zipped_elem_cls_for(vecs, elem_names).c_str(), "char", vecs.empty() ? 0 : vecs[0]->size()) {
    m_ref_type = zipped_ref_struct(vecs, elem_names, m_elem_cls, m_readable, m_writable);
    std::string body = "    typedef " + m_elem_cls + " value_t;\n    typedef " + m_ref_type + " ref_t;\n";
    StructLayout sl;
    m_view_elems.resize(vecs.size());
    for (size_t i = 0; i < vecs.size(); i++) {
        body += std::string("    ") + vecs[i]->name_view_cls() + " " + elem_names[i] + ";\n";
        m_view_elems[i] = vecs[i]->view();
        sl.add(Layout{vecs[i]->view_size(), vecs[i]->view_align()});
    }
    body += std::string("    __device__ size_t size() const\n    {\n        return ") + elem_names[0] +
            ".size();\n    }\n";
    body += "    __device__ ref_t operator [](size_t idx)\n    {\n        return {";
    for (size_t i = 0; i < vecs.size(); i++)
        body += std::string(elem_names[i]) + "[idx]" + (i + 1 < vecs.size() ? ", " : "");
    body += "};\n    }\n";
    m_name_view_cls = jit_add_struct(body);
    m_offsets = sl.offsets;
    const Layout l = sl.finish();
    m_offsets.push_back(l.size);
    m_view_size = l.size;
    m_view_align = l.align;
    layout_register(m_name_view_cls, l);
}
ViewBuf DVZipped::view() const {
    ViewBuf ret(m_offsets.back(), 0);
    for (size_t i = 0; i < m_view_elems.size(); i++)
        memcpy(ret.data() + m_offsets[i], m_view_elems[i].data(), m_view_elems[i].size());
    return ret;
}

// ------------------------------------------------------------------ DVCustomVector
// functor struct { captured views; ref_t operator()(size_t idx) { code } } wrapped in a
// view struct { size_t _size; F _op; size(); operator[](idx) -> _op(idx) }
// (fake_vectors/DVCustomVector.cpp:5-38)
DVCustomVector::DVCustomVector(const std::vector<CapturedDeviceViewable>& arg_map, const char* name_idx,
                               const char* code_body, const char* elem_cls, size_t size, bool read_only)
    : DVVectorLike(elem_cls, read_only ? elem_cls : (std::string(elem_cls) + "&").c_str(), size),
      m_size_val(size), m_read_only(read_only) {
    std::string fbody;
    StructLayout fl;
    m_view_args.resize(arg_map.size());
    for (size_t i = 0; i < arg_map.size(); i++) {
        fbody += std::string("    ") + arg_map[i].obj->name_view_cls() + " " + arg_map[i].obj_name + ";\n";
        m_view_args[i] = arg_map[i].obj->view();
        fl.add(Layout{arg_map[i].obj->view_size(), arg_map[i].obj->view_align()});
    }
    fbody += "    __device__ inline " + m_ref_type + " operator()(size_t " + name_idx + ")\n    {\n";
    fbody += code_body;
    fbody += "    }\n";
    const std::string fname = jit_add_struct(fbody);
    m_arg_offsets = fl.offsets;
    const Layout fla = fl.finish();
    m_arg_offsets.push_back(fla.size);
    layout_register(fname, fla);
    std::string body = "    typedef " + m_elem_cls + " value_t;\n    typedef " + m_ref_type + " ref_t;\n";
    body += "    size_t _size;\n    " + fname + " _op;\n";
    body += "    __device__ inline size_t size() const\n    {\n        return _size;\n    }\n";
    body += "    __device__ ref_t operator [](size_t idx)\n    {\n        return _op(idx);\n    }\n";
    m_name_view_cls = jit_add_struct(body);
    StructLayout sl;
    sl.add(Layout{8, 8});
    m_op_offset = sl.add(fla);
    m_op_size = fla.size;
    const Layout l = sl.finish();
    m_view_size = l.size;
    m_view_align = l.align;
    layout_register(m_name_view_cls, l);
}
ViewBuf DVCustomVector::view() const {
    ViewBuf ret(m_view_size, 0);
    const unsigned long long sz = m_size_val;
    memcpy(ret.data(), &sz, 8);
    for (size_t i = 0; i < m_view_args.size(); i++)
        memcpy(ret.data() + m_op_offset + m_arg_offsets[i], m_view_args[i].data(), m_view_args[i].size());
    return ret;
}
