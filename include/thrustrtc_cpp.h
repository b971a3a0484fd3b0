// thrustrtc_cpp.h -- C++ API of thrustrtc_b200 (the interface the reference's JNI and
// C++/CLI shims call: java/Sorting.cpp:4-30, CSharp/ThrustRTCLR/Sorting.cpp:13-39).
//
// Class names, constructor/method signatures and function signatures follow the
// reference's public headers so that a shim compiled against them compiles against this one:
//   DeviceViewable / ViewBuf / CapturedDeviceViewable / DV* scalars  <- DeviceViewable.h:9-157
//   DVVectorLike / DVVector / DVVectorAdaptor                        <- DVVector.h:8-60
//   Functor                                                          <- functor.h:6-17
//   DVRange, DVConstant, DVCounter, DVDiscard, DVReverse,
//   DVPermutation, DVTransform                                       <- fake_vectors/*.h
//   TRTC_Try_Init, TRTC_Size_Of, TRTC_Add_*, TRTC_Wait,
//   TRTC_Kernel, TRTC_For                                            <- TRTCContext.h:13-71
//   TRTC_Sort*, TRTC_*Scan*, TRTC_Reduce*, TRTC_Transform_Reduce,
//   TRTC_Min_Element, TRTC_Copy*, TRTC_Remove*, TRTC_Unique*,
//   TRTC_Partition*                                                  <- sort.h, scan.h, transform_scan.h,
//                                                                       reduce.h, transform_reduce.h,
//                                                                       extrema.h, copy.h, remove.h,
//                                                                       unique.h, partition.h
// The implementation behind them is new: nvcc-built sm_100a kernels for built-in types and
// operators on contiguous vectors, and NVRTC (-arch=sm_100a) instantiations of the same
// kernel templates for user Functors and non-contiguous views.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#ifndef THRUST_RTC_API
#define THRUST_RTC_API __attribute__((visibility("default")))
#endif

typedef std::vector<char> ViewBuf;

struct dim_type {
    unsigned int x, y, z;
};

// ----------------------------------------------------------------- device-viewable objects
class THRUST_RTC_API DeviceViewable {
public:
    DeviceViewable() {}
    virtual ~DeviceViewable() {}
    virtual ViewBuf view() const = 0;
    const std::string& name_view_cls() const { return m_name_view_cls; }
    // byte size / alignment of the device view struct (thrustrtc_b200 addition)
    size_t view_size() const { return m_view_size; }
    size_t view_align() const { return m_view_align; }

protected:
    std::string m_name_view_cls;
    size_t m_view_size = 1;
    size_t m_view_align = 1;
};

struct CapturedDeviceViewable {
    const char* obj_name;
    const DeviceViewable* obj;
};

class THRUST_RTC_API SomeDeviceViewable : public DeviceViewable {
public:
    SomeDeviceViewable(const char* name_view_cls, const void* data_view = "", size_t size_view = 1);
    virtual ViewBuf view() const { return m_view_buf; }

private:
    ViewBuf m_view_buf;
};

#define TRTC_DECLARE_DV_BASIC(clsname, type) \
    class THRUST_RTC_API clsname : public SomeDeviceViewable { \
    public: \
        clsname(type in) : SomeDeviceViewable(#type, &in, sizeof(type)) {} \
    };

TRTC_DECLARE_DV_BASIC(DVChar, char)
TRTC_DECLARE_DV_BASIC(DVSChar, signed char)
TRTC_DECLARE_DV_BASIC(DVUChar, unsigned char)
TRTC_DECLARE_DV_BASIC(DVShort, short)
TRTC_DECLARE_DV_BASIC(DVUShort, unsigned short)
TRTC_DECLARE_DV_BASIC(DVInt, int)
TRTC_DECLARE_DV_BASIC(DVUInt, unsigned int)
TRTC_DECLARE_DV_BASIC(DVLong, long)
TRTC_DECLARE_DV_BASIC(DVULong, unsigned long)
TRTC_DECLARE_DV_BASIC(DVLongLong, long long)
TRTC_DECLARE_DV_BASIC(DVULongLong, unsigned long long)
TRTC_DECLARE_DV_BASIC(DVFloat, float)
TRTC_DECLARE_DV_BASIC(DVDouble, double)
TRTC_DECLARE_DV_BASIC(DVBool, bool)
TRTC_DECLARE_DV_BASIC(DVInt8, int8_t)
TRTC_DECLARE_DV_BASIC(DVUInt8, uint8_t)
TRTC_DECLARE_DV_BASIC(DVInt16, int16_t)
TRTC_DECLARE_DV_BASIC(DVUInt16, uint16_t)
TRTC_DECLARE_DV_BASIC(DVInt32, int32_t)
TRTC_DECLARE_DV_BASIC(DVUInt32, uint32_t)
TRTC_DECLARE_DV_BASIC(DVInt64, int64_t)
TRTC_DECLARE_DV_BASIC(DVUInt64, uint64_t)
TRTC_DECLARE_DV_BASIC(DVSizeT, size_t)

class THRUST_RTC_API DVComplex64 : public DeviceViewable {
public:
    DVComplex64(float real, float imag);
    virtual ViewBuf view() const;
    float real() const { return m_v[0]; }
    float imag() const { return m_v[1]; }

private:
    float m_v[2];
};

class THRUST_RTC_API DVComplex128 : public DeviceViewable {
public:
    DVComplex128(double real, double imag);
    virtual ViewBuf view() const;
    double real() const { return m_v[0]; }
    double imag() const { return m_v[1]; }

private:
    double m_v[2];
};

// new heap object holding a reduction result of the named type (DeviceViewable.h:130-157)
THRUST_RTC_API DeviceViewable* dv_from_viewbuf(const ViewBuf& buf, const char* type);

class THRUST_RTC_API DVVectorLike : public DeviceViewable {
public:
    const std::string& name_elem_cls() const { return m_elem_cls; }
    const std::string& name_ref_type() const { return m_ref_type; }
    size_t elem_size() const { return m_elem_size; }
    size_t size() const { return m_size; }

    DVVectorLike(const char* elem_cls, const char* ref_type, size_t size);
    virtual ~DVVectorLike() {}
    virtual bool is_readable() const { return true; }
    virtual bool is_writable() const { return false; }
    // thrustrtc_b200 addition: device address of element 0 when the view is a plain array
    // (DVVector, DVVectorAdaptor); nullptr for computed views.
    virtual void* contiguous_data() const { return nullptr; }

protected:
    std::string m_elem_cls;
    std::string m_ref_type;
    size_t m_elem_size;
    size_t m_size;
};

class THRUST_RTC_API DVVector : public DVVectorLike {
public:
    void* data() const { return m_data; }
    DVVector(const char* elem_cls, size_t size, void* hdata = nullptr);
    ~DVVector();
    virtual bool is_writable() const { return true; }
    virtual void* contiguous_data() const { return m_data; }
    void to_host(void* hdata, size_t begin = 0, size_t end = (size_t)(-1)) const;
    virtual ViewBuf view() const;

private:
    void* m_data = nullptr;
};

class THRUST_RTC_API DVVectorAdaptor : public DVVectorLike {
public:
    void* data() const { return m_data; }
    DVVectorAdaptor(const char* elem_cls, size_t size, void* ddata);
    DVVectorAdaptor(const DVVector& vec, size_t begin = 0, size_t end = (size_t)(-1));
    DVVectorAdaptor(const DVVectorAdaptor& vec, size_t begin = 0, size_t end = (size_t)(-1));
    virtual bool is_writable() const { return true; }
    virtual void* contiguous_data() const { return m_data; }
    virtual ViewBuf view() const;

private:
    void* m_data;
};

class THRUST_RTC_API DVRange : public DVVectorLike {
public:
    DVRange(const DVVectorLike& vec_value, size_t begin = 0, size_t end = (size_t)(-1));
    virtual ViewBuf view() const;
    virtual bool is_readable() const { return m_readable; }
    virtual bool is_writable() const { return m_writable; }
    virtual void* contiguous_data() const;

private:
    bool m_readable, m_writable;
    ViewBuf m_view_value;
    size_t m_begin, m_end;
    size_t m_off[3];
    void* m_base_data;
};

class THRUST_RTC_API DVConstant : public DVVectorLike {
public:
    DVConstant(const DeviceViewable& dvobj, size_t size = (size_t)(-1));
    virtual ViewBuf view() const;

private:
    ViewBuf m_value;
    size_t m_off[2];
};

class THRUST_RTC_API DVCounter : public DVVectorLike {
public:
    DVCounter(const DeviceViewable& dvobj_init, size_t size = (size_t)(-1));
    virtual ViewBuf view() const;

private:
    ViewBuf m_value_init;
    size_t m_off[2];
};

class THRUST_RTC_API DVDiscard : public DVVectorLike {
public:
    DVDiscard(const char* elem_cls, size_t size = (size_t)(-1));
    virtual ViewBuf view() const;
    virtual bool is_readable() const { return false; }
    virtual bool is_writable() const { return true; }
};

class THRUST_RTC_API DVReverse : public DVVectorLike {
public:
    DVReverse(const DVVectorLike& vec_value);
    virtual ViewBuf view() const { return m_view_value; }
    virtual bool is_readable() const { return m_readable; }
    virtual bool is_writable() const { return m_writable; }

private:
    bool m_readable, m_writable;
    ViewBuf m_view_value;
};

class THRUST_RTC_API DVPermutation : public DVVectorLike {
public:
    DVPermutation(const DVVectorLike& vec_value, const DVVectorLike& vec_index);
    virtual ViewBuf view() const;
    virtual bool is_readable() const { return m_readable; }
    virtual bool is_writable() const { return m_writable; }

private:
    bool m_readable, m_writable;
    ViewBuf m_view_value, m_view_index;
    size_t m_off[2];
};

class THRUST_RTC_API Functor;

class THRUST_RTC_API DVTransform : public DVVectorLike {
public:
    DVTransform(const DVVectorLike& vec_in, const char* elem_cls, const Functor& op);
    virtual ViewBuf view() const;

private:
    ViewBuf m_view_in, m_view_op;
    size_t m_off[2];
};

// A struct of named device-viewable objects (DVTuple.h) -- its view struct has one member
// per object, in order.
class THRUST_RTC_API DVTuple : public DeviceViewable {
public:
    DVTuple(const std::vector<CapturedDeviceViewable>& elem_map);
    virtual ViewBuf view() const;

private:
    std::vector<ViewBuf> m_view_elems;
    std::vector<size_t> m_offsets;
};

// Vectors of equal length seen as one vector of structs (fake_vectors/DVZipped.h): element
// i is { vecs[0][i], vecs[1][i], ... } under the given member names; writable when all are.
class THRUST_RTC_API DVZipped : public DVVectorLike {
public:
    DVZipped(const std::vector<DVVectorLike*>& vecs, const std::vector<const char*>& elem_names);
    virtual ViewBuf view() const;
    virtual bool is_readable() const { return m_readable; }
    virtual bool is_writable() const { return m_writable; }

private:
    bool m_readable = true, m_writable = true;
    std::vector<ViewBuf> m_view_elems;
    std::vector<size_t> m_offsets;
};

// A vector whose element idx is computed by user code over captured objects
// (fake_vectors/DVCustomVector.h); read_only = false makes the code return a reference.
class THRUST_RTC_API DVCustomVector : public DVVectorLike {
public:
    DVCustomVector(const std::vector<CapturedDeviceViewable>& arg_map, const char* name_idx, const char* code_body,
                   const char* elem_cls, size_t size, bool read_only = true);
    virtual ViewBuf view() const;
    virtual bool is_writable() const { return !m_read_only; }

private:
    size_t m_size_val;
    bool m_read_only;
    std::vector<ViewBuf> m_view_args;
    std::vector<size_t> m_arg_offsets;
    size_t m_op_offset = 0, m_op_size = 0;
};

class THRUST_RTC_API Functor : public DeviceViewable {
public:
    Functor(const std::vector<CapturedDeviceViewable>& arg_map, const std::vector<const char*>& functor_params,
            const char* code_body);
    Functor(const char* name_built_in_view_cls);
    virtual ViewBuf view() const;
    bool is_built_in() const { return m_built_in; }

private:
    bool m_built_in = false;
    std::vector<ViewBuf> m_view_args;
    std::vector<size_t> m_offsets;
};

// ----------------------------------------------------------------- context / JIT
THRUST_RTC_API void set_libnvrtc_path(const char* path);
THRUST_RTC_API bool TRTC_Try_Init();
THRUST_RTC_API int TRTC_Get_PTX_Arch();
THRUST_RTC_API void TRTC_Set_Verbose(bool verbose = true);
THRUST_RTC_API void TRTC_Set_Kernel_Debug(bool kernel_debug = true);
THRUST_RTC_API size_t TRTC_Size_Of(const char* cls);
THRUST_RTC_API bool TRTC_Query_Struct(const char* name_struct, const std::vector<const char*>& name_members,
                                      size_t* offsets);
THRUST_RTC_API void TRTC_Add_Include_Dir(const char* path);
THRUST_RTC_API void TRTC_Add_Built_In_Header(const char* name, const char* content);
THRUST_RTC_API void TRTC_Add_Code_Block(const char* code);
THRUST_RTC_API void TRTC_Add_Inlcude_Filename(const char* fn);
THRUST_RTC_API void TRTC_Add_Constant_Object(const char* name, const DeviceViewable& obj);
THRUST_RTC_API std::string TRTC_Add_Struct(const char* struct_body);
THRUST_RTC_API void TRTC_Wait();

class THRUST_RTC_API TRTC_Kernel {
public:
    size_t num_params() const { return m_param_names.size(); }
    TRTC_Kernel(const std::vector<const char*>& param_names, const char* code_body);
    bool calc_optimal_block_size(const DeviceViewable** args, int& sizeBlock, unsigned sharedMemBytes = 0);
    bool calc_number_blocks(const DeviceViewable** args, int sizeBlock, int& numBlocks, unsigned sharedMemBytes = 0);
    bool launch(dim_type gridDim, dim_type blockDim, const DeviceViewable** args, unsigned sharedMemBytes = 0);

private:
    std::vector<std::string> m_param_names;
    std::string m_code_body;
};

class THRUST_RTC_API TRTC_For {
public:
    size_t num_params() const { return m_param_names.size(); }
    TRTC_For(const std::vector<const char*>& param_names, const char* name_iter, const char* code_body);
    bool launch(size_t begin, size_t end, const DeviceViewable** args);
    bool launch_n(size_t n, const DeviceViewable** args);

private:
    std::vector<std::string> m_param_names;
    std::string m_name_iter;
    std::string m_code_body;
};

// ----------------------------------------------------------------- hot-path algorithms
THRUST_RTC_API bool TRTC_Sort(DVVectorLike& vec);
THRUST_RTC_API bool TRTC_Sort(DVVectorLike& vec, const Functor& comp);
THRUST_RTC_API bool TRTC_Sort_By_Key(DVVectorLike& keys, DVVectorLike& values);
THRUST_RTC_API bool TRTC_Sort_By_Key(DVVectorLike& keys, DVVectorLike& values, const Functor& comp);

THRUST_RTC_API bool TRTC_Inclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Inclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& binary_op);
THRUST_RTC_API bool TRTC_Exclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Exclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out, const DeviceViewable& init);
THRUST_RTC_API bool TRTC_Exclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out, const DeviceViewable& init,
                                        const Functor& binary_op);
THRUST_RTC_API bool TRTC_Transform_Inclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out,
                                                  const Functor& unary_op, const Functor& binary_op);
THRUST_RTC_API bool TRTC_Transform_Exclusive_Scan(const DVVectorLike& vec_in, DVVectorLike& vec_out,
                                                  const Functor& unary_op, const DeviceViewable& init,
                                                  const Functor& binary_op);
THRUST_RTC_API bool TRTC_Inclusive_Scan_By_Key(const DVVectorLike& vec_key, const DVVectorLike& vec_value,
                                               DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Inclusive_Scan_By_Key(const DVVectorLike& vec_key, const DVVectorLike& vec_value,
                                               DVVectorLike& vec_out, const Functor& binary_pred);
THRUST_RTC_API bool TRTC_Inclusive_Scan_By_Key(const DVVectorLike& vec_key, const DVVectorLike& vec_value,
                                               DVVectorLike& vec_out, const Functor& binary_pred,
                                               const Functor& binary_op);
THRUST_RTC_API bool TRTC_Exclusive_Scan_By_Key(const DVVectorLike& vec_key, const DVVectorLike& vec_value,
                                               DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Exclusive_Scan_By_Key(const DVVectorLike& vec_key, const DVVectorLike& vec_value,
                                               DVVectorLike& vec_out, const DeviceViewable& init);
THRUST_RTC_API bool TRTC_Exclusive_Scan_By_Key(const DVVectorLike& vec_key, const DVVectorLike& vec_value,
                                               DVVectorLike& vec_out, const DeviceViewable& init,
                                               const Functor& binary_pred);
THRUST_RTC_API bool TRTC_Exclusive_Scan_By_Key(const DVVectorLike& vec_key, const DVVectorLike& vec_value,
                                               DVVectorLike& vec_out, const DeviceViewable& init,
                                               const Functor& binary_pred, const Functor& binary_op);

THRUST_RTC_API bool TRTC_Reduce(const DVVectorLike& vec, ViewBuf& ret);
THRUST_RTC_API bool TRTC_Reduce(const DVVectorLike& vec, const DeviceViewable& init, ViewBuf& ret);
THRUST_RTC_API bool TRTC_Reduce(const DVVectorLike& vec, const DeviceViewable& init, const Functor& binary_op,
                                ViewBuf& ret);
THRUST_RTC_API uint32_t TRTC_Reduce_By_Key(const DVVectorLike& key_in, const DVVectorLike& value_in,
                                           DVVectorLike& key_out, DVVectorLike& value_out);
THRUST_RTC_API uint32_t TRTC_Reduce_By_Key(const DVVectorLike& key_in, const DVVectorLike& value_in,
                                           DVVectorLike& key_out, DVVectorLike& value_out, const Functor& binary_pred);
THRUST_RTC_API uint32_t TRTC_Reduce_By_Key(const DVVectorLike& key_in, const DVVectorLike& value_in,
                                           DVVectorLike& key_out, DVVectorLike& value_out, const Functor& binary_pred,
                                           const Functor& binary_op);
THRUST_RTC_API bool TRTC_Transform_Reduce(const DVVectorLike& vec, const Functor& unary_op, const DeviceViewable& init,
                                          const Functor& binary_op, ViewBuf& ret);
THRUST_RTC_API bool TRTC_Min_Element(const DVVectorLike& vec, size_t& id_min);

// searches in a sorted view -- binary_search.h:10-25
THRUST_RTC_API bool TRTC_Lower_Bound(const DVVectorLike& vec, const DeviceViewable& value, size_t& result);
THRUST_RTC_API bool TRTC_Lower_Bound(const DVVectorLike& vec, const DeviceViewable& value, const Functor& comp,
                                     size_t& result);
THRUST_RTC_API bool TRTC_Upper_Bound(const DVVectorLike& vec, const DeviceViewable& value, size_t& result);
THRUST_RTC_API bool TRTC_Upper_Bound(const DVVectorLike& vec, const DeviceViewable& value, const Functor& comp,
                                     size_t& result);
THRUST_RTC_API bool TRTC_Binary_Search(const DVVectorLike& vec, const DeviceViewable& value, bool& result);
THRUST_RTC_API bool TRTC_Binary_Search(const DVVectorLike& vec, const DeviceViewable& value, const Functor& comp,
                                       bool& result);
THRUST_RTC_API bool TRTC_Lower_Bound_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result);
THRUST_RTC_API bool TRTC_Lower_Bound_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result,
                                       const Functor& comp);
THRUST_RTC_API bool TRTC_Upper_Bound_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result);
THRUST_RTC_API bool TRTC_Upper_Bound_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result,
                                       const Functor& comp);
THRUST_RTC_API bool TRTC_Binary_Search_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result);
THRUST_RTC_API bool TRTC_Binary_Search_V(const DVVectorLike& vec, const DVVectorLike& values, DVVectorLike& result,
                                         const Functor& comp);

THRUST_RTC_API bool TRTC_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_out);
THRUST_RTC_API uint32_t TRTC_Copy_If(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& pred);
THRUST_RTC_API uint32_t TRTC_Copy_If_Stencil(const DVVectorLike& vec_in, const DVVectorLike& vec_stencil,
                                             DVVectorLike& vec_out, const Functor& pred);
THRUST_RTC_API uint32_t TRTC_Remove(DVVectorLike& vec, const DeviceViewable& value);
THRUST_RTC_API uint32_t TRTC_Remove_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_out, const DeviceViewable& value);
THRUST_RTC_API uint32_t TRTC_Remove_If(DVVectorLike& vec, const Functor& pred);
THRUST_RTC_API uint32_t TRTC_Remove_Copy_If(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& pred);
THRUST_RTC_API uint32_t TRTC_Remove_If_Stencil(DVVectorLike& vec, const DVVectorLike& stencil, const Functor& pred);
THRUST_RTC_API uint32_t TRTC_Remove_Copy_If_Stencil(const DVVectorLike& vec_in, const DVVectorLike& stencil,
                                                    DVVectorLike& vec_out, const Functor& pred);
THRUST_RTC_API uint32_t TRTC_Unique(DVVectorLike& vec);
THRUST_RTC_API uint32_t TRTC_Unique(DVVectorLike& vec, const Functor& binary_pred);
THRUST_RTC_API uint32_t TRTC_Unique_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_out);
THRUST_RTC_API uint32_t TRTC_Unique_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& binary_pred);
THRUST_RTC_API uint32_t TRTC_Unique_By_Key(DVVectorLike& keys, DVVectorLike& values);
THRUST_RTC_API uint32_t TRTC_Unique_By_Key(DVVectorLike& keys, DVVectorLike& values, const Functor& binary_pred);
THRUST_RTC_API uint32_t TRTC_Unique_By_Key_Copy(const DVVectorLike& keys_in, const DVVectorLike& values_in,
                                                DVVectorLike& keys_out, DVVectorLike& values_out);
THRUST_RTC_API uint32_t TRTC_Unique_By_Key_Copy(const DVVectorLike& keys_in, const DVVectorLike& values_in,
                                                DVVectorLike& keys_out, DVVectorLike& values_out,
                                                const Functor& binary_pred);
THRUST_RTC_API uint32_t TRTC_Partition(DVVectorLike& vec, const Functor& pred);
THRUST_RTC_API uint32_t TRTC_Partition_Stencil(DVVectorLike& vec, const DVVectorLike& stencil, const Functor& pred);
THRUST_RTC_API uint32_t TRTC_Partition_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_true, DVVectorLike& vec_false,
                                            const Functor& pred);
THRUST_RTC_API uint32_t TRTC_Partition_Copy_Stencil(const DVVectorLike& vec_in, const DVVectorLike& stencil,
                                                    DVVectorLike& vec_true, DVVectorLike& vec_false,
                                                    const Functor& pred);

// the remaining algorithms -- fill.h, sequence.h, tabulate.h, transform.h, replace.h,
// for_each.h, adjacent_difference.h, gather.h, scatter.h, swap.h, count.h, equal.h,
// logical.h, extrema.h, inner_product.h, find.h, mismatch.h, partition.h, sort.h, merge.h
THRUST_RTC_API bool TRTC_Fill(DVVectorLike& vec, const DeviceViewable& value);
THRUST_RTC_API bool TRTC_Sequence(DVVectorLike& vec);
THRUST_RTC_API bool TRTC_Sequence(DVVectorLike& vec, const DeviceViewable& value_init);
THRUST_RTC_API bool TRTC_Sequence(DVVectorLike& vec, const DeviceViewable& value_init,
                                  const DeviceViewable& value_step);
THRUST_RTC_API bool TRTC_Tabulate(DVVectorLike& vec, const Functor& op);
THRUST_RTC_API bool TRTC_For_Each(DVVectorLike& vec, const Functor& f);
THRUST_RTC_API bool TRTC_Transform(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& op);
THRUST_RTC_API bool TRTC_Transform_Binary(const DVVectorLike& vec_in1, const DVVectorLike& vec_in2,
                                          DVVectorLike& vec_out, const Functor& op);
THRUST_RTC_API bool TRTC_Transform_If(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& op,
                                      const Functor& pred);
THRUST_RTC_API bool TRTC_Transform_If_Stencil(const DVVectorLike& vec_in, const DVVectorLike& vec_stencil,
                                              DVVectorLike& vec_out, const Functor& op, const Functor& pred);
THRUST_RTC_API bool TRTC_Transform_Binary_If_Stencil(const DVVectorLike& vec_in1, const DVVectorLike& vec_in2,
                                                     const DVVectorLike& vec_stencil, DVVectorLike& vec_out,
                                                     const Functor& op, const Functor& pred);
THRUST_RTC_API bool TRTC_Replace(DVVectorLike& vec, const DeviceViewable& old_value, const DeviceViewable& new_value);
THRUST_RTC_API bool TRTC_Replace_If(DVVectorLike& vec, const Functor& pred, const DeviceViewable& new_value);
THRUST_RTC_API bool TRTC_Replace_Copy(const DVVectorLike& vec_in, DVVectorLike& vec_out,
                                      const DeviceViewable& old_value, const DeviceViewable& new_value);
THRUST_RTC_API bool TRTC_Replace_Copy_If(const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& pred,
                                         const DeviceViewable& new_value);
THRUST_RTC_API bool TRTC_Adjacent_Difference(const DVVectorLike& vec_in, DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Adjacent_Difference(const DVVectorLike& vec_in, DVVectorLike& vec_out,
                                             const Functor& binary_op);
THRUST_RTC_API bool TRTC_Gather(const DVVectorLike& vec_map, const DVVectorLike& vec_in, DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Gather_If(const DVVectorLike& vec_map, const DVVectorLike& vec_stencil,
                                   const DVVectorLike& vec_in, DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Gather_If(const DVVectorLike& vec_map, const DVVectorLike& vec_stencil,
                                   const DVVectorLike& vec_in, DVVectorLike& vec_out, const Functor& pred);
THRUST_RTC_API bool TRTC_Scatter(const DVVectorLike& vec_in, const DVVectorLike& vec_map, DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Scatter_If(const DVVectorLike& vec_in, const DVVectorLike& vec_map,
                                    const DVVectorLike& vec_stencil, DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Scatter_If(const DVVectorLike& vec_in, const DVVectorLike& vec_map,
                                    const DVVectorLike& vec_stencil, DVVectorLike& vec_out, const Functor& pred);
THRUST_RTC_API bool TRTC_Swap(DVVectorLike& vec1, DVVectorLike& vec2);

THRUST_RTC_API bool TRTC_Count(const DVVectorLike& vec, const DeviceViewable& value, size_t& ret);
THRUST_RTC_API bool TRTC_Count_If(const DVVectorLike& vec, const Functor& pred, size_t& ret);
THRUST_RTC_API bool TRTC_Equal(const DVVectorLike& vec1, const DVVectorLike& vec2, bool& ret);
THRUST_RTC_API bool TRTC_Equal(const DVVectorLike& vec1, const DVVectorLike& vec2, const Functor& binary_pred,
                               bool& ret);
THRUST_RTC_API bool TRTC_All_Of(const DVVectorLike& vec, const Functor& pred, bool& ret);
THRUST_RTC_API bool TRTC_Any_Of(const DVVectorLike& vec, const Functor& pred, bool& ret);
THRUST_RTC_API bool TRTC_None_Of(const DVVectorLike& vec, const Functor& pred, bool& ret);
THRUST_RTC_API bool TRTC_Min_Element(const DVVectorLike& vec, const Functor& comp, size_t& id_min);
THRUST_RTC_API bool TRTC_Max_Element(const DVVectorLike& vec, size_t& id_max);
THRUST_RTC_API bool TRTC_Max_Element(const DVVectorLike& vec, const Functor& comp, size_t& id_max);
THRUST_RTC_API bool TRTC_MinMax_Element(const DVVectorLike& vec, size_t& id_min, size_t& id_max);
THRUST_RTC_API bool TRTC_MinMax_Element(const DVVectorLike& vec, const Functor& comp, size_t& id_min, size_t& id_max);
THRUST_RTC_API bool TRTC_Inner_Product(const DVVectorLike& vec1, const DVVectorLike& vec2, const DeviceViewable& init,
                                       ViewBuf& ret);
THRUST_RTC_API bool TRTC_Inner_Product(const DVVectorLike& vec1, const DVVectorLike& vec2, const DeviceViewable& init,
                                       ViewBuf& ret, const Functor& binary_op1, const Functor& binary_op2);

THRUST_RTC_API bool TRTC_Find(const DVVectorLike& vec, const DeviceViewable& value, size_t& result);
THRUST_RTC_API bool TRTC_Find_If(const DVVectorLike& vec, const Functor& pred, size_t& result);
THRUST_RTC_API bool TRTC_Find_If_Not(const DVVectorLike& vec, const Functor& pred, size_t& result);
THRUST_RTC_API bool TRTC_Mismatch(const DVVectorLike& vec1, const DVVectorLike& vec2, size_t& result);
THRUST_RTC_API bool TRTC_Mismatch(const DVVectorLike& vec1, const DVVectorLike& vec2, const Functor& pred,
                                  size_t& result);
THRUST_RTC_API bool TRTC_Partition_Point(const DVVectorLike& vec, const Functor& pred, size_t& result);
THRUST_RTC_API bool TRTC_Is_Partitioned(const DVVectorLike& vec, const Functor& pred, bool& result);
THRUST_RTC_API bool TRTC_Is_Sorted(const DVVectorLike& vec, bool& result);
THRUST_RTC_API bool TRTC_Is_Sorted(const DVVectorLike& vec, const Functor& comp, bool& result);
THRUST_RTC_API bool TRTC_Is_Sorted_Until(const DVVectorLike& vec, size_t& result);
THRUST_RTC_API bool TRTC_Is_Sorted_Until(const DVVectorLike& vec, const Functor& comp, size_t& result);

THRUST_RTC_API bool TRTC_Merge(const DVVectorLike& vec1, const DVVectorLike& vec2, DVVectorLike& vec_out);
THRUST_RTC_API bool TRTC_Merge(const DVVectorLike& vec1, const DVVectorLike& vec2, DVVectorLike& vec_out,
                               const Functor& comp);
THRUST_RTC_API bool TRTC_Merge_By_Key(const DVVectorLike& keys1, const DVVectorLike& keys2,
                                      const DVVectorLike& value1, const DVVectorLike& value2, DVVectorLike& keys_out,
                                      DVVectorLike& value_out);
THRUST_RTC_API bool TRTC_Merge_By_Key(const DVVectorLike& keys1, const DVVectorLike& keys2,
                                      const DVVectorLike& value1, const DVVectorLike& value2, DVVectorLike& keys_out,
                                      DVVectorLike& value_out, const Functor& comp);
