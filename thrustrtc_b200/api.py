"""Python interface of thrustrtc_b200, mirroring the reference's ``ThrustRTC`` package
(python/ThrustRTC/*.py): the same class and function names, argument order, defaults and
error behaviour (``SystemError`` on an internal failure, python/ThrustRTC/Native.py:14-37),
over the drop-in C ABI of libPyThrustRTC.so (include/thrustrtc_b200.h).
"""
import ctypes

import numpy as np

from ._native import lib, vp, u64, i32, u32, f32, f64, cstr, i64, last_error

# ---------------------------------------------------------------- C signatures
_SIGS = {
    "n_string_array_create": (vp, [u64, ctypes.POINTER(cstr)]),
    "n_string_array_destroy": (None, [vp]),
    "n_pointer_array_create": (vp, [u64, ctypes.POINTER(vp)]),
    "n_pointer_array_destroy": (None, [vp]),
    "n_dim3_create": (vp, [u32, u32, u32]),
    "n_dim3_destroy": (None, [vp]),
    "n_set_libnvrtc_path": (None, [cstr]),
    "n_trtc_try_init": (i32, []),
    "n_get_ptx_arch": (i32, []),
    "n_set_verbose": (None, [u32]),
    "n_set_kernel_debug": (None, [u32]),
    "n_add_include_dir": (None, [cstr]),
    "n_add_built_in_header": (None, [cstr, cstr]),
    "n_add_inlcude_filename": (None, [cstr]),
    "n_add_code_block": (None, [cstr]),
    "n_add_constant_object": (None, [cstr, vp]),
    "n_wait": (None, []),
    "n_kernel_create": (vp, [vp, cstr]),
    "n_kernel_destroy": (None, [vp]),
    "n_kernel_num_params": (i32, [vp]),
    "n_kernel_calc_optimal_block_size": (i32, [vp, vp, u32]),
    "n_kernel_calc_number_blocks": (i32, [vp, vp, i32, u32]),
    "n_kernel_launch": (i32, [vp, vp, vp, vp, i32]),
    "n_for_create": (vp, [vp, cstr, cstr]),
    "n_for_destroy": (None, [vp]),
    "n_for_num_params": (i32, [vp]),
    "n_for_launch": (i32, [vp, i32, i32, vp]),
    "n_for_launch_n": (i32, [vp, i32, vp]),
    "n_dv_name_view_cls": (cstr, [vp]),
    "n_dv_destroy": (None, [vp]),
    "n_dvint8_create": (vp, [i32]), "n_dvint8_value": (i32, [vp]),
    "n_dvuint8_create": (vp, [u32]), "n_dvuint8_value": (u32, [vp]),
    "n_dvint16_create": (vp, [i32]), "n_dvint16_value": (i32, [vp]),
    "n_dvuint16_create": (vp, [u32]), "n_dvuint16_value": (u32, [vp]),
    "n_dvint32_create": (vp, [i32]), "n_dvint32_value": (i32, [vp]),
    "n_dvuint32_create": (vp, [u32]), "n_dvuint32_value": (u32, [vp]),
    "n_dvint64_create": (vp, [i64]), "n_dvint64_value": (i64, [vp]),
    "n_dvuint64_create": (vp, [u64]), "n_dvuint64_value": (u64, [vp]),
    "n_dvfloat_create": (vp, [f32]), "n_dvfloat_value": (f32, [vp]),
    "n_dvdouble_create": (vp, [f64]), "n_dvdouble_value": (f64, [vp]),
    "n_dvbool_create": (vp, [i32]), "n_dvbool_value": (i32, [vp]),
    "n_dvcomplex64_create": (vp, [f32, f32]), "n_dvcomplex64_real": (f32, [vp]), "n_dvcomplex64_imag": (f32, [vp]),
    "n_dvcomplex128_create": (vp, [f64, f64]), "n_dvcomplex128_real": (f64, [vp]),
    "n_dvcomplex128_imag": (f64, [vp]),
    "n_dvvectorlike_name_elem_cls": (cstr, [vp]),
    "n_dvvectorlike_size": (u64, [vp]),
    "n_dvvector_create": (vp, [cstr, u64, vp]),
    "n_dvvector_to_host": (None, [vp, vp, u64, u64]),
    "n_dvvector_from_dvs": (vp, [vp]),
    "n_dvvectoradaptor_create": (vp, [cstr, u64, vp]),
    "n_dvrange_create": (vp, [vp, u64, u64]),
    "n_dvconstant_create": (vp, [vp, u64]),
    "n_dvcounter_create": (vp, [vp, u64]),
    "n_dvdiscard_create": (vp, [cstr, u64]),
    "n_dvpermutation_create": (vp, [vp, vp]),
    "n_dvreverse_create": (vp, [vp]),
    "n_dvtransform_create": (vp, [vp, cstr, vp]),
    "n_dvtuple_create": (vp, [vp, vp]), "n_dvzipped_create": (vp, [vp, vp]),
    "n_dvcustomvector_create": (vp, [vp, vp, cstr, cstr, cstr, u64, u32]),
    "n_functor_create": (vp, [vp, vp, vp, cstr]),
    "n_built_in_functor_create": (vp, [cstr]),
    "n_copy": (i32, [vp, vp]),
    "n_reduce": (vp, [vp, vp, vp]),
    "n_reduce_by_key": (u32, [vp, vp, vp, vp, vp, vp]),
    "n_min_element": (u64, [vp, vp]),
    "n_lower_bound": (u64, [vp, vp, vp]), "n_upper_bound": (u64, [vp, vp, vp]),
    "n_binary_search": (i32, [vp, vp, vp]), "n_lower_bound_v": (i32, [vp, vp, vp, vp]),
    "n_upper_bound_v": (i32, [vp, vp, vp, vp]), "n_binary_search_v": (i32, [vp, vp, vp, vp]),
    "n_transform_reduce": (vp, [vp, vp, vp, vp]),
    "n_inclusive_scan": (i32, [vp, vp, vp]),
    "n_exclusive_scan": (i32, [vp, vp, vp, vp]),
    "n_inclusive_scan_by_key": (i32, [vp, vp, vp, vp, vp]),
    "n_exclusive_scan_by_key": (i32, [vp, vp, vp, vp, vp, vp]),
    "n_transform_inclusive_scan": (i32, [vp, vp, vp, vp]),
    "n_transform_exclusive_scan": (i32, [vp, vp, vp, vp, vp]),
    "n_copy_if": (u32, [vp, vp, vp]),
    "n_copy_if_stencil": (u32, [vp, vp, vp, vp]),
    "n_remove": (u32, [vp, vp]),
    "n_remove_copy": (u32, [vp, vp, vp]),
    "n_remove_if": (u32, [vp, vp]),
    "n_remove_copy_if": (u32, [vp, vp, vp]),
    "n_remove_if_stencil": (u32, [vp, vp, vp]),
    "n_remove_copy_if_stencil": (u32, [vp, vp, vp, vp]),
    "n_unique": (u32, [vp, vp]),
    "n_unique_copy": (u32, [vp, vp, vp]),
    "n_unique_by_key": (u32, [vp, vp, vp]),
    "n_unique_by_key_copy": (u32, [vp, vp, vp, vp, vp]),
    "n_partition": (u32, [vp, vp]),
    "n_partition_stencil": (u32, [vp, vp, vp]),
    "n_partition_copy": (u32, [vp, vp, vp, vp]),
    "n_partition_copy_stencil": (u32, [vp, vp, vp, vp, vp]),
    "n_sort": (i32, [vp, vp]),
    "n_sort_by_key": (i32, [vp, vp, vp]),
    "n_fill": (i32, [vp, vp]),
    "n_replace": (i32, [vp, vp, vp]), "n_replace_if": (i32, [vp, vp, vp]),
    "n_replace_copy": (i32, [vp, vp, vp, vp]), "n_replace_copy_if": (i32, [vp, vp, vp, vp]),
    "n_for_each": (i32, [vp, vp]),
    "n_adjacent_difference": (i32, [vp, vp, vp]),
    "n_sequence": (i32, [vp, vp, vp]),
    "n_tabulate": (i32, [vp, vp]),
    "n_transform": (i32, [vp, vp, vp]),
    "n_transform_binary": (i32, [vp, vp, vp, vp]),
    "n_transform_if": (i32, [vp, vp, vp, vp]),
    "n_transform_if_stencil": (i32, [vp, vp, vp, vp, vp]),
    "n_transform_binary_if_stencil": (i32, [vp, vp, vp, vp, vp, vp]),
    "n_gather": (i32, [vp, vp, vp]), "n_gather_if": (i32, [vp, vp, vp, vp, vp]),
    "n_scatter": (i32, [vp, vp, vp]), "n_scatter_if": (i32, [vp, vp, vp, vp, vp]),
    "n_swap": (i32, [vp, vp]),
    "n_count": (u64, [vp, vp]), "n_count_if": (u64, [vp, vp]),
    "n_equal": (i32, [vp, vp, vp]),
    "n_max_element": (u64, [vp, vp]),
    "n_minmax_element": (i32, [vp, vp, ctypes.POINTER(u64)]),
    "n_inner_product": (vp, [vp, vp, vp, vp, vp]),
    "n_all_of": (i32, [vp, vp]), "n_any_of": (i32, [vp, vp]), "n_none_of": (i32, [vp, vp]),
    "n_is_partitioned": (i32, [vp, vp]),
    "n_is_sorted": (i32, [vp, vp]),
    "n_find": (i64, [vp, vp]), "n_find_if": (i64, [vp, vp]), "n_find_if_not": (i64, [vp, vp]),
    "n_mismatch": (i64, [vp, vp, vp]),
    "n_partition_point": (u64, [vp, vp]),
    "n_is_sorted_until": (u64, [vp, vp]),
    "n_merge": (i32, [vp, vp, vp, vp]),
    "n_merge_by_key": (i32, [vp, vp, vp, vp, vp, vp, vp]),
}
for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def _fail(msg="An internal error happend"):
    detail = last_error()
    raise SystemError(msg + (": " + detail if detail else ""))


def check_i(r):
    if r == -1:
        _fail()
    if r == -2:
        raise ValueError("Wrong number of arguments.")
    if r == -100:
        raise ImportError("cannot import ThrustRTC")
    return r


def check_u(r):
    if r == 0xFFFFFFFF:
        _fail()
    return r


def check_ull(r):
    if r == 0xFFFFFFFFFFFFFFFF:
        _fail()
    return r


def check_cptr(p):
    if not p:
        _fail()
    return p


def _p(obj):
    return None if obj is None else obj.m_cptr


class _StrArray:
    def __init__(self, strs):
        enc = [s.encode("utf-8") for s in strs]
        arr = (cstr * max(1, len(enc)))(*enc)
        self.m_cptr = lib.n_string_array_create(len(enc), arr)

    def __del__(self):
        lib.n_string_array_destroy(self.m_cptr)


class _ObjArray:
    def __init__(self, objs):
        arr = (vp * max(1, len(objs)))(*[o.m_cptr for o in objs])
        self.m_cptr = lib.n_pointer_array_create(len(objs), arr)

    def __del__(self):
        lib.n_pointer_array_destroy(self.m_cptr)


class _Dim3:
    def __init__(self, t):
        v = [1, 1, 1]
        if isinstance(t, tuple):
            v[: len(t)] = t
        else:
            v[0] = t
        self.m_cptr = lib.n_dim3_create(*v)

    def __del__(self):
        lib.n_dim3_destroy(self.m_cptr)


# ---------------------------------------------------------------- context
def set_libnvrtc_path(path):
    lib.n_set_libnvrtc_path(path.encode("utf-8"))


def Set_Verbose(verbose=True):
    lib.n_set_verbose(1 if verbose else 0)


def Set_Kernel_Debug(kernel_debug=True):
    lib.n_set_kernel_debug(1 if kernel_debug else 0)


def Get_PTX_Arch():
    return lib.n_get_ptx_arch()


def Add_Include_Dir(path):
    lib.n_add_include_dir(path.encode("utf-8"))


def Add_Built_In_Header(filename, filecontent):
    lib.n_add_built_in_header(filename.encode("utf-8"), filecontent.encode("utf-8"))


def Add_Inlcude_Filename(filename):
    lib.n_add_inlcude_filename(filename.encode("utf-8"))


def Add_Code_Block(code):
    lib.n_add_code_block(code.encode("utf-8"))


def Add_Constant_Object(name, dv):
    lib.n_add_constant_object(name.encode("utf-8"), dv.m_cptr)


def Wait():
    lib.n_wait()


class Kernel:
    def __init__(self, param_names, body):
        names = _StrArray(param_names)
        self.m_cptr = check_cptr(lib.n_kernel_create(names.m_cptr, body.encode("utf-8")))

    def __del__(self):
        lib.n_kernel_destroy(self.m_cptr)

    def num_params(self):
        return lib.n_kernel_num_params(self.m_cptr)

    def calc_optimal_block_size(self, args, sharedMemBytes=0):
        a = _ObjArray(args)
        return check_i(lib.n_kernel_calc_optimal_block_size(self.m_cptr, a.m_cptr, sharedMemBytes))

    def calc_number_blocks(self, args, size_block, sharedMemBytes=0):
        a = _ObjArray(args)
        return check_i(lib.n_kernel_calc_number_blocks(self.m_cptr, a.m_cptr, size_block, sharedMemBytes))

    def launch(self, gridDim, blockDim, args, sharedMemBytes=0):
        g, b, a = _Dim3(gridDim), _Dim3(blockDim), _ObjArray(args)
        return check_i(lib.n_kernel_launch(self.m_cptr, g.m_cptr, b.m_cptr, a.m_cptr, sharedMemBytes))


class For:
    def __init__(self, param_names, name_iter, body):
        names = _StrArray(param_names)
        self.m_cptr = check_cptr(lib.n_for_create(names.m_cptr, name_iter.encode("utf-8"), body.encode("utf-8")))

    def __del__(self):
        lib.n_for_destroy(self.m_cptr)

    def num_params(self):
        return lib.n_for_num_params(self.m_cptr)

    def launch(self, begin, end, args):
        a = _ObjArray(args)
        check_i(lib.n_for_launch(self.m_cptr, begin, end, a.m_cptr))

    def launch_n(self, n, args):
        a = _ObjArray(args)
        check_i(lib.n_for_launch_n(self.m_cptr, n, a.m_cptr))


# ---------------------------------------------------------------- device viewables
class DeviceViewable:
    m_cptr = None

    def name_view_cls(self):
        return lib.n_dv_name_view_cls(self.m_cptr).decode("utf-8")

    def __del__(self):
        if self.m_cptr:
            lib.n_dv_destroy(self.m_cptr)
            self.m_cptr = None

    def value(self):
        return "[Device-viewable object, type: %s]" % self.name_view_cls()


def _scalar_class(clsname, prefix, conv=None):
    create = getattr(lib, "n_dv%s_create" % prefix)
    getv = getattr(lib, "n_dv%s_value" % prefix)

    def __init__(self, value):
        self.m_cptr = check_cptr(create(value))

    def value(self):
        v = getv(self.m_cptr)
        return conv(v) if conv else v

    return type(clsname, (DeviceViewable,), {"__init__": __init__, "value": value})


DVInt8 = _scalar_class("DVInt8", "int8")
DVUInt8 = _scalar_class("DVUInt8", "uint8")
DVInt16 = _scalar_class("DVInt16", "int16")
DVUInt16 = _scalar_class("DVUInt16", "uint16")
DVInt32 = _scalar_class("DVInt32", "int32")
DVUInt32 = _scalar_class("DVUInt32", "uint32")
DVInt64 = _scalar_class("DVInt64", "int64")
DVUInt64 = _scalar_class("DVUInt64", "uint64")
DVFloat = _scalar_class("DVFloat", "float")
DVDouble = _scalar_class("DVDouble", "double")
DVBool = _scalar_class("DVBool", "bool", lambda v: v != 0)


class DVComplex64(DeviceViewable):
    def __init__(self, value):
        self.m_cptr = check_cptr(lib.n_dvcomplex64_create(value.real, value.imag))

    def value(self):
        return complex(lib.n_dvcomplex64_real(self.m_cptr), lib.n_dvcomplex64_imag(self.m_cptr))


class DVComplex128(DeviceViewable):
    def __init__(self, value):
        self.m_cptr = check_cptr(lib.n_dvcomplex128_create(value.real, value.imag))

    def value(self):
        return complex(lib.n_dvcomplex128_real(self.m_cptr), lib.n_dvcomplex128_imag(self.m_cptr))


_VALUE_OF = {
    "int8_t": "n_dvint8_value", "uint8_t": "n_dvuint8_value", "int16_t": "n_dvint16_value",
    "uint16_t": "n_dvuint16_value", "int32_t": "n_dvint32_value", "uint32_t": "n_dvuint32_value",
    "int64_t": "n_dvint64_value", "uint64_t": "n_dvuint64_value", "float": "n_dvfloat_value",
    "double": "n_dvdouble_value",
}


def _value_from_dvptr(cptr):
    cls = lib.n_dv_name_view_cls(cptr).decode("utf-8")
    if cls in _VALUE_OF:
        return getattr(lib, _VALUE_OF[cls])(cptr)
    if cls == "bool":
        return lib.n_dvbool_value(cptr) != 0
    if cls == "cuFloatComplex":
        return complex(lib.n_dvcomplex64_real(cptr), lib.n_dvcomplex64_imag(cptr))
    if cls == "cuDoubleComplex":
        return complex(lib.n_dvcomplex128_real(cptr), lib.n_dvcomplex128_imag(cptr))
    return "[Device-viewable object, type: %s]" % cls


# ---------------------------------------------------------------- vectors
_NP_OF = {
    "int8_t": np.int8, "uint8_t": np.uint8, "int16_t": np.int16, "uint16_t": np.uint16,
    "int32_t": np.int32, "uint32_t": np.uint32, "int64_t": np.int64, "uint64_t": np.uint64,
    "float": np.float32, "double": np.float64, "bool": np.bool_,
    "cuFloatComplex": np.complex64, "cuDoubleComplex": np.complex128,
}
_CLS_OF = {np.dtype(v): k for k, v in _NP_OF.items()}


class DVVectorLike(DeviceViewable):
    def name_elem_cls(self):
        return lib.n_dvvectorlike_name_elem_cls(self.m_cptr).decode("utf-8")

    def size(self):
        return lib.n_dvvectorlike_size(self.m_cptr)

    def range(self, begin=0, end=-1):
        return DVRange(self, begin, end)


class DVRange(DVVectorLike):
    def __init__(self, src, begin=0, end=-1):
        self.m_src = src
        self.m_cptr = check_cptr(lib.n_dvrange_create(src.m_cptr, ctypes.c_ulonglong(begin).value,
                                                      ctypes.c_ulonglong(end).value))


class DVVector(DVVectorLike):
    def __init__(self, cptr):
        self.m_cptr = cptr

    def to_host(self, begin=0, end=-1):
        dt = _NP_OF[self.name_elem_cls()]
        if end == -1:
            end = self.size()
        out = np.empty(end - begin, dtype=dt)
        if end > begin:
            lib.n_dvvector_to_host(self.m_cptr, out.ctypes.data, begin, end)
        return out


def device_vector(elem_cls, size, ptr_host_data=None):
    if size < 1:
        raise ValueError("0-size vector not allowed")
    return DVVector(check_cptr(lib.n_dvvector_create(elem_cls.encode("utf-8"), size, ptr_host_data)))


def device_vector_from_numpy(nparr):
    nparr = np.ascontiguousarray(nparr)
    return device_vector(_CLS_OF[nparr.dtype], len(nparr), nparr.ctypes.data)


def device_vector_from_list(lst, elem_cls):
    arr = np.array(lst, dtype=_NP_OF[elem_cls])
    return device_vector(elem_cls, len(lst), arr.ctypes.data)


def device_vector_from_dvs(lst_dv):
    if len(lst_dv) < 1:
        raise ValueError("0-size vector not allowed")
    a = _ObjArray(lst_dv)
    return DVVector(check_cptr(lib.n_dvvector_from_dvs(a.m_cptr)))


class DVVectorAdaptor(DVVectorLike):
    """A non-owning view of device memory (the reference's DVNumbaVector / DVCupyVector)."""

    def __init__(self, elem_cls, size, ptr, owner=None):
        self.m_owner = owner
        self.m_cptr = check_cptr(lib.n_dvvectoradaptor_create(elem_cls.encode("utf-8"), size, ptr))


class _CudaArrayVector(DVVectorAdaptor):
    """A non-owning view of any contiguous 1-D device array that exposes the CUDA Array
    Interface (``__cuda_array_interface__``: CuPy, Numba, PyTorch, ...); keeps a reference."""

    def __init__(self, arr):
        cai = arr.__cuda_array_interface__
        dt = np.dtype(cai["typestr"])
        if dt not in _CLS_OF:
            raise ValueError("unsupported element type %s" % dt)
        shape = tuple(cai["shape"])
        size = int(np.prod(shape)) if shape else 1
        strides = cai.get("strides")
        if strides is not None and len(shape) == 1 and strides[0] != dt.itemsize:
            raise ValueError("the array must be contiguous")
        DVVectorAdaptor.__init__(self, _CLS_OF[dt], size, ctypes.c_void_p(cai["data"][0]), owner=arr)


class DVCupyVector(_CudaArrayVector):
    """A CuPy device array as a vector (Python DVVector.py:178-212)."""

    def __init__(self, cparr):
        self.cparr = cparr
        _CudaArrayVector.__init__(self, cparr)


class DVNumbaVector(_CudaArrayVector):
    """A Numba device array as a vector (Python DVVector.py:141-176)."""

    def __init__(self, nbarr):
        self.nbarr = nbarr
        _CudaArrayVector.__init__(self, nbarr)


class DVTorchVector(DVVectorAdaptor):
    """Adapts a contiguous 1-D CUDA torch tensor (keeps a reference to it)."""

    _TORCH = {"int8": "int8_t", "uint8": "uint8_t", "int16": "int16_t", "int32": "int32_t", "int64": "int64_t",
              "float32": "float", "float64": "double", "bool": "bool", "uint16": "uint16_t", "uint32": "uint32_t",
              "uint64": "uint64_t"}

    def __init__(self, tensor, elem_cls=None):
        if elem_cls is None:
            elem_cls = self._TORCH[str(tensor.dtype).replace("torch.", "")]
        DVVectorAdaptor.__init__(self, elem_cls, tensor.numel(), tensor.data_ptr(), owner=tensor)


class DVConstant(DVVectorLike):
    def __init__(self, dvobj, size=-1):
        self.m_dv = dvobj
        self.m_cptr = check_cptr(lib.n_dvconstant_create(dvobj.m_cptr, ctypes.c_ulonglong(size).value))


class DVCounter(DVVectorLike):
    def __init__(self, dvobj_init, size=-1):
        self.m_dv = dvobj_init
        self.m_cptr = check_cptr(lib.n_dvcounter_create(dvobj_init.m_cptr, ctypes.c_ulonglong(size).value))


class DVDiscard(DVVectorLike):
    def __init__(self, elem_cls, size=-1):
        self.m_cptr = check_cptr(lib.n_dvdiscard_create(elem_cls.encode("utf-8"), ctypes.c_ulonglong(size).value))


class DVPermutation(DVVectorLike):
    def __init__(self, vec_value, vec_index):
        self.m_value, self.m_index = vec_value, vec_index
        self.m_cptr = check_cptr(lib.n_dvpermutation_create(vec_value.m_cptr, vec_index.m_cptr))


class DVReverse(DVVectorLike):
    def __init__(self, vec_value):
        self.m_value = vec_value
        self.m_cptr = check_cptr(lib.n_dvreverse_create(vec_value.m_cptr))


class DVTransform(DVVectorLike):
    def __init__(self, vec_in, elem_cls, op):
        self.m_in, self.m_op = vec_in, op
        self.m_cptr = check_cptr(lib.n_dvtransform_create(vec_in.m_cptr, elem_cls.encode("utf-8"), op.m_cptr))


class DVZipped(DVVectorLike):
    """FakeVectors.py:37-42"""

    def __init__(self, vecs, elem_names):
        self.m_vecs = vecs
        o_vecs, o_names = _ObjArray(vecs), _StrArray(elem_names)
        self.m_cptr = check_cptr(lib.n_dvzipped_create(o_vecs.m_cptr, o_names.m_cptr))


class DVCustomVector(DVVectorLike):
    """FakeVectors.py:44-55"""

    def __init__(self, arg_map, name_idx, code_body, elem_cls, size=-1, read_only=True):
        self.m_arg_map = arg_map
        o_names = _StrArray(list(arg_map.keys()))
        o_elems = _ObjArray(list(arg_map.values()))
        self.m_cptr = check_cptr(lib.n_dvcustomvector_create(
            o_elems.m_cptr, o_names.m_cptr, name_idx.encode("utf-8"), code_body.encode("utf-8"),
            elem_cls.encode("utf-8"), ctypes.c_ulonglong(size).value, 1 if read_only else 0))


class DVTuple(DeviceViewable):
    """DVTuple.py:5-12"""

    def __init__(self, elem_map):
        self.m_elem_map = elem_map
        o_names = _StrArray(list(elem_map.keys()))
        o_elems = _ObjArray(list(elem_map.values()))
        self.m_cptr = check_cptr(lib.n_dvtuple_create(o_elems.m_cptr, o_names.m_cptr))


# ---------------------------------------------------------------- functors
class Functor(DeviceViewable):
    def __init__(self, arg_map, functor_params, code_body):
        self.m_arg_map = arg_map
        names = _StrArray(list(arg_map.keys()))
        objs = _ObjArray(list(arg_map.values()))
        params = _StrArray(functor_params)
        self.m_cptr = check_cptr(lib.n_functor_create(objs.m_cptr, names.m_cptr, params.m_cptr,
                                                      code_body.encode("utf-8")))


def _built_in(name):
    def __init__(self):
        self.m_cptr = check_cptr(lib.n_built_in_functor_create(name.encode("utf-8")))
    return type(name, (DeviceViewable,), {"__init__": __init__})


Identity = _built_in("Identity")
Maximum = _built_in("Maximum")
Minimum = _built_in("Minimum")
EqualTo = _built_in("EqualTo")
NotEqualTo = _built_in("NotEqualTo")
Greater = _built_in("Greater")
Less = _built_in("Less")
GreaterEqual = _built_in("GreaterEqual")
LessEqual = _built_in("LessEqual")
Plus = _built_in("Plus")
Minus = _built_in("Minus")
Multiplies = _built_in("Multiplies")
Divides = _built_in("Divides")
Modulus = _built_in("Modulus")
Negate = _built_in("Negate")


# ---------------------------------------------------------------- algorithms
def Copy(vec_in, vec_out):
    check_i(lib.n_copy(vec_in.m_cptr, vec_out.m_cptr))


def Sort(vec, comp=None):
    check_i(lib.n_sort(vec.m_cptr, _p(comp)))


def Sort_By_Key(keys, values, comp=None):
    check_i(lib.n_sort_by_key(keys.m_cptr, values.m_cptr, _p(comp)))


def Inclusive_Scan(vec_in, vec_out, binary_op=None):
    check_i(lib.n_inclusive_scan(vec_in.m_cptr, vec_out.m_cptr, _p(binary_op)))


def Exclusive_Scan(vec_in, vec_out, value_init=None, binary_op=None):
    check_i(lib.n_exclusive_scan(vec_in.m_cptr, vec_out.m_cptr, _p(value_init), _p(binary_op)))


def Transform_Inclusive_Scan(vec_in, vec_out, unary_op, binary_op):
    check_i(lib.n_transform_inclusive_scan(vec_in.m_cptr, vec_out.m_cptr, unary_op.m_cptr, binary_op.m_cptr))


def Transform_Exclusive_Scan(vec_in, vec_out, unary_op, value_init, binary_op):
    check_i(lib.n_transform_exclusive_scan(vec_in.m_cptr, vec_out.m_cptr, unary_op.m_cptr, value_init.m_cptr,
                                           binary_op.m_cptr))


def Inclusive_Scan_By_Key(vec_key, vec_value, vec_out, binary_pred=None, binary_op=None):
    check_i(lib.n_inclusive_scan_by_key(vec_key.m_cptr, vec_value.m_cptr, vec_out.m_cptr, _p(binary_pred),
                                        _p(binary_op)))


def Exclusive_Scan_By_Key(vec_key, vec_value, vec_out, value_init=None, binary_pred=None, binary_op=None):
    check_i(lib.n_exclusive_scan_by_key(vec_key.m_cptr, vec_value.m_cptr, vec_out.m_cptr, _p(value_init),
                                        _p(binary_pred), _p(binary_op)))


def Reduce(vec, value_init=None, binary_op=None):
    dvptr = check_cptr(lib.n_reduce(vec.m_cptr, _p(value_init), _p(binary_op)))
    ret = _value_from_dvptr(dvptr)
    lib.n_dv_destroy(dvptr)
    return ret


def Reduce_By_Key(key_in, value_in, key_out, value_out, binary_pred=None, binary_op=None):
    return check_u(lib.n_reduce_by_key(key_in.m_cptr, value_in.m_cptr, key_out.m_cptr, value_out.m_cptr,
                                       _p(binary_pred), _p(binary_op)))


def Transform_Reduce(vec, unary_op, value_init, binary_op):
    dvptr = check_cptr(lib.n_transform_reduce(vec.m_cptr, unary_op.m_cptr, value_init.m_cptr, binary_op.m_cptr))
    ret = _value_from_dvptr(dvptr)
    lib.n_dv_destroy(dvptr)
    return ret


def Min_Element(vec, comp=None):
    return check_ull(lib.n_min_element(vec.m_cptr, _p(comp)))


# ---------------------------------------------------------------- searches (Searching.py:30-84)
def Lower_Bound(vec, value, comp=None):
    return check_ull(lib.n_lower_bound(vec.m_cptr, value.m_cptr, _p(comp)))


def Upper_Bound(vec, value, comp=None):
    return check_ull(lib.n_upper_bound(vec.m_cptr, value.m_cptr, _p(comp)))


def Binary_Search(vec, value, comp=None):
    res = check_i(lib.n_binary_search(vec.m_cptr, value.m_cptr, _p(comp)))
    return res != 0


def Lower_Bound_V(vec, values, result, comp=None):
    check_i(lib.n_lower_bound_v(vec.m_cptr, values.m_cptr, result.m_cptr, _p(comp)))


def Upper_Bound_V(vec, values, result, comp=None):
    check_i(lib.n_upper_bound_v(vec.m_cptr, values.m_cptr, result.m_cptr, _p(comp)))


def Binary_Search_V(vec, values, result, comp=None):
    check_i(lib.n_binary_search_v(vec.m_cptr, values.m_cptr, result.m_cptr, _p(comp)))


def Copy_If(vec_in, vec_out, pred):
    return check_u(lib.n_copy_if(vec_in.m_cptr, vec_out.m_cptr, pred.m_cptr))


def Copy_If_Stencil(vec_in, vec_stencil, vec_out, pred):
    return check_u(lib.n_copy_if_stencil(vec_in.m_cptr, vec_stencil.m_cptr, vec_out.m_cptr, pred.m_cptr))


def Remove(vec, value):
    return check_u(lib.n_remove(vec.m_cptr, value.m_cptr))


def Remove_Copy(vec_in, vec_out, value):
    return check_u(lib.n_remove_copy(vec_in.m_cptr, vec_out.m_cptr, value.m_cptr))


def Remove_If(vec, pred):
    return check_u(lib.n_remove_if(vec.m_cptr, pred.m_cptr))


def Remove_Copy_If(vec_in, vec_out, pred):
    return check_u(lib.n_remove_copy_if(vec_in.m_cptr, vec_out.m_cptr, pred.m_cptr))


def Remove_If_Stencil(vec, stencil, pred):
    return check_u(lib.n_remove_if_stencil(vec.m_cptr, stencil.m_cptr, pred.m_cptr))


def Remove_Copy_If_Stencil(vec_in, stencil, vec_out, pred):
    return check_u(lib.n_remove_copy_if_stencil(vec_in.m_cptr, stencil.m_cptr, vec_out.m_cptr, pred.m_cptr))


def Unique(vec, binary_pred=None):
    return check_u(lib.n_unique(vec.m_cptr, _p(binary_pred)))


def Unique_Copy(vec_in, vec_out, binary_pred=None):
    return check_u(lib.n_unique_copy(vec_in.m_cptr, vec_out.m_cptr, _p(binary_pred)))


def Unique_By_Key(keys, values, binary_pred=None):
    return check_u(lib.n_unique_by_key(keys.m_cptr, values.m_cptr, _p(binary_pred)))


def Unique_By_Key_Copy(keys_in, values_in, keys_out, values_out, binary_pred=None):
    return check_u(lib.n_unique_by_key_copy(keys_in.m_cptr, values_in.m_cptr, keys_out.m_cptr, values_out.m_cptr,
                                            _p(binary_pred)))


def Partition(vec, pred):
    return check_u(lib.n_partition(vec.m_cptr, pred.m_cptr))


def Partition_Stencil(vec, stencil, pred):
    return check_u(lib.n_partition_stencil(vec.m_cptr, stencil.m_cptr, pred.m_cptr))


def Partition_Copy(vec_in, vec_true, vec_false, pred):
    return check_u(lib.n_partition_copy(vec_in.m_cptr, vec_true.m_cptr, vec_false.m_cptr, pred.m_cptr))


def Partition_Copy_Stencil(vec_in, stencil, vec_true, vec_false, pred):
    return check_u(lib.n_partition_copy_stencil(vec_in.m_cptr, stencil.m_cptr, vec_true.m_cptr, vec_false.m_cptr,
                                                pred.m_cptr))


# ---------------------------------------------------------------- transformations (Transformations.py)
def Fill(vec, value):
    check_i(lib.n_fill(vec.m_cptr, value.m_cptr))


def Replace(vec, old_value, new_value):
    check_i(lib.n_replace(vec.m_cptr, old_value.m_cptr, new_value.m_cptr))


def Replace_If(vec, pred, new_value):
    check_i(lib.n_replace_if(vec.m_cptr, pred.m_cptr, new_value.m_cptr))


def Replace_Copy(vec_in, vec_out, old_value, new_value):
    check_i(lib.n_replace_copy(vec_in.m_cptr, vec_out.m_cptr, old_value.m_cptr, new_value.m_cptr))


def Replace_Copy_If(vec_in, vec_out, pred, new_value):
    check_i(lib.n_replace_copy_if(vec_in.m_cptr, vec_out.m_cptr, pred.m_cptr, new_value.m_cptr))


def For_Each(vec, f):
    check_i(lib.n_for_each(vec.m_cptr, f.m_cptr))


def Adjacent_Difference(vec_in, vec_out, binary_op=None):
    check_i(lib.n_adjacent_difference(vec_in.m_cptr, vec_out.m_cptr, _p(binary_op)))


def Sequence(vec, value_init=None, value_step=None):
    check_i(lib.n_sequence(vec.m_cptr, _p(value_init), _p(value_step)))


def Tabulate(vec, op):
    check_i(lib.n_tabulate(vec.m_cptr, op.m_cptr))


def Transform(vec_in, vec_out, op):
    check_i(lib.n_transform(vec_in.m_cptr, vec_out.m_cptr, op.m_cptr))


def Transform_Binary(vec_in1, vec_in2, vec_out, op):
    check_i(lib.n_transform_binary(vec_in1.m_cptr, vec_in2.m_cptr, vec_out.m_cptr, op.m_cptr))


def Transform_If(vec_in, vec_out, op, pred):
    check_i(lib.n_transform_if(vec_in.m_cptr, vec_out.m_cptr, op.m_cptr, pred.m_cptr))


def Transform_If_Stencil(vec_in, vec_stencil, vec_out, op, pred):
    check_i(lib.n_transform_if_stencil(vec_in.m_cptr, vec_stencil.m_cptr, vec_out.m_cptr, op.m_cptr, pred.m_cptr))


def Transform_Binary_If_Stencil(vec_in1, vec_in2, vec_stencil, vec_out, op, pred):
    check_i(lib.n_transform_binary_if_stencil(vec_in1.m_cptr, vec_in2.m_cptr, vec_stencil.m_cptr, vec_out.m_cptr,
                                              op.m_cptr, pred.m_cptr))


# ---------------------------------------------------------------- copying (Copying.py)
def Gather(vec_map, vec_in, vec_out):
    check_i(lib.n_gather(vec_map.m_cptr, vec_in.m_cptr, vec_out.m_cptr))


def Gather_If(vec_map, vec_stencil, vec_in, vec_out, pred=None):
    check_i(lib.n_gather_if(vec_map.m_cptr, vec_stencil.m_cptr, vec_in.m_cptr, vec_out.m_cptr, _p(pred)))


def Scatter(vec_in, vec_map, vec_out):
    check_i(lib.n_scatter(vec_in.m_cptr, vec_map.m_cptr, vec_out.m_cptr))


def Scatter_If(vec_in, vec_map, vec_stencil, vec_out, pred=None):
    check_i(lib.n_scatter_if(vec_in.m_cptr, vec_map.m_cptr, vec_stencil.m_cptr, vec_out.m_cptr, _p(pred)))


def Swap(vec1, vec2):
    check_i(lib.n_swap(vec1.m_cptr, vec2.m_cptr))


# ---------------------------------------------------------------- reductions (Reductions.py)
def Count(vec, value):
    return check_ull(lib.n_count(vec.m_cptr, value.m_cptr))


def Count_If(vec, pred):
    return check_ull(lib.n_count_if(vec.m_cptr, pred.m_cptr))


def _bool(r):
    return check_i(r) != 0


def Equal(vec1, vec2, binary_pred=None):
    return _bool(lib.n_equal(vec1.m_cptr, vec2.m_cptr, _p(binary_pred)))


def Max_Element(vec, comp=None):
    return check_ull(lib.n_max_element(vec.m_cptr, _p(comp)))


def MinMax_Element(vec, comp=None):
    arr = np.zeros(2, dtype=np.uint64)
    check_i(lib.n_minmax_element(vec.m_cptr, _p(comp), arr.ctypes.data_as(ctypes.POINTER(u64))))
    return (arr[0], arr[1])


def Inner_Product(vec1, vec2, value_init, binary_op1=None, binary_op2=None):
    dvptr = check_cptr(lib.n_inner_product(vec1.m_cptr, vec2.m_cptr, value_init.m_cptr, _p(binary_op1),
                                           _p(binary_op2)))
    ret = _value_from_dvptr(dvptr)
    lib.n_dv_destroy(dvptr)
    return ret


def All_Of(vec, pred):
    return _bool(lib.n_all_of(vec.m_cptr, _p(pred)))


def Any_Of(vec, pred):
    return _bool(lib.n_any_of(vec.m_cptr, _p(pred)))


def None_Of(vec, pred):
    return _bool(lib.n_none_of(vec.m_cptr, _p(pred)))


def Is_Partitioned(vec, pred):
    return _bool(lib.n_is_partitioned(vec.m_cptr, pred.m_cptr))


def Is_Sorted(vec, comp=None):
    return _bool(lib.n_is_sorted(vec.m_cptr, _p(comp)))


# ---------------------------------------------------------------- searching (Searching.py)
def _index(r, size):
    r = check_i(r)
    return None if r >= size else r


def Find(vec, value):
    return _index(lib.n_find(vec.m_cptr, value.m_cptr), vec.size())


def Find_If(vec, pred):
    return _index(lib.n_find_if(vec.m_cptr, pred.m_cptr), vec.size())


def Find_If_Not(vec, pred):
    return _index(lib.n_find_if_not(vec.m_cptr, pred.m_cptr), vec.size())


def Mismatch(vec1, vec2, pred=None):
    r = check_i(lib.n_mismatch(vec1.m_cptr, vec2.m_cptr, _p(pred)))
    if r >= vec1.size() and r >= vec2.size():
        return None
    return r


def Partition_Point(vec, pred):
    return check_ull(lib.n_partition_point(vec.m_cptr, pred.m_cptr))


def Is_Sorted_Until(vec, comp=None):
    return check_ull(lib.n_is_sorted_until(vec.m_cptr, _p(comp)))


# ---------------------------------------------------------------- merging (Merging.py)
def Merge(vec1, vec2, vec_out, comp=None):
    check_i(lib.n_merge(vec1.m_cptr, vec2.m_cptr, vec_out.m_cptr, _p(comp)))


def Merge_By_Key(keys1, keys2, value1, value2, keys_out, value_out, comp=None):
    check_i(lib.n_merge_by_key(keys1.m_cptr, keys2.m_cptr, value1.m_cptr, value2.m_cptr, keys_out.m_cptr,
                               value_out.m_cptr, _p(comp)))


# ---------------------------------------------------------------- helper names of the reference package
# (utils.py:3-30, DeviceViewable.py:3-40): argument packers and the value reader
StrArray = _StrArray
ObjArray = _ObjArray
Dim3 = _Dim3
ValueFromDVPtr = _value_from_dvptr
