"""The oracle behind a ThrustRTC-shaped Python API (test infrastructure).

Lets tests/golden/ref_cases.py run on the CPU oracle exactly as it runs on the reference
package and on thrustrtc_b200, so the oracle is checked against the reference's recorded
outputs case by case.  Vectors are numpy arrays; only the functors the cases use exist.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import oracle as O  # noqa: E402

_NP = {"int8_t": np.int8, "uint8_t": np.uint8, "int16_t": np.int16, "uint16_t": np.uint16, "int32_t": np.int32,
       "uint32_t": np.uint32, "int64_t": np.int64, "uint64_t": np.uint64, "float": np.float32, "double": np.float64}


class Vec:
    def __init__(self, a):
        self.a = a

    def to_host(self, begin=0, end=-1):
        return (self.a[begin:] if end == -1 else self.a[begin:end]).copy()


def device_vector_from_numpy(a):
    return Vec(np.array(a, copy=True))


def device_vector(elem_cls, n):
    return Vec(np.zeros(n, dtype=_NP[elem_cls]))


class _Scalar:
    def __init__(self, v):
        self.v = v


DVInt32 = _Scalar


class _Op:
    def __init__(self, name):
        self.name = name


def Greater():
    return _Op("Greater")


def Plus():
    return _Op("Plus")


def Maximum():
    return _Op("Maximum")


def EqualTo():
    return _Op("EqualTo")


def Negate():
    return _Op("Negate")


class Functor:
    """Only the predicates the cases use: ``x % 2 == 0`` and ``(x & 1) != 0``."""

    def __init__(self, arg_map, params, body):
        b = body.replace(" ", "")
        if "x%2==0" in b:
            self.f = lambda x: (x % 2) == 0
        elif "(x&1)!=0" in b:
            self.f = lambda x: (x & 1) != 0
        else:
            raise NotImplementedError(body)


def _opname(op):
    return "Plus" if op is None else op.name


def Sort(v, comp=None):
    v.a[:] = O.sort(v.a, descending=comp is not None and comp.name == "Greater")


def Sort_By_Key(k, v, comp=None):
    ko, vo = O.sort_by_key(k.a, v.a, descending=comp is not None and comp.name == "Greater")
    k.a[:], v.a[:] = ko, vo


def Min_Element(v, comp=None):
    return O.min_element(v.a)


def Inclusive_Scan(i, o, op=None):
    o.a[:] = O.scan(i.a, _opname(op))


def Exclusive_Scan(i, o, init=None, op=None):
    o.a[:] = O.scan(i.a, _opname(op), exclusive=True, init=None if init is None else init.v)


def _unary(u, x):
    assert u.name == "Negate"
    return (-x.astype(np.int64)).astype(x.dtype)


def Transform_Inclusive_Scan(i, o, u, op):
    o.a[:] = O.scan(_unary(u, i.a), _opname(op))


def Transform_Exclusive_Scan(i, o, u, init, op):
    o.a[:] = O.scan(_unary(u, i.a), _opname(op), exclusive=True, init=init.v)


def Inclusive_Scan_By_Key(k, v, o, pred=None, op=None):
    o.a[:] = O.scan_by_key(k.a, v.a, _opname(op))


def Exclusive_Scan_By_Key(k, v, o, init=None, pred=None, op=None):
    o.a[:] = O.scan_by_key(k.a, v.a, _opname(op), exclusive=True, init=0 if init is None else init.v)


def _put(o, x):
    o.a[:len(x)] = x
    return len(x)


def Copy_If(i, o, pred):
    return _put(o, O.copy_if(i.a, pred.f(i.a)))


def Copy_If_Stencil(i, s, o, pred):
    return _put(o, O.copy_if(i.a, pred.f(s.a)))


def Partition(v, pred):
    v.a[:], c = O.partition(v.a, pred.f(v.a))
    return c


def Partition_Stencil(v, s, pred):
    v.a[:], c = O.partition(v.a, pred.f(s.a))
    return c


def Partition_Copy(i, t, f, pred):
    fl = pred.f(i.a)
    _put(f, i.a[~fl])
    return _put(t, i.a[fl])


def Partition_Copy_Stencil(i, s, t, f, pred):
    fl = pred.f(s.a)
    _put(f, i.a[~fl])
    return _put(t, i.a[fl])


def Remove_If(v, pred):
    return _put(v, O.copy_if(v.a, ~pred.f(v.a)))


def Remove_Copy_If(i, o, pred):
    return _put(o, O.copy_if(i.a, ~pred.f(i.a)))


def Remove_If_Stencil(v, s, pred):
    return _put(v, O.copy_if(v.a, ~pred.f(s.a)))


def Remove_Copy_If_Stencil(i, s, o, pred):
    return _put(o, O.copy_if(i.a, ~pred.f(s.a)))


def Remove(v, value):
    return _put(v, O.copy_if(v.a, O.remove_flags(v.a, value.v)))


def Remove_Copy(i, o, value):
    return _put(o, O.copy_if(i.a, O.remove_flags(i.a, value.v)))


def Unique(v, pred=None):
    return _put(v, O.copy_if(v.a, O.unique_flags(v.a)))


def Unique_Copy(i, o, pred=None):
    return _put(o, O.copy_if(i.a, O.unique_flags(i.a)))


def Unique_By_Key(k, v, pred=None):
    f = O.unique_flags(k.a)
    _put(v, v.a[:len(k.a)][f])
    return _put(k, k.a[f])


def Unique_By_Key_Copy(ki, vi, ko, vo, pred=None):
    f = O.unique_flags(ki.a)
    _put(vo, vi.a[:len(ki.a)][f])
    return _put(ko, ki.a[f])


def Reduce_By_Key(ki, vi, ko, vo, pred=None, op=None):
    k, s = O.reduce_by_key(ki.a, vi.a, _opname(op))
    _put(vo, s)
    return _put(ko, k)


def Reduce(v, init=None, op=None):
    r = O.reduce(v.a, None if init is None else init.v, _opname(op))
    return r.item() if hasattr(r, "item") else r
