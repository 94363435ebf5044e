"""ctypes binding of the reference's own kernels compiled for the CPU (``oracle/_ref``).

TEST INFRASTRUCTURE ONLY (oracle).  Used by the golden-vector generator (through a
numpy-backed stand-in for pycuda) and by ``bench.py``'s CPU reference arm.  The
product never imports this module.

``load()`` returns a :class:`RefKernels` whose attributes are callables with the
pycuda calling convention of the reference (mainPropElastic3D_MT.py:518-530)::

    k = load()
    k.kernel_Tau(Tauxx, ..., np.float32(dx), ..., np.int32(nz), grid=(gx, gy, gz), block=(32, 2, 4))

Array arguments are numpy arrays (C-contiguous, float32 / int32) or objects with a
``.arr`` numpy attribute.
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_CT = {"float*": ctypes.c_void_p, "int*": ctypes.c_void_p, "float": ctypes.c_float,
       "int": ctypes.c_int}


class RefKernels:
    def __init__(self, lib_path: str, sig_path: str, parallel: bool = True):
        self.lib = ctypes.CDLL(lib_path)
        with open(sig_path) as f:
            self.signatures = json.load(f)
        with open(os.path.join(os.path.dirname(lib_path), "kernels.sha256")) as f:
            self.sha256 = f.read().strip()
        self.parallel = parallel
        for name, params in self.signatures.items():
            fn = getattr(self.lib, "ref_" + name)
            fn.restype = None
            fn.argtypes = ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
                           + [_CT[t] for t, _ in params])
            setattr(self, name, self._make_caller(name, fn, params))

    def _make_caller(self, name, fn, params):
        def call(*args, grid, block, **_unused):
            if len(args) != len(params):
                raise TypeError(f"{name}: expected {len(params)} args, got {len(args)}")
            conv = []
            keep = []
            for (t, pname), a in zip(params, args):
                if t.endswith("*"):
                    arr = getattr(a, "arr", a)
                    want = np.float32 if t == "float*" else np.int32
                    if not isinstance(arr, np.ndarray) or arr.dtype != want \
                            or not arr.flags.c_contiguous:
                        raise TypeError(f"{name}.{pname}: need C-contiguous {want.__name__} array")
                    keep.append(arr)
                    conv.append(arr.ctypes.data)
                elif t == "float":
                    conv.append(float(np.float32(a)))
                else:
                    conv.append(int(a))
            g = (ctypes.c_uint * 3)(*[int(v) for v in (tuple(grid) + (1, 1, 1))[:3]])
            b = (ctypes.c_uint * 3)(*[int(v) for v in (tuple(block) + (1, 1, 1))[:3]])
            fn(g, b, 1 if self.parallel else 0, *conv)
        call.__name__ = name
        return call


def available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "librefkern.so"))


def load(parallel: bool = True) -> RefKernels:
    so = os.path.join(REF_DIR, "librefkern.so")
    if not os.path.exists(so):
        raise FileNotFoundError(
            "oracle/_ref/librefkern.so is missing; build it with `python oracle/build_ref.py` "
            "where the reference tree is present")
    return RefKernels(so, os.path.join(REF_DIR, "signatures.json"), parallel=parallel)
