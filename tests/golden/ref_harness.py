"""Import the reference module itself on a CPU-only machine, for golden vectors.

FIXTURE-GENERATION INFRASTRUCTURE ONLY.  Used by ``make_golden.py`` in a container that
has the reference tree; never used by the product, the GPU tests or the bench.

The reference (``mainPropElastic3D_MT.py``) imports pycuda and mpi4py at module level
and JIT-compiles its kernels through ``pycuda.compiler.SourceModule``.  Neither package
exists here, so this module installs small stand-ins before the import:

* ``pycuda.gpuarray.GPUArray`` is a numpy array holder (``to_gpu``/``get``/``astype``
  and the scalar ``+=`` the reference's ``addSource`` performs, done in float32 as
  pycuda's ``axpbz`` kernel does).
* ``pycuda.compiler.SourceModule`` checks that the string it receives is byte-for-byte
  the kernel string compiled by ``oracle/build_ref.py`` and hands out those compiled
  CPU kernels (``oracle/refkern.py``).
* ``mpi4py.MPI.COMM_WORLD`` is a single rank (rank 0, size 1).
* ``matplotlib``/``imageio`` become no-op stubs (the reference plots interactively).

Everything else -- the driver classes, time loops, residual, misfit, L-BFGS, line
search, gradient post-processing -- is the reference's own Python code.
"""
from __future__ import annotations

import hashlib
import importlib
import os
import sys
import types

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_DIR = os.environ.get("EFM_REFERENCE_DIR", "/root/reference/Elastic3DGPU_MT_VP_VS_RHO_MPI")


# --------------------------------------------------------------------------- stubs
class _Anything:
    """Absorbs any attribute access or call (plot stubs)."""

    def __getattr__(self, name):
        return _Anything()

    def __call__(self, *a, **k):
        return _Anything()

    def __iter__(self):
        return iter(())


def _stub_module(name):
    mod = types.ModuleType(name)
    mod.__getattr__ = lambda attr: _Anything()  # type: ignore[attr-defined]
    return mod


class GPUArray:
    """numpy-backed stand-in for ``pycuda.gpuarray.GPUArray``."""

    def __init__(self, arr):
        self.arr = np.ascontiguousarray(arr)

    # pycuda API used by the reference
    def get(self):
        return self.arr.copy()

    def astype(self, dtype):
        return GPUArray(self.arr.astype(dtype))

    @property
    def shape(self):
        return self.arr.shape

    @property
    def dtype(self):
        return self.arr.dtype

    def __len__(self):
        return len(self.arr)

    def __getitem__(self, key):
        return _ElementRef(self.arr, key)

    def __setitem__(self, key, value):
        if isinstance(value, _ElementRef) and value.base is self.arr and value.key == key:
            return
        self.arr[key] = getattr(value, "arr", value)

    def __reduce__(self):
        return (GPUArray, (self.arr,))


class _ElementRef:
    """Result of ``gpuarray[y, z, x]``; supports the in-place scalar add of addSource."""

    def __init__(self, base, key):
        self.base, self.key = base, key

    def __iadd__(self, other):
        # pycuda: x += b runs z = a*x + b with a, b cast to the array dtype (float32)
        t = self.base.dtype.type
        b = t(np.asarray(other).reshape(-1)[0])
        self.base[self.key] = t(self.base[self.key]) + b
        return self

    def get(self):
        return np.array(self.base[self.key])


def _to_gpu(a):
    return GPUArray(np.array(a))


class _Context:
    def push(self):
        pass

    def pop(self):
        pass

    def detach(self):
        pass


class _Device:
    def __init__(self, i):
        self.i = i

    def make_context(self):
        return _Context()

    @staticmethod
    def count():
        return 1


class _SourceModule:
    def __init__(self, src, *a, **k):
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        try:
            import refkern
        finally:
            sys.path.pop(0)
        self._k = refkern.load(parallel=True)
        if hashlib.sha256(src.encode()).hexdigest() != self._k.sha256:
            raise RuntimeError("reference kernel string differs from the compiled oracle/_ref library")

    def get_function(self, name):
        return getattr(self._k, name)


class _Comm:
    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def Barrier(self):
        pass

    def bcast(self, obj, root=0):
        return obj

    def reduce(self, obj, op=None, root=0):
        return obj

    def send(self, *a, **k):
        raise RuntimeError("single-rank stand-in: send")

    def recv(self, *a, **k):
        raise RuntimeError("single-rank stand-in: recv")

    Send = send
    Recv = recv


def install():
    """Register the stand-in modules in ``sys.modules``."""
    pycuda = types.ModuleType("pycuda")
    autoinit = types.ModuleType("pycuda.autoinit")
    driver = types.ModuleType("pycuda.driver")
    driver.init = lambda: None
    driver.Device = _Device
    gpuarray = types.ModuleType("pycuda.gpuarray")
    gpuarray.GPUArray = GPUArray
    gpuarray.to_gpu = _to_gpu
    compiler = types.ModuleType("pycuda.compiler")
    compiler.SourceModule = _SourceModule
    pycuda.autoinit, pycuda.driver, pycuda.gpuarray, pycuda.compiler = autoinit, driver, gpuarray, compiler
    mpi4py = types.ModuleType("mpi4py")
    MPI = types.ModuleType("mpi4py.MPI")
    MPI.COMM_WORLD = _Comm()
    MPI.SUM = "SUM"
    MPI.FLOAT = "FLOAT"
    mpi4py.MPI = MPI
    mpl = _stub_module("matplotlib")
    plt = _stub_module("matplotlib.pyplot")
    mpl.pyplot = plt
    mods = {
        "pycuda": pycuda, "pycuda.autoinit": autoinit, "pycuda.driver": driver,
        "pycuda.gpuarray": gpuarray, "pycuda.compiler": compiler,
        "mpi4py": mpi4py, "mpi4py.MPI": MPI,
        "matplotlib": mpl, "matplotlib.pyplot": plt, "imageio": _stub_module("imageio"),
    }
    for k, v in mods.items():
        sys.modules.setdefault(k, v)


def import_reference():
    """Import ``mainPropElastic3D_MT`` and ``lbfgs`` from the reference tree."""
    install()
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    main = importlib.import_module("mainPropElastic3D_MT")
    lbfgs = importlib.import_module("lbfgs")
    return main, lbfgs


def set_globals(main, **kw):
    """Define the module globals the reference's classes read (mainPropElastic3D_MT.py:2743-2766)."""
    defaults = dict(threadBlockX=32, threadBlockY=2, threadBlockZ=4, H_STENCIL=2, SrcIdx=0,
                    rank=0, sizeRank=1, corte=0)
    defaults.update(kw)
    for k, v in defaults.items():
        setattr(main, k, v)
