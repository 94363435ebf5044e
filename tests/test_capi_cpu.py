"""C-ABI library checks that need no GPU: it builds, loads, exports every symbol that
include/efm.h declares, and rejects bad arguments with a status code (never a crash)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO


def _declared_symbols():
    with open(os.path.join(REPO, "include", "efm.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"EFM_API\s+[\w\s\*]+?\b(efm_\w+)\s*\(", text)))


def test_header_declares_the_api():
    syms = _declared_symbols()
    for s in ("efm_create", "efm_forward", "efm_gradient", "efm_residual_misfit",
              "efm_lbfgs_history", "efm_lbfgs_direction", "efm_smooth_mask"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from elastic_fm_vp_vs_rho_b200 import _lib
    L = _lib.load()
    for s in _declared_symbols():
        assert hasattr(L, s), s
    assert set(_lib.SIGNATURES) == set(_declared_symbols())


def test_library_is_built_for_sm100a():
    from elastic_fm_vp_vs_rho_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)
    assert os.path.exists(build.LIB)


def test_argument_errors_return_status():
    from elastic_fm_vp_vs_rho_b200 import _lib
    L = _lib.load()
    ctx = ctypes.c_void_p()
    assert L.efm_create(ctypes.byref(ctx)) == _lib.EFM_OK
    try:
        d = _lib.InstanceDesc(nx=8, ny=8, nz=8, lenpml=10, dx=1.0, dt=1e-3, nt=10, nsrc=1, nrec=1)
        rc = L.efm_add_instance(ctx, ctypes.byref(d), None)
        assert rc == _lib.EFM_ERR_ARG
        assert b"CPML" in L.efm_last_error() or b"small" in L.efm_last_error()
        cp = np.zeros(2 * (40 + 40 + 40), np.float32)
        src = np.array([1, 20, 20], np.int32)  # x = 1 is outside the updated interior
        mt = np.zeros(6, np.float32)
        rec = np.array([20, 20, 2], np.int32)
        d = _lib.InstanceDesc(nx=40, ny=40, nz=40, lenpml=10, dx=1.0, dt=1e-3, nt=10,
                              cpml_host=cp.ctypes.data, nsrc=1, src_host=src.ctypes.data,
                              mt_host=mt.ctypes.data, nrec=1, rec_host=rec.ctypes.data)
        assert L.efm_add_instance(ctx, ctypes.byref(d), None) == _lib.EFM_ERR_ARG
        assert b"source" in L.efm_last_error()
        # no instances: a forward is a state error, not a crash
        assert L.efm_forward(ctx, None, 0, None) != _lib.EFM_OK
        assert L.efm_num_instances(ctx) == 0
        assert L.efm_set_option(ctx, _lib.EFM_OPT_WAIT_LIMIT, -1) == _lib.EFM_ERR_ARG
        assert L.efm_set_option(ctx, _lib.EFM_OPT_WAIT_LIMIT, 4) == _lib.EFM_OK
        assert L.efm_set_option(ctx, _lib.EFM_OPT_WAIT_LIMIT, 0) == _lib.EFM_OK
        assert L.efm_set_option(ctx, _lib.EFM_OPT_EXACT_FORM, 3) == _lib.EFM_ERR_ARG
        for form in (_lib.EFM_EXACT_TWO_PASS, _lib.EFM_EXACT_GATHER, _lib.EFM_EXACT_STREAM):
            assert L.efm_set_option(ctx, _lib.EFM_OPT_EXACT_FORM, form) == _lib.EFM_OK
        assert L.efm_set_option(ctx, _lib.EFM_OPT_CHECKPOINT_EVERY, -1) == _lib.EFM_ERR_ARG
        assert L.efm_set_option(ctx, _lib.EFM_OPT_CHECKPOINT_EVERY, 0) == _lib.EFM_OK  # automatic
        assert L.efm_set_option(ctx, _lib.EFM_OPT_CHECKPOINT_EVERY, 25) == _lib.EFM_OK
        assert L.efm_smooth_mask(None, None, 1, 1, 1, 1.0, 0, 0, None) == _lib.EFM_ERR_ARG
        assert L.efm_lbfgs_history(None, None, None, None, 1, 0, 0, None) == _lib.EFM_ERR_ARG
    finally:
        L.efm_destroy(ctx)


def test_error_raises_efm_error():
    from elastic_fm_vp_vs_rho_b200 import _lib
    with pytest.raises(_lib.EfmError) as e:
        _lib.check(_lib.load().efm_smooth_mask(None, None, 0, 0, 0, 1.0, 0, 0, None))
    assert e.value.code == _lib.EFM_ERR_ARG
