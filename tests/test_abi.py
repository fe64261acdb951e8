"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(mstmg_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ["mstmg_ctx_create", "mstmg_ctx_destroy", "mstmg_interaction", "mstmg_bicg", "mstmg_fixed_orientation",
              "mstmg_planewave"]:
        assert n in names


def test_library_exports_all_declared_symbols():
    from mstm_b200 import _lib
    from mstm_b200 import build as B
    if not os.path.exists(_lib.LIB_PATH):
        B.build()
    L = _lib.lib()
    for n in declared_symbols():
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, n


def test_missing_library_fails_loudly(monkeypatch):
    from mstm_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libmstm_b200.so")
    with pytest.raises(RuntimeError):
        _lib.lib()


@pytest.mark.parametrize("bad", ["nan_position", "inf_index", "zero_radius"])
def test_ctx_create_rejects_invalid_host_inputs(bad):
    """Non-finite positions or indices and non-positive radii are rejected with
    MSTMG_ERR_ARG before anything reaches a GPU (runs on a machine without one)."""
    import ctypes

    import numpy as np

    from mstm_b200 import _lib
    from mstm_b200 import build as B
    if not os.path.exists(_lib.LIB_PATH):
        B.build()
    L = _lib.lib()
    pos = np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0]])
    rad = np.array([1.0, 1.0])
    ri = np.array([[1.5, 0.01], [1.5, 0.01]])
    if bad == "nan_position":
        pos[1, 2] = np.nan
    elif bad == "inf_index":
        ri[0, 1] = np.inf
    else:
        rad[1] = 0.0
    ctx = ctypes.c_void_p()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.mstmg_ctx_create(ctypes.byref(ctx), 2, p(pos), p(rad), p(ri), -3.0, None)
    assert rc == -1 and not ctx.value
    msg = L.mstmg_last_error().decode()
    assert ("sphere 2" if bad != "inf_index" else "sphere 1") in msg


@pytest.mark.parametrize("field,value", [("gmres_restart", -1), ("mixed_solver", 3)])
def test_ctx_create_rejects_invalid_solver_options(field, value):
    """Out-of-range solver options are rejected with MSTMG_ERR_ARG before any
    device call (runs on a machine without a GPU)."""
    import ctypes

    import numpy as np

    from mstm_b200 import _lib
    from mstm_b200 import build as B
    if not os.path.exists(_lib.LIB_PATH):
        B.build()
    L = _lib.lib()
    opts = _lib.MstmgOpts()
    L.mstmg_default_opts(ctypes.byref(opts))
    assert opts.mixed_solver == 2 and opts.gmres_restart == 0
    setattr(opts, field, value)
    pos = np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0]])
    rad = np.array([1.0, 1.0])
    ri = np.array([[1.5, 0.01], [1.5, 0.01]])
    ctx = ctypes.c_void_p()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.mstmg_ctx_create(ctypes.byref(ctx), 2, p(pos), p(rad), p(ri), -3.0, ctypes.byref(opts))
    assert rc == -1 and not ctx.value
    assert "gmres_restart" in L.mstmg_last_error().decode()


@pytest.mark.parametrize("starts", [[1, 2, 4], [0, 2, 3], [0, 2, 2, 4]])
def test_ensemble_create_rejects_bad_config_start(starts):
    """config_start must run from 0 to nsphere with every configuration
    non-empty; checked before any device call."""
    import ctypes

    import numpy as np

    from mstm_b200 import _lib
    from mstm_b200 import build as B
    if not os.path.exists(_lib.LIB_PATH):
        B.build()
    L = _lib.lib()
    pos = np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0], [0.0, 3.0, 0.0], [0.0, 0.0, 3.0]])
    rad = np.ones(4)
    ri = np.tile([1.5, 0.01], (4, 1))
    cs = np.array(starts, np.int32)
    ctx = ctypes.c_void_p()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.mstmg_ensemble_create(ctypes.byref(ctx), len(starts) - 1, p(cs), 4, p(pos), p(rad), p(ri), -3.0, None)
    assert rc == -1 and not ctx.value
    assert "mstmg_ensemble_create" in L.mstmg_last_error().decode()
