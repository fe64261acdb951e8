"""mstmg_planewave_noalloc: the incident-field coefficients for callers that
cannot allocate device memory (a host code that owns every device buffer, or
one held to a fixed device-memory budget).  It must reproduce mstmg_planewave,
the context-based entry point, on consecutive calls that share its built-in
scratch array.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_planewave_noalloc_matches_context_entry_point():
    import torch
    from mstm_b200 import _lib, api, configs
    L = _lib.lib()
    w = configs.workload("cluster20")
    g = api.SphereCluster(w["pos"], w["radius"], w["ref_index"], mie_epsilon=-w["order"])
    order = int(g.sphere_order[0])
    n = len(w["pos"])
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(np.ascontiguousarray(w["pos"], dtype=np.float64)).to(dev)
    out_d = torch.zeros(2 * g.number_eqns * 2, dtype=torch.float64, device=dev)
    # two calls in a row with different incidence: the second must not see the first's tables
    for alpha, sinc in [(0.7, 0.4), (0.0, 0.0)]:
        ref = g.sphereplanewavecoef(alpha, sinc, 1)
        out_d.zero_()
        torch.cuda.synchronize()
        rc = L.mstmg_planewave_noalloc(n, order, ctypes.c_void_p(pos_d.data_ptr()), alpha, sinc, 1,
                                       ctypes.c_void_p(out_d.data_ptr()), None)
        assert rc == 0, L.mstmg_last_error()
        torch.cuda.synchronize()
        got = out_d.cpu().numpy().view(np.complex128).reshape(2, -1).T
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    g.close()


def test_planewave_noalloc_rejects_what_it_cannot_hold():
    import torch
    from mstm_b200 import _lib
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    pos_d = torch.zeros(3, dtype=torch.float64, device=dev)
    out_d = torch.zeros(2 * 2 * 17 * 19 * 2, dtype=torch.float64, device=dev)
    rc = L.mstmg_planewave_noalloc(1, 17, ctypes.c_void_p(pos_d.data_ptr()), 0.0, 0.0, 1, ctypes.c_void_p(out_d.data_ptr()), None)
    assert rc == -3 and b"scratch limit" in L.mstmg_last_error()
    host = np.zeros(3)
    rc = L.mstmg_planewave_noalloc(1, 7, host.ctypes.data_as(ctypes.c_void_p), 0.0, 0.0, 1,
                                   ctypes.c_void_p(out_d.data_ptr()), None)
    assert rc == -1
