"""mstmg_planewave_noalloc: the incident-field coefficients for callers that
cannot allocate device memory (a host code that owns every device buffer, or
one held to a fixed device-memory budget).  It must reproduce mstmg_planewave,
the context-based entry point, on consecutive calls that share its built-in
scratch array, and must leave the device's free memory unchanged.  This file
is collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(L, n, order, pos_d, alpha, sinc, direction, out_d, stream=None):
    return L.mstmg_planewave_noalloc(n, order, ctypes.c_void_p(pos_d.data_ptr()), alpha, sinc, direction,
                                     ctypes.c_void_p(out_d.data_ptr()), stream)


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
    # calls in a row with different incidence and direction: none may see the previous call's tables
    for alpha, sinc, direction in [(0.7, 0.4, 1), (0.0, 0.0, 1), (1.1, 0.6, 2), (0.0, 0.0, 2)]:
        ref = g.sphereplanewavecoef(alpha, sinc, direction)
        out_d.zero_()
        torch.cuda.synchronize()
        rc = _noalloc(L, n, order, pos_d, alpha, sinc, direction, out_d)
        assert rc == 0, L.mstmg_last_error()
        torch.cuda.synchronize()
        got = out_d.cpu().numpy().view(np.complex128).reshape(2, -1).T
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    g.close()


def test_planewave_noalloc_largest_order_on_a_stream_allocates_nothing():
    import torch
    from mstm_b200 import _lib, api
    L = _lib.lib()
    n, order = 3, 16
    pos = np.array([[0.0, 0.0, 0.0], [2.5, 0.4, -0.3], [-0.6, 2.7, 1.1]])
    g = api.SphereCluster(pos, np.full(n, 1.0), np.full(n, 1.4 + 0.01j), mie_epsilon=-order)
    assert int(g.sphere_order[0]) == order
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(np.ascontiguousarray(pos, dtype=np.float64)).to(dev)
    out_d = torch.zeros(2 * g.number_eqns * 2, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    # the first call may load the library's device module; measure after it
    assert _noalloc(L, n, order, pos_d, 0.3, 0.2, 1, out_d, sp) == 0, L.mstmg_last_error()
    stream.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for alpha, sinc, direction in [(0.3, 0.2, 1), (0.9, 0.5, 2)]:
        ref = g.sphereplanewavecoef(alpha, sinc, direction)
        stream.synchronize()
        assert _noalloc(L, n, order, pos_d, alpha, sinc, direction, out_d, sp) == 0, L.mstmg_last_error()
        stream.synchronize()
        got = out_d.cpu().numpy().view(np.complex128).reshape(2, -1).T
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    for _ in range(5):
        assert _noalloc(L, n, order, pos_d, 0.1, 0.1, 1, out_d, sp) == 0
    stream.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    g.close()


def test_planewave_noalloc_rejects_what_it_cannot_hold():
    import torch
    from mstm_b200 import _lib
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    pos_d = torch.zeros(3, dtype=torch.float64, device=dev)
    out_d = torch.zeros(2 * 2 * 17 * 19 * 2, dtype=torch.float64, device=dev)
    rc = _noalloc(L, 1, 17, pos_d, 0.0, 0.0, 1, out_d)
    assert rc == -3 and b"scratch limit" in L.mstmg_last_error()
    host = np.zeros(3)
    rc = L.mstmg_planewave_noalloc(1, 7, host.ctypes.data_as(ctypes.c_void_p), 0.0, 0.0, 1,
                                   ctypes.c_void_p(out_d.data_ptr()), None)
    assert rc == -1
