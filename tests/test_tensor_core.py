"""The tensor-core translation pass (tcgen05, TF32 hi/lo split) through the C ABI.

The pass applies the same operator as the rotation kernels, from dense
gentranmatrix records of every ordered pair; with three products per real
product it is accurate to FP32 level, so it is compared with the FP64 pass
at 1e-5 of the largest output (random columns over all orders make outputs
of 1e10 next to 1e-2; the hi/lo products carry about 2^-21 of each term),
for sphere orders whose mode blocks need padding (L = 7: 63 -> 64, L = 9: 99 -> 112) and one that does not (L = 8),
column counts inside one M tile and across two, and against the FP32
rotation kernel.  The T-matrix solve that runs its many-column passes on
the tensor cores must give the oracle's T matrix as the rotation path does.
"""
import numpy as np
import pytest

from mstm_b200 import configs as C

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _cluster(n, x, fv, seed, m):
    pos, _ = C.rsa_sphere(n, x, fv, seed=seed)
    return pos, np.full(n, x), np.full(n, m), -float(C.truncation_order(x))


@pytest.mark.parametrize("n,x,ncols", [(20, 1.0, 12), (24, 1.5, 40), (24, 1.5, 150), (16, 2.0, 33)])
def test_tensor_core_pass_matches_fp64(n, x, ncols):
    from mstm_b200 import api
    pos, rad, ri, em = _cluster(n, x, 0.15, 7, 1.5 + 0.02j)
    g = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="mixed")
    rng = np.random.default_rng(ncols)
    xx = rng.normal(size=(g.number_eqns, ncols)) + 1j * rng.normal(size=(g.number_eqns, ncols))
    y64 = g.translation_pass(xx, None, "fp64")
    ytc = g.translation_pass(xx, None, "tc")
    s = np.abs(y64).max()
    assert np.abs(ytc - y64).max() <= TOL * s, np.abs(ytc - y64).max() / s
    # and the FP32 rotation kernel on the same columns (a context without the tensor-core pass)
    r = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="mixed", tensor_core=-1)
    y32 = r.translation_pass(xx, None, "fp32")
    assert np.abs(ytc - y32).max() <= TOL * s
    # a second pass on the same context reuses the operator images
    ytc2 = g.translation_pass(2.0 * xx, None, "tc")
    assert np.abs(ytc2 - 2.0 * ytc).max() <= 1e-6 * s
    g.close()
    r.close()


def test_tensor_core_pass_after_new_positions():
    """Moving the spheres rebuilds the dense operators."""
    from mstm_b200 import api
    pos, rad, ri, em = _cluster(18, 1.5, 0.15, 8, 1.6 + 0.005j)
    g = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="mixed")
    rng = np.random.default_rng(2)
    xx = rng.normal(size=(g.number_eqns, 16)) + 1j * rng.normal(size=(g.number_eqns, 16))
    g.translation_pass(xx, None, "tc")
    pos2 = pos * 1.1
    g.set_positions(pos2)
    ytc = g.translation_pass(xx, None, "tc")
    y64 = g.translation_pass(xx, None, "fp64")
    assert np.abs(ytc - y64).max() <= TOL * np.abs(y64).max()
    g.close()


def test_tensor_core_pass_refuses_what_it_cannot_do():
    from mstm_b200 import api
    from mstm_b200._lib import MstmgError
    pos, rad, ri, em = _cluster(12, 1.0, 0.1, 3, 1.5 + 0.01j)
    g = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="mixed")
    xx = np.ones((g.number_eqns, 4), np.complex128)
    with pytest.raises(MstmgError):
        g.translation_pass(xx, [0, 1, 0, 1], "tc")    # conjugate-transpose columns
    off = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="mixed", tensor_core=-1)
    with pytest.raises(MstmgError):
        off.translation_pass(xx, None, "tc")
    g.close()
    off.close()


def test_tmatrix_on_tensor_cores_matches_oracle_and_rotation_path(oracle_mod):
    from mstm_b200 import api
    w = C.workload("cluster20")
    pos, rad, ri, em = w["pos"], w["radius"], w["ref_index"], -float(w["order"])
    o = oracle_mod.Oracle(pos, rad, ri, mie_eps=em, store_matrix=True, nthreads=8)
    ro = o.tmatrix_solution(convergence_eps=1e-6, solution_eps=1e-14)
    res = {}
    for tc in (0, -1):
        g = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="mixed", tensor_core=tc)
        T = g.t_matrix_order()
        res[tc] = g.tmatrix_solution(T, solution_eps=1e-14, convergence_eps=1e-6)
        g.close()
    for tc, rg in res.items():
        assert rg["istat"] == 0 and rg["order"] == ro["order"], tc
        assert np.allclose(rg["qtot"], ro["qtot"], rtol=1e-6), tc
        assert np.abs(rg["tmat"] - ro["tmat"]).max() <= 1e-6 * np.abs(ro["tmat"]).max(), tc
