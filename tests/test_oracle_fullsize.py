"""The benchmark workloads at full size against the oracle's frozen results.

tests/golden/oracle_*.npz hold the oracle's FP64 solutions of the very
configurations the benchmark solves (made by tests/golden/make_oracle_fixtures.py,
minutes of CPU time each):
  fractal500     500-monomer aggregate, x = 2 (L = 9, 99,000 unknowns), both
                 polarisations to ||r||^2/||b||^2 < 1e-12, plus the
                 azimuth-averaged scattering matrix at 181 angles and g;
  cylinder_fft   5000 spheres on the FFT translation path (630,000 unknowns);
  tmatrix100     100-sphere cluster T matrix (x = 1.5, 720 columns at order 18)
                 and its orientation averages;
  ensemble_tmatrix_c*  the two smallest configurations of the 256-configuration
                 T-matrix ensemble;
  host1000       a host sphere holding 1000 inclusions (host spheres, FP64).
Tolerances (stated per output): the FP64 drop-in path follows the reference's
iteration, so 1e-9 relative on efficiencies, solutions and the scattering
matrix (of its largest element); the mixed path and the tensor-core T-matrix
passes 1e-6 relative on efficiencies and 1e-4 on scattering-matrix elements
(of S11's largest value); the FFT path (its kernel spectra are single
precision, the oracle sums node translations directly) 1e-6 on efficiencies.
The CPU tests check the fixtures themselves: they belong to the seeded
configurations the generators make, and they are converged.
"""
import os

import numpy as np
import pytest

from mstm_b200 import configs as C

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLD, "oracle_%s.npz" % name)))


def _ensemble_cfgs():
    from mstm_b200 import ensemble as EN
    cfgs = EN.ensemble_configs(256, seed=4, nmin=50, nmax=400)
    small = sorted(range(len(cfgs)), key=lambda k: (cfgs[k]["n"], k))[:2]
    return [(k, cfgs[k]) for k in small]


# ---------------------------------------------------------------------------
# CPU: the fixtures belong to the generators' configurations and converged
# ---------------------------------------------------------------------------
def test_fixtures_match_the_seeded_configurations():
    f = _load("fractal500")
    assert np.array_equal(f["pos"], C.workload("fractal500")["pos"])
    assert f["status"] == 0 and f["maxerr"] < 1e-12 and list(f["iterations"]) == [79, 78]
    assert abs(f["qtot"][2, 0] - (f["qtot"][0, 0] - f["qtot"][1, 0])) < 1e-3 * f["qtot"][0, 0]
    cyl = _load("cylinder_fft")
    assert np.array_equal(cyl["pos"], C.rsa_cylinder(5000, 1.0, 0.25, 1.0, seed=3)[0])
    assert cyl["status"] == 0 and cyl["maxerr"] < 1e-12 and list(cyl["cell_dim"]) == [12, 12, 12]
    t = _load("tmatrix100")
    assert np.array_equal(t["pos"], C.rsa_sphere(100, 1.5, 0.20, seed=4)[0])
    assert t["status"] == 0 and t["order_used"] == 18 and t["t_matrix_order"] == 24
    assert abs(t["qext_t"] / t["qtot"][0] - 1) < 1e-6
    for k, cfg in _ensemble_cfgs():
        e = _load("ensemble_tmatrix_c%d" % k)
        assert np.array_equal(e["pos"], cfg["pos"]) and e["status"] == 0
    h = _load("host1000")
    w = C.host_inclusions(1000, 0.5, 0.15, seed=7)
    assert np.array_equal(h["pos"], w["pos"]) and np.array_equal(h["radius"], w["radius"])
    assert h["status"] == 0 and h["maxerr"] < 1e-12 and h["order"][0] == 12


# ---------------------------------------------------------------------------
# GPU against the fixtures
# ---------------------------------------------------------------------------
def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fractal500_against_oracle(precision):
    from mstm_b200 import api
    f = _load("fractal500")
    n = len(f["pos"])
    g = api.SphereCluster(f["pos"], np.full(n, 2.0), np.full(n, 1.6 + 0.05j), mie_epsilon=-9, precision=precision)
    r = g.fixedorsoln(eps=1e-12, niter=10000)
    s = g.scattering(r["amnp"])
    s11 = np.abs(f["smat"][:, 0, 0]).max()
    off = g.sphere_offset
    norms = np.array([[np.linalg.norm(r["amnp"][off[i]:off[i + 1], p]) for p in range(2)] for i in range(n)])
    assert s["t_matrix_order"] == f["t_matrix_order"]
    if precision == "fp64":
        assert list(r["iterations"]) == list(f["iterations"])
        assert _rel(r["qtot"], f["qtot"]) <= 1e-9
        assert _rel(r["qeff"], f["qeff"]) <= 1e-9
        assert _rel(norms, f["sphere_norms"]) <= 1e-9
        assert _rel(r["amnp"][:off[4]], f["amnp_head"]) <= 1e-9
        assert np.abs(s["smat"] - f["smat"]).max() <= 1e-9 * s11
        assert abs(s["g"] - f["g"]) <= 1e-9 * abs(f["g"])
    else:
        assert r["maxerr"] < 1e-12
        assert np.allclose(r["qtot"], f["qtot"], rtol=1e-6)
        assert _rel(norms, f["sphere_norms"]) <= 1e-5
        assert np.abs(s["smat"] - f["smat"]).max() <= 1e-4 * s11
        assert abs(s["g"] - f["g"]) <= 1e-6 * abs(f["g"])
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cylinder5000_fft_against_oracle(precision):
    from mstm_b200 import api
    f = _load("cylinder_fft")
    n = len(f["pos"])
    g = api.SphereCluster(f["pos"], np.full(n, 1.0), np.full(n, 1.31 + 0j), mie_epsilon=-7, precision=precision)
    grid = g.fft_setup(d_cell=4.0)
    assert list(grid["cell_dim"]) == list(f["cell_dim"]) and grid["near_pairs"] == f["near_pairs"]
    assert grid["node_order"] == f["node_order"]
    r = g.fixedorsoln(eps=1e-12, niter=10000)
    assert r["maxerr"] < 1e-12
    assert np.allclose(r["qtot"], f["qtot"], rtol=1e-6)
    s = g.scattering(r["amnp"])
    assert np.abs(s["smat"] - f["smat"]).max() <= 1e-4 * np.abs(f["smat"][:, 0, 0]).max()
    g.close()


def _tmatrix_check(g, f, tol_q, tol_t):
    T = g.t_matrix_order()
    assert T == f["t_matrix_order"]
    r = g.tmatrix_solution(T, solution_eps=1e-12, convergence_eps=1e-6)
    assert r["istat"] == 0 and r["order"] == f["order_used"]
    u = r["order"]
    nb = 2 * u * (u + 2)
    tm = np.asfortranarray(r["tmat"][:nb, :nb])
    assert np.allclose(r["qtot"], f["qtot"], rtol=tol_q)
    assert _rel(np.linalg.norm(tm, axis=0), f["col_norms"]) <= tol_t
    assert _rel(tm[:, :f["cols_head"].shape[1]], f["cols_head"]) <= tol_t
    qe, qs = g.tmatrix_qext_qsca(tm, u)
    assert abs(qe / f["qext_t"] - 1) <= tol_q and abs(qs / f["qsca_t"] - 1) <= tol_q
    ro = g.ranorientscatmatrix(tm, u)
    assert np.abs(ro["smat"] - f["smat"]).max() <= 1e-4 * np.abs(f["smat"][:, 0, 0]).max()
    return r


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tensor_core", [("mixed", 0), ("mixed", -1), ("fp64", 0)])
def test_tmatrix100_against_oracle(precision, tensor_core):
    from mstm_b200 import api
    f = _load("tmatrix100")
    n = len(f["pos"])
    g = api.SphereCluster(f["pos"], np.full(n, 1.5), np.full(n, 1.6 + 0.005j), mie_epsilon=-8, precision=precision,
                          tensor_core=tensor_core)
    if precision == "fp64":
        r = _tmatrix_check(g, f, 1e-9, 1e-9)
        assert r["maxiter"] == f["maxiter"]
    else:
        _tmatrix_check(g, f, 1e-6, 1e-6)
    g.close()


@pytest.mark.gpu
def test_ensemble_tmatrix_configurations_against_oracle():
    from mstm_b200 import api
    for k, cfg in _ensemble_cfgs():
        f = _load("ensemble_tmatrix_c%d" % k)
        n = cfg["n"]
        g = api.SphereCluster(cfg["pos"], np.full(n, 1.5), np.full(n, 1.6 + 0.005j), mie_epsilon=-8, precision="mixed")
        _tmatrix_check(g, f, 1e-6, 1e-6)
        g.close()


@pytest.mark.gpu
def test_host1000_against_oracle():
    """Host spheres at the benchmark's size: a host holding 1000 inclusions,
    the FP64 BiCG (same iterations as the oracle; efficiencies, per-sphere
    solution norms and the leading solution blocks to 1e-9) and the mixed
    GMRES (Qext to 1e-6, the other efficiencies to 5e-6 of Qext)."""
    from mstm_b200 import api
    f = _load("host1000")
    g = api.SphereCluster(f["pos"], f["radius"], f["ref_index"], mie_epsilon=float(f["mie_eps"]), precision="fp64")
    assert np.array_equal(g.sphere_order, f["order"]) and np.array_equal(g.sphere_offset, f["offset"])
    r = g.fixedorsoln(eps=float(f["eps"]), niter=10000)
    assert r["istat"] == 0 and list(r["iterations"]) == list(f["iterations"])
    assert _rel(r["qtot"], f["qtot"]) <= 1e-9
    assert _rel(r["qeff"], f["qeff"]) <= 1e-9
    off = f["offset"]
    norms = np.array([[np.linalg.norm(r["amnp"][off[i]:off[i + 1], p]) for p in range(2)] for i in range(len(off) - 1)])
    assert _rel(norms, f["sphere_norms"]) <= 1e-9
    assert _rel(r["amnp"][:off[4]], f["amnp_head"]) <= 1e-9
    g.close()
    # the mixed solve: Qext to 1e-6; both solves stop at ||r||/||b|| < 1e-6,
    # so the other efficiencies to a few times that (5e-6 of Qext)
    m = api.SphereCluster(f["pos"], f["radius"], f["ref_index"], mie_epsilon=float(f["mie_eps"]), precision="mixed")
    rm = m.fixedorsoln(eps=float(f["eps"]), niter=10000)
    assert rm["istat"] == 0
    assert abs(rm["qtot"][0, 0] / f["qtot"][0, 0] - 1) <= 1e-6
    assert np.abs(rm["qtot"] - f["qtot"]).max() <= 5e-6 * f["qtot"][0, 0]
    assert np.abs(rm["qeff"] - f["qeff"]).max() <= 5e-6 * np.abs(f["qeff"]).max()
    m.close()
