"""Ensemble solves: concurrent, autotuned T-matrix orientation averages agree
with one-at-a-time solves and with the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_ensemble_concurrent_autotuned_matches_sequential_and_oracle(oracle_mod):
    from mstm_b200 import ensemble as E
    cfgs = E.ensemble_configs(4, seed=7, nmin=12, nmax=30, x=1.0, m=1.5 + 0.01j, fv=0.15)
    tuner = E.Autotuner(reps=2)
    ens = E.solve_ensemble(cfgs, precision="mixed", workers=4, tuner=tuner, solution_eps=1e-12)
    assert len(tuner.log) >= 1 and all(t["best"] in E.Autotuner.CANDIDATES for t in tuner.log)
    seq = [E.solve_one(c, "fp64", solution_eps=1e-12) for c in cfgs]
    for r_e, r_s in zip(ens["per_config"], seq):
        assert r_e["order"] == r_s["order"]
        assert np.allclose(r_e["qtot"], r_s["qtot"], rtol=1e-6)
        assert np.abs(r_e["smat"] - r_s["smat"]).max() <= 1e-4 * np.abs(r_s["smat"][:, 0, 0]).max()
    assert abs(ens["qext"] - np.mean([r["qtot"][0] for r in seq])) <= 1e-6 * ens["qext"]
    # one configuration against the oracle's T matrix and random-orientation matrix
    c = cfgs[0]
    o = oracle_mod.Oracle(c["pos"], np.full(len(c["pos"]), c["x"]), np.full(len(c["pos"]), c["m"]), mie_eps=-c["order"])
    ro = o.tmatrix_solution(convergence_eps=1e-6, solution_eps=1e-12)
    assert ro["order"] == seq[0]["order"]
    assert np.allclose(seq[0]["qtot"], ro["qtot"], rtol=1e-9)
    u = ro["order"]
    nb = 2 * u * (u + 2)
    rr = oracle_mod.ranorientscatmatrix(u, np.asfortranarray(ro["tmat"][:nb, :nb]))
    assert np.abs(seq[0]["smat"] - rr["smat"]).max() <= 1e-8 * np.abs(rr["smat"][:, 0, 0]).max()


def test_fixed_ensemble_concurrent_matches_fp64():
    """Concurrent mixed-precision fixed-orientation solves of small clusters
    (four streams) give the efficiencies of one-at-a-time FP64 solves."""
    from mstm_b200 import ensemble as E
    from mstm_b200 import configs as C
    pos = [C.rsa_sphere(n, 1.0, 0.10, seed=200 + n)[0] for n in (12, 18, 25, 31, 16, 22)]
    ens = E.solve_fixed_ensemble(pos, 1.0, 1.5 + 0.01j, precision="mixed", workers=4)
    seq = E.solve_fixed_ensemble(pos, 1.0, 1.5 + 0.01j, precision="fp64", workers=1)
    for a, b in zip(ens["per_config"], seq["per_config"]):
        assert a["istat"] == 0 and b["istat"] == 0
        assert np.allclose(a["qtot"], b["qtot"], rtol=1e-6)


def _mie_times(an, order, f):
    """Mie multiply (LR-basis 2x2 per degree) of MSTM-layout columns f."""
    out = np.zeros_like(f)
    off, moff = 0, 0
    for L in order:
        hb = L * (L + 2)
        loc = np.arange(hb)
        row, col = loc % (L + 2), loc // (L + 2) + 1
        n = np.where(row <= col, col, row - 1)
        a = [an[moff + 4 * (n - 1) + k][:, None] for k in range(4)]
        u0, u1 = f[off:off + hb], f[off + hb:off + 2 * hb]
        out[off:off + hb] = a[0] * u0 + a[2] * u1
        out[off + hb:off + 2 * hb] = a[1] * u0 + a[3] * u1
        off += 2 * hb
        moff += 4 * L
    return out


@pytest.mark.parametrize("mixed_orders", [False, True])
def test_one_context_ensemble_matches_separate_solves(oracle_mod, mixed_orders):
    """An ensemble context (no pairs between configurations; one translation
    pass a step for all of them) gives every configuration the efficiencies
    of its own mixed-precision solve and of the FP64 oracle within 1e-6, each
    system meets the criterion on its own configuration, and the returned
    coefficients satisfy each configuration's FP64 system.  With mixed_orders
    the configurations have two sphere orders (the non-tiled pair path)."""
    from mstm_b200 import api
    from mstm_b200 import configs as C
    sizes = (12, 18, 25, 31, 16, 22)
    xs = [1.0 if (not mixed_orders or k % 2 == 0) else 1.4 for k in range(len(sizes))]
    cfgs = [(C.rsa_sphere(n, x, 0.10, seed=500 + n)[0], np.full(n, x), 1.5 + 0.01j) for n, x in zip(sizes, xs)]
    em = 1e-6 if mixed_orders else -C.truncation_order(1.0)
    ens = api.SphereEnsemble(cfgs, mie_epsilon=em)
    r = ens.fixedorsoln(eps=1e-12, niter=4000)
    assert r["istat"] == 0 and (r["errors"] < 1e-12).all()
    an, _, _ = ens.miecoefcalc()
    f = np.zeros((ens.number_eqns, 2), complex)
    for k, (pos, rad, m) in enumerate(cfgs):
        g = api.SphereCluster(pos, rad, np.full(len(rad), m), mie_epsilon=em, precision="mixed")
        rs = g.fixedorsoln(eps=1e-12, niter=4000)
        assert np.allclose(r["qtot"][k], rs["qtot"], rtol=1e-6), k
        assert abs(int(r["iterations"][k].max()) - int(rs["maxiter"])) <= 2
        # this configuration's FP64 system (I - M H) x = M f, checked on its own context
        x = r["amnp_of"](k)
        fk = g.sphereplanewavecoef()
        ank, _, _ = g.miecoefcalc()
        bm = _mie_times(ank, g.sphere_order, fk)
        res = bm - x + g.sphereinteraction(x, initial_run=True)
        for p in range(2):
            rel = np.vdot(res[:, p], res[:, p]).real / np.vdot(bm[:, p], bm[:, p]).real
            assert rel < 1e-11, (k, p, rel)
        if k == 0:
            o = oracle_mod.Oracle(pos, rad, np.full(len(rad), m), mie_eps=em)
            ro = o.fixedorsoln(eps=1e-12, niter=4000)
            assert np.allclose(r["qtot"][k], ro["qtot"], rtol=1e-6)
        g.close()


def test_ensemble_context_refuses_single_cluster_entry_points():
    """Entry points that treat a context as one cluster return
    MSTMG_ERR_UNSUPPORTED on an ensemble; the block-diagonal matvec is the
    configurations' own matvecs side by side."""
    import ctypes
    from mstm_b200 import _lib, api
    from mstm_b200 import configs as C
    cfgs = [(C.rsa_sphere(n, 1.0, 0.10, seed=700 + n)[0], np.full(n, 1.0), 1.5 + 0.01j) for n in (9, 14)]
    ens = api.SphereEnsemble(cfgs, mie_epsilon=-C.truncation_order(1.0))
    L = _lib.lib()
    amnp = np.zeros((ens.number_eqns, 2), np.complex128)
    me, mi = ctypes.c_double(0.0), ctypes.c_int(0)
    rc = L.mstmg_fixed_orientation(ens.ctx, 0.0, 0.0, 1, 1e-12, 100, amnp.ctypes.data_as(ctypes.c_void_p), None, None,
                                   ctypes.byref(me), ctypes.byref(mi))
    assert rc == -3 and "ensemble" in L.mstmg_last_error().decode()
    rng = np.random.default_rng(3)
    x = rng.normal(size=(ens.number_eqns, 2)) + 1j * rng.normal(size=(ens.number_eqns, 2))
    y = ens.sphereinteraction(x, initial_run=True)
    off = ens.sphere_offset
    for k, (pos, rad, m) in enumerate(cfgs):
        g = api.SphereCluster(pos, rad, np.full(len(rad), m), mie_epsilon=-C.truncation_order(1.0), precision="fp64")
        a, b = off[ens.config_start[k]], off[ens.config_start[k + 1]]
        yk = g.sphereinteraction(x[a:b], initial_run=True)
        assert np.abs(y[a:b] - yk).max() <= 1e-12 * np.abs(yk).max()
        g.close()


def test_ensemble_edge_configurations(oracle_mod):
    """Configurations of one and two spheres beside larger ones, and GMRES
    cycles of 4 steps: every system meets the criterion and the single sphere
    gives its Mie efficiency (no pairs: the Mie start is the solution)."""
    from mstm_b200 import api
    from mstm_b200 import configs as C
    L = C.truncation_order(1.0)
    cfgs = [(np.zeros((1, 3)), np.full(1, 1.0), 1.5 + 0.01j),
            (np.array([[0.0, 0.0, 0.0], [2.5, 0.0, 0.0]]), np.full(2, 1.0), 1.5 + 0.01j),
            (C.rsa_sphere(15, 1.0, 0.10, seed=801)[0], np.full(15, 1.0), 1.5 + 0.01j)]
    ens = api.SphereEnsemble(cfgs, mie_epsilon=-L, gmres_restart=4)
    r = ens.fixedorsoln(eps=1e-12, niter=4000)
    assert r["istat"] == 0 and (r["errors"] < 1e-12).all()
    _, qe, _ = ens.miecoefcalc()
    assert abs(r["qtot"][0][0, 0] / qe[0] - 1) < 1e-12
    for k in (1, 2):
        pos, rad, m = cfgs[k]
        o = oracle_mod.Oracle(pos, rad, np.full(len(rad), m), mie_eps=-L)
        ro = o.fixedorsoln(eps=1e-12, niter=4000)
        assert np.allclose(r["qtot"][k], ro["qtot"], rtol=1e-6), k


def test_sharded_ensemble_single_rank_matches_batched():
    """solve_fixed_ensemble_sharded on one rank (no process group) solves the
    whole ensemble in one context: its means are those of its own
    per-configuration results, and agree with a separate batched solve to far
    below the solution criterion (two solves differ only in the FP32 passes'
    summation order)."""
    from mstm_b200 import ensemble as E
    from mstm_b200 import configs as C
    pos = [C.rsa_sphere(n, 1.0, 0.10, seed=600 + n)[0] for n in (10, 17, 24)]
    sh = E.solve_fixed_ensemble_sharded(pos, 1.0, 1.5 + 0.01j, rank=0, world=1)
    assert sh["indices"] == [0, 1, 2] and sh["count"] == 3
    own = np.array([r["qtot"] for r in sh["per_config"]])
    assert abs(sh["qext_mean"] / own[:, 0, 0].mean() - 1) < 1e-14
    assert abs(sh["qsca_mean"] / own[:, 2, 0].mean() - 1) < 1e-14
    b = E.solve_fixed_ensemble_batched(pos, 1.0, 1.5 + 0.01j)
    q = np.array([r["qtot"] for r in b["per_config"]])
    assert abs(sh["qext_mean"] / q[:, 0, 0].mean() - 1) < 1e-8
