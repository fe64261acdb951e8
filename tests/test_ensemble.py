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
