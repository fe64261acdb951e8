"""The seeded generators behind every benchmark configuration (CPU).

* PCA aggregates: the fractal law N = kf (Rg/a)^Df holds for the growing
  aggregate (Df and kf recovered by a log-log fit over N = 10..N), every
  monomer after the first touches an earlier one, and no two overlap.
* Random sequential addition in a sphere and in a cylinder (the reference's
  sample_position / add_sphere_to_cluster rules,
  random_configuration-10.f90:327-364, 479-540): the requested volume
  fraction, every sphere inside the boundary, no overlaps.
* Position files in the `x y z r` format read_sphere_data_input_file reads
  (mstm-input-37.f90:2886-2923) round-trip.
* The warm-start network file the benchmark loads was trained on the
  solver's solutions of 20,000 configurations drawn by these generators.
"""
import math

import numpy as np
import pytest

from mstm_b200 import configs as C


def _pair_dist(pos):
    d = np.sqrt(((pos[:, None, :] - pos[None, :, :]) ** 2).sum(-1))
    np.fill_diagonal(d, np.inf)
    return d


@pytest.mark.parametrize("n,x,df,kf,seed", [(500, 2.0, 1.8, 1.3, 2), (200, 1.0, 2.2, 1.1, 7)])
def test_pca_aggregate_fractal_law_contacts_and_overlaps(n, x, df, kf, seed):
    pos = C.pca_aggregate(n, x, df, kf, seed=seed)
    Ns = np.arange(10, n + 1)
    rg = np.array([C.radius_of_gyration(pos[:N]) for N in Ns])
    A = np.vstack([np.ones(len(Ns)), np.log(rg / x)]).T
    coef, *_ = np.linalg.lstsq(A, np.log(Ns), rcond=None)
    assert abs(coef[1] - df) < 0.02 * df, coef
    assert abs(math.exp(coef[0]) - kf) < 0.02 * kf, coef
    # the whole aggregate meets the law to 1 %
    assert abs(n / (C.radius_of_gyration(pos) / x) ** df / kf - 1.0) < 0.01
    d = _pair_dist(pos)
    assert d.min() >= 2.0 * x * (1.0 - 1e-12)
    gaps = [np.abs(d[k, :k] - 2.0 * x).min() for k in range(1, n)]
    assert max(gaps) < 1e-9 * x
    assert np.abs(pos.mean(axis=0)).max() < 1e-9


def test_pca_is_seeded():
    a = C.pca_aggregate(60, 2.0, 1.8, 1.3, seed=3)
    b = C.pca_aggregate(60, 2.0, 1.8, 1.3, seed=3)
    c = C.pca_aggregate(60, 2.0, 1.8, 1.3, seed=4)
    assert np.array_equal(a, b) and not np.allclose(a, c)


@pytest.mark.parametrize("n,x,fv,seed", [(20, 1.0, 0.10, 1), (400, 1.5, 0.20, 4), (300, 1.0, 0.30, 9)])
def test_rsa_sphere_volume_fraction_boundary_overlaps(n, x, fv, seed):
    pos, R = C.rsa_sphere(n, x, fv, seed=seed)
    assert pos.shape == (n, 3)
    assert abs(n * x ** 3 / R ** 3 - fv) < 1e-12
    assert np.sqrt((pos ** 2).sum(1)).max() <= R - x + 1e-12
    assert _pair_dist(pos).min() >= 2.0 * x


@pytest.mark.parametrize("n,x,fv,aspect,seed", [(1000, 1.0, 0.25, 1.0, 3), (300, 1.0, 0.15, 2.0, 5)])
def test_rsa_cylinder_volume_fraction_boundary_overlaps(n, x, fv, aspect, seed):
    pos, (Rc, H) = C.rsa_cylinder(n, x, fv, aspect, seed=seed)
    assert abs(H / (2.0 * Rc) - aspect) < 1e-12
    vol = math.pi * Rc ** 2 * H
    assert abs(n * 4.0 / 3.0 * math.pi * x ** 3 / vol - fv) < 1e-12
    assert np.sqrt(pos[:, 0] ** 2 + pos[:, 1] ** 2).max() <= Rc - x + 1e-12
    assert np.abs(pos[:, 2]).max() <= 0.5 * H - x + 1e-12
    assert _pair_dist(pos).min() >= 2.0 * x


def test_position_file_round_trip(tmp_path):
    pos = C.pca_aggregate(40, 2.0, 1.8, 1.3, seed=2)
    rad = np.full(40, 2.0)
    p = tmp_path / "agg.pos"
    C.write_position_file(str(p), pos, rad)
    lines = p.read_text().splitlines()
    assert len(lines) == 40 and all(len(l.split()) == 4 for l in lines)
    pos2, rad2 = C.read_position_file(str(p))
    assert np.allclose(pos2, pos, rtol=1e-10, atol=1e-10) and np.array_equal(rad2, rad)
    # with refractive indices (x y z r Re(m) Im(m)), the columns the reference reads after r
    ri = np.full(40, 1.6 + 0.05j)
    C.write_position_file(str(p), pos, rad, ri)
    rows = np.loadtxt(str(p))
    assert rows.shape == (40, 6) and np.allclose(rows[:, 4], 1.6) and np.allclose(rows[:, 5], 0.05)
    pos3, _ = C.read_position_file(str(p))
    assert np.allclose(pos3, pos, rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("n,x,fv,seed", [(300, 1.0, 0.30, 3), (120, 2.0, 0.05, 8)])
def test_rsa_sphere_batched(n, x, fv, seed):
    """The batched sampler of the warm-start study: n spheres, inside the
    bounding sphere of rsa_sphere's radius, no overlaps, seeded."""
    pos, R = C.rsa_sphere_batched(n, x, fv, seed=seed)
    assert pos.shape == (n, 3)
    assert abs(n * x ** 3 / R ** 3 - fv) < 1e-12
    assert np.sqrt((pos ** 2).sum(1)).max() <= R - x + 1e-12
    assert _pair_dist(pos).min() >= 2.0 * x
    assert np.array_equal(pos, C.rsa_sphere_batched(n, x, fv, seed=seed)[0])


def test_committed_warm_start_network_file():
    """The weights the benchmark's warm-start row loads: the network trained on
    the solver's solutions of 20,000 seeded configurations, with its held-out
    study (1,000 configurations) in the file's description."""
    import json
    import os
    from mstm_b200 import warmstart as W
    d = np.load(os.path.join(os.path.dirname(W.__file__), "data", "warmstart_net.npz"))
    meta = json.loads(str(d["meta"]))
    assert meta["n_train"] == 20000 and meta["n_eval"] == 1000 and meta["epochs"] == 20
    r = meta["fallback_1"]
    assert r["polarisations"] == 2000 and r["iterations_warm"] < r["iterations_mie_start"]
    assert int(d["hidden"]) > 0 and int(d["layers"]) > 0 and d["params"].dtype == np.float32
