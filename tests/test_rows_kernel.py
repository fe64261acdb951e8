"""The FP32 row kernel (translate_rows.cu) of the tiled path through the C ABI.

It applies the operator of the rotation-tiled kernel with the back rotation
and the i -> j axial product rewritten as row sweeps through the symmetries
of the Wigner functions and the axial blocks, from FP32 row records.  Checked
against the FP64 pass at 2e-6 of the largest output (FP32 rounding of
records and sums) and against the rotation-tiled kernel's FP32 pass
(tile_pairs 1), for every sphere order the tiled path takes (3..10; for
3 and 4 the FP64 pass runs the order-generic kernel on the tile-ordered
pairs, checked against a context of the generic pair order), column
counts the kernel runs directly (1, 2, 4) and in groups (3, 5, 8), plain and
conjugate-transpose columns, cluster sizes with partial tiles, and the FFT
path's grouped tiles of near pairs.
"""
import numpy as np
import pytest

from mstm_b200 import configs as C

pytestmark = pytest.mark.gpu

TOL = 2e-6


def _cluster_arrays(n, seed):
    pos, _ = C.rsa_sphere(n, 1.0, 0.15, seed=seed)
    return pos, np.full(n, 1.0), np.full(n, 1.45 + 0.01j)


def _pair(L, n, seed, **kw):
    from mstm_b200 import api
    pos, rad, ri = _cluster_arrays(n, seed)
    rows = api.SphereCluster(pos, rad, ri, mie_epsilon=-L, precision="mixed", **kw)
    rot = api.SphereCluster(pos, rad, ri, mie_epsilon=-L, precision="mixed", tile_pairs=1, **kw)
    return rows, rot


@pytest.mark.parametrize("L,n", [(3, 24), (4, 30), (5, 30), (6, 17), (7, 30), (8, 22), (9, 30), (10, 13)])
def test_row_kernel_matches_fp64_and_rotation_kernel(L, n):
    rows, rot = _pair(L, n, seed=L)
    rng = np.random.default_rng(L)
    if L < 5:
        # small orders: the FP64 pass on the tile-ordered pairs against the generic pair order
        from mstm_b200 import api
        gen = api.SphereCluster(*_cluster_arrays(n, L), mie_epsilon=-L, precision="fp64", generic_kernel=1)
        x = rng.normal(size=(rows.number_eqns, 2)) + 1j * rng.normal(size=(rows.number_eqns, 2))
        yt = rows.translation_pass(x, [0, 1], "fp64")
        yg = gen.translation_pass(x, [0, 1], "fp64")
        assert np.abs(yt - yg).max() <= 1e-12 * np.abs(yg).max()
        gen.close()
    for ct in ([0], [1], [0, 1], [1, 0], [0, 1, 1], [1, 0, 0, 1], [0, 0, 1, 1, 0], [0, 1] * 4):
        x = rng.normal(size=(rows.number_eqns, len(ct))) + 1j * rng.normal(size=(rows.number_eqns, len(ct)))
        y64 = rows.translation_pass(x, ct, "fp64")
        s = np.abs(y64).max()
        yr = rows.translation_pass(x, ct, "fp32")
        yo = rot.translation_pass(x, ct, "fp32")
        assert np.abs(yr - y64).max() <= TOL * s, (ct, np.abs(yr - y64).max() / s)
        assert np.abs(yr - yo).max() <= TOL * s, ct
    rows.close()
    rot.close()


def test_row_kernel_in_solves():
    """Mixed GMRES solves on the row kernel reach the FP64 solution's efficiencies."""
    from mstm_b200 import api
    w = C.workload("fractal60")
    kw = dict(mie_epsilon=-float(w["order"]))
    g = api.SphereCluster(w["pos"], w["radius"], w["ref_index"], precision="mixed", **kw)
    f = api.SphereCluster(w["pos"], w["radius"], w["ref_index"], precision="fp64", **kw)
    # eps bounds ||r||^2 / ||b||^2: 1e-14 leaves 1e-7 relative residuals
    rg = g.fixedorsoln(eps=1e-14, niter=4000)
    rf = f.fixedorsoln(eps=1e-14, niter=4000)
    assert rg["maxerr"] < 1e-14
    assert np.allclose(rg["qtot"], rf["qtot"], rtol=1e-6)
    g.close()
    f.close()


def test_row_kernel_on_grouped_fft_tiles():
    """The near pairs of the FFT path (grouped tiles) on the row kernel."""
    from mstm_b200 import api
    pos, _ = C.rsa_cylinder(300, 1.0, 0.25, 1.0, seed=3)
    n = len(pos)
    g = api.SphereCluster(pos, np.full(n, 1.0), np.full(n, 1.31 + 0j), mie_epsilon=-7, precision="mixed")
    o = api.SphereCluster(pos, np.full(n, 1.0), np.full(n, 1.31 + 0j), mie_epsilon=-7, precision="mixed", tile_pairs=1)
    for k in (g, o):
        k.fft_setup(d_cell=4.0)
    rng = np.random.default_rng(4)
    x = rng.normal(size=(g.number_eqns, 2)) + 1j * rng.normal(size=(g.number_eqns, 2))
    y64 = g.translation_pass(x, [0, 1], "fp64")
    s = np.abs(y64).max()
    yr = g.translation_pass(x, [0, 1], "fp32")
    yo = o.translation_pass(x, [0, 1], "fp32")
    assert np.abs(yr - yo).max() <= TOL * s
    assert np.abs(yr - y64).max() <= 1e-5 * s
    g.close()
    o.close()
