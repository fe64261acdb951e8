"""Host spheres: spheres inside other spheres (findhostspheres,
december2023/mstm-modules-33.f90:5230-5276; external_to_internal_expansion,
:6533-6608; the host branch of multmiecoeffmult, :5690-5747).

CPU: the oracle's host branch is pinned by two known answers -- a core
concentric in a shell is the coated sphere of Aden and Kerker (written here
from the published formulas with scipy's spherical Bessel functions), and a
host whose index matches the medium is transparent (the spheres inside it
scatter and absorb as the same cluster in free space, with the same
scattering matrix), and the coated sphere's T matrix averages to its Qext and
Qsca -- and by its BiCG
against its dense solve.  GPU: the device path against the oracle on a
cluster with two host levels, coincident and offset centres, small spheres
on the dense path and spheres outside: host map, orders, layout, Mie
coefficients (1e-12), sphereinteraction in every argument form (1e-12), the
FP64 solves (same iterations, efficiencies to 1e-9), the mixed solve (1e-6),
the scattering matrix (1e-9 of S11's largest value), the cluster T matrix
(1e-9 FP64, 1e-6 mixed) and the refusals of the entry points built for
spheres in the medium.
"""
import numpy as np
import pytest
from scipy.special import spherical_jn, spherical_yn


def coated_sphere(x, y, m1, m2, nmax):
    """Qext, Qsca of a sphere of size parameter x and index m1 inside a
    concentric shell of size parameter y and index m2 (Aden-Kerker; the
    coefficients as Bohren and Huffman write them, section 8.1)."""
    n = np.arange(1, nmax + 1)

    def psi(z):
        return z * spherical_jn(n, z)

    def dpsi(z):
        return spherical_jn(n, z) + z * spherical_jn(n, z, derivative=True)

    def chi(z):
        return -z * spherical_yn(n, z)

    def dchi(z):
        return -spherical_yn(n, z) - z * spherical_yn(n, z, derivative=True)

    def xi(z):
        return psi(z) - 1j * chi(z)

    def dxi(z):
        return dpsi(z) - 1j * dchi(z)

    A = (m2 * psi(m2 * x) * dpsi(m1 * x) - m1 * dpsi(m2 * x) * psi(m1 * x)) / \
        (m2 * chi(m2 * x) * dpsi(m1 * x) - m1 * dchi(m2 * x) * psi(m1 * x))
    B = (m2 * psi(m1 * x) * dpsi(m2 * x) - m1 * psi(m2 * x) * dpsi(m1 * x)) / \
        (m2 * dchi(m2 * x) * psi(m1 * x) - m1 * dpsi(m1 * x) * chi(m2 * x))
    u, du = psi(m2 * y) - A * chi(m2 * y), dpsi(m2 * y) - A * dchi(m2 * y)
    v, dv = psi(m2 * y) - B * chi(m2 * y), dpsi(m2 * y) - B * dchi(m2 * y)
    a = (psi(y) * du - m2 * dpsi(y) * u) / (xi(y) * du - m2 * dxi(y) * u)
    b = (m2 * psi(y) * dv - dpsi(y) * v) / (m2 * xi(y) * dv - dxi(y) * v)
    f = 2 * n + 1
    return 2 / y ** 2 * np.sum(f * (a + b).real), 2 / y ** 2 * np.sum(f * (np.abs(a) ** 2 + np.abs(b) ** 2))


def host_cluster():
    """Host A (radius 2.5) holding a concentric core, sphere F and sphere B,
    which holds the small sphere C; outside, sphere D and the small sphere E
    (orders below 3: dense pairs)."""
    pos = np.array([
        [0.0, 0.0, 0.0],     # A host
        [0.0, 0.0, 0.0],     # core, concentric in A
        [1.55, 0.0, 0.1],    # B, in A, holds C
        [1.62, 0.12, 0.05],  # C, in B
        [-0.9, 1.3, -0.4],   # F, in A
        [4.2, 0.3, 0.6],     # D, outside
        [-3.6, 1.1, -0.2],   # E, outside, small
    ])
    rad = np.array([2.5, 0.7, 0.5, 0.15, 0.45, 0.7, 0.2])
    ri = np.array([1.33 + 0.001j, 1.6 + 0.05j, 1.5 + 0.01j, 1.7 + 0.1j, 1.45 + 0.0j, 1.55 + 0.02j, 1.4 + 0.0j])
    return pos, rad, ri


# ---------------------------------------------------------------------------
# CPU: the oracle's host branch against known answers
# ---------------------------------------------------------------------------
def test_oracle_finds_hosts_and_raises_orders(oracle_mod):
    pos, rad, ri = host_cluster()
    o = oracle_mod.Oracle(pos, rad, ri, mie_eps=1e-6)
    host, nh = o.hosts()
    assert host.tolist() == [-1, 0, 0, 2, 0, -1, -1] and nh == 4
    # a host's order is at least that of every sphere inside it
    assert o.order[0] >= o.order[[1, 2, 3, 4]].max() and o.order[2] >= o.order[3]
    # layout: the hosts' blocks are followed by their internal blocks
    nb = 2 * o.order * (o.order + 2)
    assert np.array_equal(np.diff(o.offset), nb * np.array([2, 1, 2, 1, 1, 1, 1]))
    assert o.order[6] < 3


def test_oracle_coated_sphere_is_aden_kerker(oracle_mod):
    x, y, m1, m2 = 1.2, 2.0, 1.6 + 0.05j, 1.33 + 0.01j
    o = oracle_mod.Oracle([[0, 0, 0], [0, 0, 0]], [y, x], [m2, m1], mie_eps=-14)
    r = o.fixedorsoln(eps=1e-20, niter=300)
    qe, qs = coated_sphere(x, y, m1, m2, 14)
    # the shell's efficiencies (its absorption net of the core's, then the
    # core's added back, as qtotcalc forms them) are the coated sphere's
    assert abs(r["qeff"][0, 0, 0] - qe) <= 1e-9 * qe
    assert abs((r["qeff"][0, 0, 0] - r["qeff"][1, 0, 0]) - qs) <= 1e-9 * qs
    # qtot differs only by vol_radius's single-precision exponent
    xg = o.vol_radius()
    assert abs(r["qtot"][0, 0] * xg ** 2 - qe * y ** 2) <= 1e-9 * qe * y ** 2


def test_oracle_index_matched_host_is_transparent(oracle_mod):
    inner = np.array([[0.8, 0.0, 0.1], [-0.7, 0.3, -0.2], [0.0, -0.6, 0.7]])
    ri_in = np.array([1.5 + 0.02j, 1.45 + 0.0j, 1.6 + 0.1j])
    rin = np.array([0.5, 0.55, 0.45])
    L = 14
    free = oracle_mod.Oracle(inner, rin, ri_in, mie_eps=-L)
    rf = free.fixedorsoln(eps=1e-20, niter=300)
    h = oracle_mod.Oracle(np.vstack([[0, 0, 0], inner]), np.r_[2.0, rin], np.r_[1.0 + 0j, ri_in], mie_eps=-L)
    rh = h.fixedorsoln(eps=1e-20, niter=300)
    cf = rf["qtot"][:, 0] * free.vol_radius() ** 2
    ch = rh["qtot"][:, 0] * h.vol_radius() ** 2
    assert np.allclose(ch, cf, rtol=1e-7, atol=0)
    assert np.allclose(rh["qeff"][1, 0, [1, 3]], rf["qeff"][1, 0, [0, 2]], rtol=1e-8)
    # the far field too: merged about the host's centre (the one sphere
    # outside) against the free cluster merged about its own centroid
    sf, sh = free.scattering(rf["amnp"]), h.scattering(rh["amnp"])
    assert np.abs(sh["smat"] - sf["smat"]).max() <= 1e-7 * np.abs(sf["smat"][:, 0, 0]).max()
    assert abs(sh["g"] - sf["g"]) <= 1e-7 * abs(sf["g"])


def test_oracle_coated_sphere_t_matrix(oracle_mod):
    """The T matrix of a coated sphere (the core's excitation reaches it
    through the shell's internal field only): its orientation-averaged Qext
    and Qsca are the Aden-Kerker ones."""
    x, y, m1, m2 = 1.2, 2.0, 1.6 + 0.05j, 1.33 + 0.01j
    o = oracle_mod.Oracle([[0, 0, 0], [0, 0, 0]], [y, x], [m2, m1], mie_eps=-10)
    r = o.tmatrix_solution(solution_eps=1e-20, convergence_eps=1e-12, maxt=10)
    u = r["order"]
    nb = 2 * u * (u + 2)
    qe, qs = oracle_mod.tmatrix_qext_qsca(u, np.asfortranarray(r["tmat"][:nb, :nb]), y)
    qe0, qs0 = coated_sphere(x, y, m1, m2, 10)
    # T entries are single precision in the orientation average
    assert abs(qe / qe0 - 1) < 1e-7 and abs(qs / qs0 - 1) < 1e-7


def test_oracle_host_bicg_matches_dense_solve(oracle_mod):
    pos, rad, ri = host_cluster()
    o = oracle_mod.Oracle(pos, rad, ri, mie_eps=1e-6)
    b = o.planewave()
    pnp = o.multmie(b[:, 0])
    x, it, err, rc = o.cbicg(pnp, pnp.copy(), niter=500, eps=1e-24)
    assert rc == 0 and err < 1e-24
    xd = o.direct_solve(pnp)
    assert np.abs(x - xd).max() <= 1e-9 * np.abs(xd).max()


# ---------------------------------------------------------------------------
# GPU: the device path against the oracle
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def pair(oracle_mod):
    from mstm_b200 import api
    pos, rad, ri = host_cluster()
    g = api.SphereCluster(pos, rad, ri, mie_epsilon=1e-6, precision="fp64")
    o = oracle_mod.Oracle(pos, rad, ri, mie_eps=1e-6, store_matrix=True, nthreads=4)
    yield g, o
    g.close()
    o.close()


@pytest.mark.gpu
def test_host_layout_and_mie_coefficients(pair):
    g, o = pair
    host, nh = g.host_spheres()
    ho, nho = o.hosts()
    assert np.array_equal(host, ho) and nh == nho == 4
    assert np.array_equal(g.sphere_order, o.order) and np.array_equal(g.sphere_offset, o.offset)
    assert g.number_eqns == o.neqns
    an_g, qe_g, qa_g = g.miecoefcalc()
    an_o, _, qe_o, qa_o = o.mie()
    assert np.abs(an_g - an_o).max() <= 1e-12 * np.abs(an_o).max()
    for cg, co in zip(g.host_mie_coefficients(), o.host_mie()):
        assert np.abs(cg - co).max() <= 1e-12 * np.abs(co).max()
    assert np.allclose(qe_g, qe_o, rtol=1e-12)
    assert abs(g.vol_radius - o.vol_radius()) <= 1e-14 * o.vol_radius()


@pytest.mark.gpu
def test_host_sphereinteraction(pair):
    g, o = pair
    rng = np.random.default_rng(5)
    x = rng.standard_normal((g.number_eqns, 4)) + 1j * rng.standard_normal((g.number_eqns, 4))
    for ct, mm in (([0, 1, 0, 1], [1, 1, 0, 0]), ([1, 0, 1, 0], [1, 0, 1, 0])):
        yg = g.sphereinteraction(x, con_tran=ct, mie_mult=mm, initial_run=True)
        yo = o.sphereinteraction(x, con_tran=ct, mie_mult=mm, initial_run=True)
        assert np.abs(yg - yo).max() <= 1e-12 * np.abs(yo).max()
    # the host couplings alone (skip_external_translation)
    yg = g.sphereinteraction_ex(x[:, :2], con_tran=[0, 1], skip_external_translation=True)
    yo = o.sphereinteraction(x[:, :2], con_tran=[0, 1], skip_external=True)
    assert np.abs(yo).max() > 0
    assert np.abs(yg - yo).max() <= 1e-12 * np.abs(yo).max()
    # the incident wave reaches the spheres outside every other only
    pg = g.sphereplanewavecoef()
    po = o.planewave()
    assert np.abs(pg - po).max() <= 1e-13 * np.abs(po).max()
    off = o.offset
    assert np.abs(po[off[1]:off[5]]).max() == 0.0


@pytest.mark.gpu
def test_host_fixedorsoln(pair):
    g, o = pair
    ro = o.fixedorsoln(eps=1e-12, niter=500)
    rg = g.fixedorsoln(eps=1e-12, niter=500)
    assert rg["istat"] == ro["status"] == 0
    assert rg["iterations"] == ro["iterations"]
    assert np.abs(rg["amnp"] - ro["amnp"]).max() <= 1e-8 * np.abs(ro["amnp"]).max()
    assert np.allclose(rg["qeff"], ro["qeff"], rtol=1e-9, atol=1e-12)
    assert np.allclose(rg["qtot"], ro["qtot"], rtol=1e-9)
    # efficiencies of a given solution, and the right-hand sides
    q = g.efficiencies(ro["amnp"])
    assert np.allclose(q["qtot"], ro["qtot"], rtol=1e-10)
    b = g.fixed_orientation_rhs()
    po = o.planewave()
    assert np.abs(b[:, 0] - o.multmie(po[:, 0])).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.gpu
def test_host_scattering_matrix(pair):
    """The scattering matrix and g of a host cluster: the spheres outside
    every other merged about their centroid (merge_to_common_origin with
    origin_host 0, scatprops:631)."""
    g, o = pair
    ro = o.fixedorsoln(eps=1e-12, niter=500)
    so = o.scattering(ro["amnp"])
    sg = g.scattering(ro["amnp"])
    assert sg["t_matrix_order"] == so["t_matrix_order"]
    assert np.abs(sg["amnp0"] - so["amnp0"]).max() <= 1e-10 * np.abs(so["amnp0"]).max()
    assert np.abs(sg["smat"] - so["smat"]).max() <= 1e-9 * np.abs(so["smat"][:, 0, 0]).max()
    assert abs(sg["g"] - so["g"]) <= 1e-9 * abs(so["g"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_host_t_matrix(pair, precision):
    """tmatrix_solution with host spheres: the excitation distributed to the
    spheres outside every other, the per-column efficiencies through the
    interaction, the merge of the outside spheres; FP64 against the oracle to
    1e-9 (T matrix, sums, order kept), mixed GMRES to 1e-6."""
    from mstm_b200 import api
    _, o = pair
    pos, rad, ri = host_cluster()
    g = api.SphereCluster(pos, rad, ri, mie_epsilon=1e-6, precision=precision)
    ro = o.tmatrix_solution(convergence_eps=1e-6, solution_eps=1e-12 if precision == "fp64" else 1e-16)
    T = g.t_matrix_order()
    assert T == ro["tmo"]
    rg = g.tmatrix_solution(T, solution_eps=1e-12, convergence_eps=1e-6)
    assert rg["istat"] == 0 and rg["order"] == ro["order"]
    tol = 1e-9 if precision == "fp64" else 1e-6
    assert np.abs(rg["tmat"] - ro["tmat"]).max() <= tol * np.abs(ro["tmat"]).max()
    assert np.abs(rg["qtot"] - ro["qtot"]).max() <= tol * ro["qtot"][0]
    assert np.abs(rg["sphere_qeff"] - ro["sphere_qeff"]).max() <= tol * np.abs(ro["sphere_qeff"]).max()
    g.close()


@pytest.mark.gpu
def test_host_solver_modes(pair):
    """niter 0 (the host couplings applied twice, solver:509-518) and the
    order-of-scattering iteration (niter < 0)."""
    g, o = pair
    for niter in (0, -60):
        ro = o.fixedorsoln(eps=1e-10, niter=niter)
        rg = g.fixedorsoln(eps=1e-10, niter=niter)
        assert rg["iterations"][1] == ro["maxiter"]
        assert np.abs(rg["amnp"] - ro["amnp"]).max() <= 1e-9 * np.abs(ro["amnp"]).max()
        assert np.allclose(rg["qtot"], ro["qtot"], rtol=1e-9)


@pytest.mark.gpu
def test_host_mixed_precision(pair):
    """The mixed solve (FP32 GMRES passes with the host couplings in FP32,
    FP64 true residuals) against the oracle to the mixed path's 1e-6, and the
    FP32 translation pass against the FP64 one."""
    from mstm_b200 import api
    g, o = pair
    pos, rad, ri = host_cluster()
    m = api.SphereCluster(pos, rad, ri, mie_epsilon=1e-6, precision="mixed")
    rm = m.fixedorsoln(eps=1e-12, niter=500)
    ro = o.fixedorsoln(eps=1e-16, niter=1000)
    assert rm["istat"] == 0
    # to 1e-6 of the extinction (absorption is a small difference here)
    assert np.abs(rm["qtot"] - ro["qtot"]).max() <= 1e-6 * ro["qtot"][0, 0]
    assert np.abs(rm["qeff"] - ro["qeff"]).max() <= 1e-6 * np.abs(ro["qeff"]).max()
    rng = np.random.default_rng(8)
    x = rng.standard_normal((g.number_eqns, 2)) + 1j * rng.standard_normal((g.number_eqns, 2))
    y64 = g.translation_pass(x, [0, 1], "fp64")
    y32 = g.translation_pass(x, [0, 1], "fp32")
    assert np.abs(y32 - y64).max() <= 2e-6 * np.abs(y64).max()
    m.close()


@pytest.mark.gpu
def test_host_contexts_refuse_the_medium_only_paths(pair):
    from mstm_b200 import api
    from mstm_b200._lib import MstmgError
    g, _ = pair
    pos, rad, ri = host_cluster()
    m = api.SphereCluster(pos, rad, ri, mie_epsilon=1e-6, precision="mixed", mixed_solver=1)
    with pytest.raises(MstmgError):
        m.fixedorsoln(eps=1e-8)
    m.close()
    with pytest.raises(MstmgError):
        g.fft_setup(d_cell=2.0)
    with pytest.raises(MstmgError):
        g.set_positions(pos + 0.01)
    x = np.ones((g.number_eqns, 16), np.complex128)
    with pytest.raises(MstmgError):
        g.translation_pass(x, None, "tc")


@pytest.mark.gpu
def test_moving_a_sphere_inside_another_needs_a_new_context():
    from mstm_b200 import api
    from mstm_b200._lib import MstmgError
    pos = np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0], [0.0, 3.5, 0.0]])
    rad = np.array([1.5, 0.5, 0.6])
    g = api.SphereCluster(pos, rad, np.full(3, 1.5 + 0.01j), mie_epsilon=1e-6, precision="fp64")
    assert g.host_spheres()[1] == 0
    moved = pos.copy()
    moved[1] = [0.5, 0.0, 0.0]     # now inside sphere 0
    with pytest.raises(MstmgError):
        g.set_positions(moved)
    g.set_positions(pos + 0.25)    # still outside: accepted
    g.close()


COATED_DECK = """! a coated sphere: core concentric in a shell, read as host spheres
number_spheres
2
sphere_data
0.d0,0.d0,0.d0,2.d0,(1.33d0,0.01d0)
0.d0,0.d0,0.d0,1.2d0,(1.6d0,0.05d0)
end_of_sphere_data
mie_epsilon
-14.d0
solution_epsilon
1.d-16
incident_beta_deg
0.d0
end_of_options
"""


@pytest.mark.gpu
def test_coated_sphere_deck():
    """An input deck with a core inside a shell runs through the library's
    host-sphere path: Qext and Qsca are the Aden-Kerker values, the run's
    sphere table names the host."""
    from mstm_b200 import inputfile as I
    from mstm_b200.output import run_variables
    run = I.parse(COATED_DECK)[0]
    out = I.execute(run, "fp64")
    qe, qs = coated_sphere(1.2, 2.0, 1.6 + 0.05j, 1.33 + 0.01j, 14)
    xg = out["vol_radius"]
    assert abs(out["qtot"][0, 0] * xg ** 2 / (qe * 4.0) - 1) < 1e-9
    assert abs(out["qtot"][2, 0] * xg ** 2 / (qs * 4.0) - 1) < 1e-9
    assert list(out["host"]) == [-1, 0]
    L = run_variables(run, out)
    i = L.index(" sphere properties and associations")
    assert L[i + 3][:16] == "       2       1"


@pytest.mark.gpu
@pytest.mark.parametrize("order", [4, 6])
def test_host_inclusions_on_tiles(oracle_mod, order):
    """Inclusions of one order inside a host: their pairs run on the tiled
    kernels (grouped tiles, each sphere's block at its own offset): the
    interaction to 1e-12, the FP64 solve (same iterations, 1e-9) and the
    mixed one (1e-6) against the oracle."""
    from mstm_b200 import api, configs as C
    w = C.host_inclusions(40, 0.5, 0.15, seed=order)
    # the host's order is raised to the inclusions' (forced) order
    g = api.SphereCluster(w["pos"], w["radius"], w["ref_index"], mie_epsilon=-order, precision="fp64")
    o = oracle_mod.Oracle(w["pos"], w["radius"], w["ref_index"], mie_eps=-order, nthreads=4)
    assert np.array_equal(g.sphere_offset, o.offset)
    rng = np.random.default_rng(order)
    x = rng.standard_normal((g.number_eqns, 2)) + 1j * rng.standard_normal((g.number_eqns, 2))
    yg = g.sphereinteraction(x, con_tran=[0, 1], initial_run=True)
    yo = o.sphereinteraction(x, con_tran=[0, 1], initial_run=True)
    assert np.abs(yg - yo).max() <= 1e-12 * np.abs(yo).max()
    y32 = g.translation_pass(x, [0, 1], "fp32")
    y64 = g.translation_pass(x, [0, 1], "fp64")
    assert np.abs(y32 - y64).max() <= 2e-6 * np.abs(y64).max()
    ro = o.fixedorsoln(eps=1e-12, niter=500)
    rg = g.fixedorsoln(eps=1e-12, niter=500)
    assert rg["iterations"] == ro["iterations"]
    assert np.allclose(rg["qtot"], ro["qtot"], rtol=1e-9)
    m = api.SphereCluster(w["pos"], w["radius"], w["ref_index"], mie_epsilon=-order, precision="mixed")
    rm = m.fixedorsoln(eps=1e-12, niter=500)
    assert np.abs(rm["qtot"] - ro["qtot"]).max() <= 5e-6 * ro["qtot"][0, 0]
    for k in (g, m, o):
        k.close()
