"""MSTM input decks: parsing (CPU) and runs through the library (GPU)."""
import numpy as np
import pytest

from mstm_b200 import inputfile as I

DECK = """! a 3-sphere cluster
output_file
out.dat
number_spheres
3
sphere_data
0.d0,0.d0,0.d0,1.d0,(1.5d0,0.01d0)
2.5d0 0.d0 0.d0 1.d0 1.5d0 0.01d0
0.d0,2.6d0,0.4d0,1.d0,(1.5d0,0.01d0)
end_of_sphere_data
length_scale_factor
1.d0
mie_epsilon
-5.d0
solution_epsilon
1.d-12
incident_beta_deg
0.d0
calculate_scattering_matrix
t
new_run
random_orientation
t
t_matrix_convergence_epsilon
1.d-8
end_of_options
this line is after the end and is not read
"""


def test_parse_deck_and_literals():
    runs = I.parse(DECK)
    assert len(runs) == 2
    r0, r1 = runs
    assert r0["number_spheres"] == 3 and r0["mie_epsilon"] == -5.0 and r0["solution_epsilon"] == 1e-12
    assert r0["random_orientation"] is False and r1["random_orientation"] is True
    assert r1["t_matrix_convergence_epsilon"] == 1e-8 and r1["solution_epsilon"] == 1e-12   # inherited
    pos, rad, ri = I.cluster_arrays(r0)
    assert pos.shape == (3, 3) and np.allclose(pos[1], [2.5, 0, 0]) and np.allclose(ri, 1.5 + 0.01j)
    assert I._complex("(1.6d0,0.d0)") == 1.6 + 0j and I._real("1.d-15") == 1e-15
    alpha, sinc, d = I.incidence(dict(incident_beta_deg=120.0, incident_alpha_deg=30.0), 1.0 + 0j)
    assert d == 2 and abs(sinc - np.sin(120 * I.REF_PI / 180)) < 1e-15


def test_run_structure_and_loop_variable():
    """new_run separates runs that inherit settings, end_of_options ends the
    input, loop_variable repeats a run over start..stop (stop included within
    1e-6) in nested order, and leaves the variable one step past the end."""
    deck = ("number_spheres\n1\nsphere_data\n0 0 0 1 1.5 0\nend_of_sphere_data\n"
            "loop_variable\nincident_beta_deg\n0.d0,90.d0,45.d0\n"
            "loop_variable\nmax_iterations\n10 20 10\n"
            "new_run\nmie_epsilon\n-3\nend_of_options\nbogus_option\n1\n")
    runs = I.parse(deck)
    assert [(r["incident_beta_deg"], r["max_iterations"]) for r in runs[:6]] == \
        [(0.0, 10), (0.0, 20), (45.0, 10), (45.0, 20), (90.0, 10), (90.0, 20)]
    assert len(runs) == 7 and runs[6]["mie_epsilon"] == -3.0
    assert runs[6]["incident_beta_deg"] == 135.0 and runs[6]["max_iterations"] == 30
    vals, after = I._loop_values("r", 1.0, 0.0, -0.25)
    assert vals == [1.0, 0.75, 0.5, 0.25, 0.0] and after == -0.25
    with pytest.raises(NotImplementedError):
        I.parse("loop_variable\nsphere_number\n2\nsphere_radius\n1 2 1\nend_of_options\n")


def test_options_outside_the_path_are_rejected():
    deck = "number_spheres\n1\nsphere_data\n0 0 0 1 1.5 0\nend_of_sphere_data\nnumber_plane_boundaries\n2\nend_of_options\n"
    run = I.parse(deck)[0]
    with pytest.raises(NotImplementedError):
        I.check_supported(run)
    with pytest.raises(NotImplementedError):
        I.parse("calculate_near_field_plane\nt\n")


@pytest.mark.gpu
def test_deck_runs_match_oracle(oracle_mod, tmp_path):
    runs = I.parse(DECK)
    fixed = I.execute(runs[0], "fp64")
    pos, rad, ri = I.cluster_arrays(runs[0])
    o = oracle_mod.Oracle(pos, rad, ri, mie_eps=-5.0)
    ro = o.fixedorsoln(eps=1e-12)
    assert np.allclose(fixed["qtot"], ro["qtot"], rtol=1e-9)
    sc = o.scattering(ro["amnp"])
    assert abs(fixed["g_asym"] - sc["g"]) < 1e-9
    # azimuthal_average false (the default): the plane of incidence, -180..180
    th, sm = oracle_mod.incident_plane_scattering(sc["t_matrix_order"], sc["amnp0"], increment=1.0)
    assert fixed["smat"].shape == (361, 4, 4) and np.array_equal(fixed["theta"], th)
    assert np.abs(fixed["smat"] - sm).max() <= 1e-8 * np.abs(sm[:, 0, 0]).max()
    avg = dict(runs[0], azimuthal_average=True, scattering_map_increment=5.0)
    fa = I.execute(avg, "fp64")
    gs = oracle_mod.gsf_scattering(sc["t_matrix_order"], sc["amnp0"], nangles=37)
    ga = gs["smat"]
    assert fa["smat"].shape == (37, 4, 4) and np.abs(fa["smat"] - ga).max() <= 1e-8 * np.abs(ga[:, 0, 0]).max()
    from mstm_b200.output import calculation_results, es
    L = calculation_results(avg, fa)
    i = L.index(" azimuthal averaged scattering matrix expansion coefficients, total field")
    assert L[i + 2][:33] == "    0" + es(gs["s00"][0], 14, 6) + es(gs["s00"][15], 14, 6)
    assert len(L) == i + 2 + 2 * sc["t_matrix_order"] + 1
    rand = I.execute(runs[1], "fp64")
    rt = o.tmatrix_solution(convergence_eps=1e-8, solution_eps=1e-12)
    assert rand["t_matrix_order"] == rt["order"]
    assert np.allclose(rand["qtot"], rt["qtot"], rtol=1e-9)
    assert "asymmetry parameter" in I.report(rand) and "efficiencies" in I.report(fixed)
    # the reference-layout output file of both runs
    from mstm_b200.output import write_output, es
    p = tmp_path / "out.dat"
    write_output(str(p), [(dict(runs[0], _run_number=1), fixed), (dict(runs[1], _run_number=2), rand)])
    text = p.read_text().splitlines()
    assert text.count(" calculation results for run ") == 2
    i = text.index(" total extinction, absorption, scattering efficiencies (unpol, par, perp incidence)")
    assert text[i + 1][:12] == es(ro["qtot"][0, 0])
    i = text.index(" total extinction, absorption, scattering efficiencies (unpolarized incidence)")
    assert text[i + 1][:12] == es(rt["qtot"][0])


def test_fortran_edit_descriptors():
    from mstm_b200.output import es, fd, iw
    assert es(0.0) == "  0.0000E+00" and es(-1.0) == " -1.0000E+00" and es(12.3456789) == "  1.2346E+01"
    assert es(9.99996) == "  1.0000E+01" and es(1.0e100) == "  1.0000+100" and es(-2.5e-101) == " -2.5000-101"
    assert es(1.23456789, 15, 7) == "  1.2345679E+00" and es(5.0, 14, 6) == "  5.000000E+00"
    assert fd(-180.0, 8, 2) == " -180.00" and fd(3.14159, 8, 3) == "   3.142" and iw(42, 6) == "    42"


def test_output_blocks_layout():
    """The run-variable and result blocks in the reference's record layout
    (labels, record order, field widths) for a synthetic fixed-orientation
    and random-orientation result."""
    from mstm_b200 import output as O
    run = I.parse(DECK)[0]
    n = 3
    fixed = dict(kind="fixed_orientation", run_number=1, neqns=210, max_mie_order=5, mean_mie=(2.0, 0.1), vol_radius=1.44,
                 sinc=0.0, direction=1, t_matrix_order=8, iterations_max=12, error_max=3e-13, solution_time=0.01,
                 sphere_qeff_unpol=np.ones((n, 3)), qtot=np.arange(9.0).reshape(3, 3, order="F") + 1,
                 theta=np.linspace(-180, 180, 361), smat=np.tile(np.eye(4), (361, 1, 1)))
    L = O.run_variables(run, fixed) + O.calculation_results(run, fixed)
    assert L[0] == "*" * 52 and L[1] == " input variables for run     1"
    i = L.index(" number spheres")
    assert L[i + 1] == "      3"
    i = L.index(" calculation results for run ")
    assert L[i + 1].strip() == "1"
    i = L.index(" number iterations, error, solution time ")
    assert L[i + 1] == "    12  3.0000E-13  1.0000E-02"
    i = L.index(" total extinction, absorption, scattering efficiencies (unpol, par, perp incidence)")
    assert L[i + 1] == "".join(O.es(v) for v in range(1, 10))
    i = L.index(" scattering matrix in incident plane: 0 deg= z axis")
    assert L[i + 2] == "   361    16" and L[i + 3].startswith("   theta     11          12     ")
    assert L[i + 4].startswith(" -180.00") and len(L[i + 4]) == 8 + 16 * 12
    # S11 scaled by 1/(pi r^2 Qsca), the rest divided by S11
    assert abs(float(L[i + 4][8:20]) - 1.0 / (1.44 ** 2 * O.REF_PI * 3.0)) < 1e-4 / (1.44 ** 2 * O.REF_PI * 3.0)
    rnd = dict(fixed, kind="random_orientation", t_matrix_order_estimate=9, qtot=np.array([3.0, 0.5, 2.5]),
               theta=np.linspace(0, 180, 181), smat=np.tile(np.eye(4), (181, 1, 1)),
               sm_coef=np.ones((17, 4, 4)), smcf_coef=np.ones((17, 4, 4)))
    rrun = I.parse(DECK)[1]
    L = O.run_variables(rrun, rnd) + O.calculation_results(rrun, rnd)
    assert " random orientation, estimated t matrix order:" in L and " calculated t matrix order:" in L
    i = L.index(" total scattering")
    assert L[i + 2] == "   181     6" and L[i + 3] == "   theta     11          12          22          33          34          44     "
    i = L.index(" orientation averaged scattering matrix expansion coefficients")
    assert L[i + 2] == "    0" + O.es(1.0, 14, 6) * 6 and len(L) == i + 2 + 17 + 2 + 17
