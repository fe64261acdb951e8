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
end_of_options
random_orientation
t
t_matrix_convergence_epsilon
1.d-8
end_of_options
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


def test_options_outside_the_path_are_rejected():
    deck = "number_spheres\n1\nsphere_data\n0 0 0 1 1.5 0\nend_of_sphere_data\nnumber_plane_boundaries\n2\nend_of_options\n"
    run = I.parse(deck)[0]
    with pytest.raises(NotImplementedError):
        I.check_supported(run)
    with pytest.raises(NotImplementedError):
        I.parse("calculate_up_down_scattering\nt\n")


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
    ga = oracle_mod.gsf_scattering(sc["t_matrix_order"], sc["amnp0"], nangles=37)["smat"]
    assert fa["smat"].shape == (37, 4, 4) and np.abs(fa["smat"] - ga).max() <= 1e-8 * np.abs(ga[:, 0, 0]).max()
    rand = I.execute(runs[1], "fp64")
    rt = o.tmatrix_solution(convergence_eps=1e-8, solution_eps=1e-12)
    assert rand["t_matrix_order"] == rt["order"]
    assert np.allclose(rand["qtot"], rt["qtot"], rtol=1e-9)
    assert "asymmetry parameter" in I.report(rand) and "efficiencies" in I.report(fixed)
