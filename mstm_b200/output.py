"""The reference's output file for a run of the solver path: the run-variable
block of print_run_variables (mstm-input-37.f90:3137-3304) and the results
block of print_calculation_results (mstm-input-37.f90:3340-3751), with the
same labels, record order and Fortran edit descriptors, for the branches this
library covers (no plane boundaries, periodic lattices, configuration or
incidence averages, near fields or Gaussian beams).  Not written: the down and
up hemispherical scattering efficiencies (`calculate_up_down_scattering`,
default on in the reference), which the reference computes with its
plane-boundary routines (sphere_boundary_scattering), outside this path; a
deck with `calculate_up_down_scattering f` gives the reference's records.
"""
import math

import numpy as np

REF_PI = 3.1415927410125732   # the reference's pi constant (single-precision literal)


# ---- Fortran edit descriptors -------------------------------------------------
def es(x, w=12, d=4):
    """ESw.d: one nonzero digit before the point, d after, a 2- or 3-digit
    exponent (E+dd, or +ddd without the E once |exponent| > 99)."""
    x = float(x)
    if not math.isfinite(x):
        return ("NaN" if x != x else ("Infinity" if x > 0 else "-Infinity")).rjust(w)
    s = f"{x:.{d}E}"
    mant, ex = s.split("E")
    e = int(ex)
    if abs(e) <= 99:
        t = f"{mant}E{'+' if e >= 0 else '-'}{abs(e):02d}"
    else:
        t = f"{mant}{'+' if e >= 0 else '-'}{abs(e):03d}"
    return t.rjust(w) if len(t) <= w else "*" * w


def fd(x, w, d):
    """Fw.d"""
    t = f"{float(x):.{d}f}"
    return t.rjust(w) if len(t) <= w else "*" * w


def iw(n, w):
    """Iw"""
    t = str(int(n))
    return t.rjust(w) if len(t) <= w else "*" * w


def line(*fields):
    """A record: Fortran writes a leading blank only in list-directed and
    quoted-label records; edit-descriptor records start with their field."""
    return "".join(fields)


def label(text):
    return " " + text


def listed_int(n):
    """List-directed output of one default integer."""
    return f"{int(n):12d}"


# ---- geometry and Mie summaries as the reference forms them -------------------
def cluster_radii(pos, rad, host=None):
    """(volume radius, area-mean radius, circumscribing radius) as spheredata's
    set-up forms them (mstm-modules-33.f90:5257-5379): circumscribing about the
    mean position of the spheres outside every other; the volume and
    area-mean radii over those spheres (host: the holding sphere of each
    sphere, -1 for none; None: every sphere is outside)."""
    pos = np.asarray(pos, np.float64).reshape(-1, 3)
    rad = np.asarray(rad, np.float64)
    out = np.ones(len(rad), bool) if host is None else (np.asarray(host) < 0)
    vol = float(np.sum(rad[out] ** 3) ** (1.0 / 3.0))
    area = float(math.sqrt(np.mean(rad[out] ** 2)))
    org = pos[out].mean(axis=0)
    circ = float(np.max(np.sqrt(((pos - org) ** 2).sum(axis=1)) + rad))
    return vol, area, circ


def mean_mie(rad, qext, qabs, host=None):
    """Area-weighted mean Mie efficiencies of the spheres outside every other
    (mstm-modules-33.f90:5364-5379)."""
    rad = np.asarray(rad, np.float64)
    out = np.ones(len(rad), bool) if host is None else (np.asarray(host) < 0)
    r, qe, qa = rad[out], np.asarray(qext)[out], np.asarray(qabs)[out]
    a2 = float(np.mean(r ** 2))
    return float(np.sum(qe * r ** 2) / a2 / len(r)), float(np.sum(qa * r ** 2) / a2 / len(r))


def scaled_scat_mat(s):
    """scaled_scat_mat: S11 kept, the other 15 elements divided by S11."""
    s = np.asarray(s, np.float64).reshape(16)
    if s[0] == 0.0:
        return np.zeros(16)
    out = s.copy()
    out[1:] = s[1:] / s[0]
    return out


SMVEC = (1, 5, 6, 11, 15, 16)
SMVEC0 = (1, 5, 9, 13, 2, 6, 10, 14, 3, 7, 11, 15, 4, 8, 12, 16)
SMLABEL = ("11", "21", "31", "41", "12", "22", "32", "42", "13", "23", "33", "43", "14", "24", "34", "44")


def output_header(input_file, when=None):
    """output_header (mstm-input-37.f90:3120-3135): written once at the top of
    an output file."""
    import datetime
    t = when or datetime.datetime.now()
    stamp = t.strftime("%Y%m%d") + " " + t.strftime("%H%M%S.") + "%03d" % (t.microsecond // 1000)
    return ["*" * 52, "*" * 52, label("mstm calculation results"), label("date, time:"), stamp, label("input file:"), input_file]


def run_variables(run, out):
    """print_run_variables for one run: a list of records."""
    from .inputfile import cluster_arrays, medium_index
    pos, rad, ri = cluster_arrays(run)
    n = len(rad)
    host = out.get("host")
    vol, area, circ = cluster_radii(pos, rad, host)
    med = medium_index(run)
    L = ["*" * 52, label(f"input variables for run {iw(out.get('run_number', 1), 5)}")]
    L += [label("sphere data input file:"), run["sphere_data_input_file"] or ""]
    L += [label("number spheres"), iw(n, 7)]
    L += [label("length, ref index scale factors"),
          es(run["length_scale_factor"], 15, 7) + es(complex(run["ref_index_scale_factor"]).real, 15, 7)
          + es(complex(run["ref_index_scale_factor"]).imag, 15, 7)]
    L += [label("volume cluster radius, area mean sphere radius, circumscribing radius, cross section radius"),
          es(vol, 15, 7) + es(area, 15, 7) + es(circ, 15, 7) + es(vol, 15, 7)]
    if run.get("print_sphere_data", True):
        L += [label("sphere properties and associations"),
              label("  sphere    host   layer radius     x       y       z           ref indx")]
        for i in range(n):
            h = 0 if host is None else int(host[i]) + 1   # 1-based, 0 outside every sphere
            L.append(iw(i + 1, 8) + iw(h, 8) + iw(0, 8) + fd(rad[i], 8, 3) + fd(pos[i, 0], 8, 3) + fd(pos[i, 1], 8, 3)
                     + fd(pos[i, 2], 8, 3) + es(ri[i].real) + es(ri[i].imag))
    if out["kind"] == "random_orientation":
        L += [label("random orientation, estimated t matrix order:"), iw(out["t_matrix_order_estimate"], 6)]
    else:
        L.append(label("incident plane wave"))
        if "incident_beta_deg" in run.get("_specified", ()):
            L += [label("incident alpha, beta(deg)"), es(run["incident_alpha_deg"]) + es(run["incident_beta_deg"])]
        else:
            L += [label("incident alpha(deg), incident sin(beta), incident direction"),
                  es(run["incident_alpha_deg"]) + es(out.get("sinc", 0.0)) + iw(3 - 2 * out.get("direction", 1), 3)]
        if "t_matrix_order" in out:
            L += [label("t matrix order:"), iw(out["t_matrix_order"], 6)]
    L += [label("layer 0 refractive index"), es(med.real) + es(med.imag)]
    L += [label("number of plane boundaries "), iw(0, 3)]
    L += [label("max_iterations,solution_epsilon, mie_epsilon, interaction radius"),
          iw(run["max_iterations"], 10) + es(run["solution_epsilon"]) + es(run["mie_epsilon"]) + es(1.0e10)]
    L += [label("maximum Mie order, number of equations:"), iw(out["max_mie_order"], 4) + iw(out["neqns"], 10)]
    qe, qa = out["mean_mie"]
    L += [label("mean sphere Mie extinction, absorption efficiencies, albedo"), es(qe) + es(qa) + es(1.0 - qa / qe if qe else 0.0)]
    if "fft_grid" in out:
        fg = out["fft_grid"]
        L += [label("fft translation option implemented"), label("cell width, cell volume fraction, cell dimension:"),
              "".join(iw(v, 8) for v in fg["cell_dim"]) + es(run["cell_volume_fraction"]) + es(fg["d_cell"]),
              label("number of neighbor nodes, node order:"),
              iw({0: 1, 1: 7, 2: 19}.get(run["neighbor_node_model"], 19), 5) + iw(fg["node_order"], 5)]
    L += ["*" * 52, label("calculation results for run "), listed_int(out.get("run_number", 1))]
    return L


def calculation_results(run, out):
    """print_calculation_results for one run: a list of records."""
    L = [label("number iterations, error, solution time "),
         iw(out["iterations_max"], 6) + es(out["error_max"]) + es(out["solution_time"])]
    random = out["kind"] == "random_orientation"
    if random:
        L += [label("calculated t matrix order:"), iw(out["t_matrix_order"], 6)]
    if run.get("print_sphere_data", True):
        L += [label("sphere extinction, absorption, volume absorption efficiencies (unpolarized incidence)"),
              label("  sphere   Qext        Qabs        Qvabs")]
        sq = out["sphere_qeff_unpol"]   # (N, 3): ext, abs, sca
        for i in range(sq.shape[0]):
            L.append(iw(i + 1, 8) + es(sq[i, 0]) + es(sq[i, 1]) + es(sq[i, 1]))
    q = np.asarray(out["qtot"])
    if random:
        L += [label("total extinction, absorption, scattering efficiencies (unpolarized incidence)"), "".join(es(v) for v in q[:3])]
    else:
        L += [label("total extinction, absorption, scattering efficiencies (unpol, par, perp incidence)"),
              "".join(es(q[r, c]) for c in range(3) for r in range(3))]
    if "smat" in out:
        vol = out["vol_radius"]
        qsca = float(q[2] if random else q[2, 0])
        s11scale = 1.0 / (vol ** 2 * REF_PI * qsca) if run.get("normalize_s11", True) else 2.0 * REF_PI
        six = random or run["azimuthal_average"]
        vec = SMVEC if six else SMVEC0
        if random:
            L.append(label("total scattering"))
        elif run["azimuthal_average"]:
            L.append(label("azimuthal averaged scattering matrix"))
        else:
            L.append(label("scattering matrix in incident plane: 0 deg= z axis"))
        sm, theta = out["smat"], out["theta"]
        L += [label("number directions, number SM elements:"), iw(sm.shape[0], 6) + iw(len(vec), 6),
              "   theta" + "".join("     " + SMLABEL[k - 1] + "     " for k in vec)]
        for i in range(sm.shape[0]):
            smt = scaled_scat_mat(np.asarray(sm[i]).reshape(4, 4).T.reshape(16))   # Fortran sm(4,4) order
            smt[0] *= s11scale
            L.append(fd(theta[i], 8, 2) + "".join(es(smt[k - 1]) for k in vec))
        if (not random) and run["azimuthal_average"] and "gsf" in out:
            c = out["gsf"]   # (2T+1, 4, 4) [w][i][j] each
            L += [label("azimuthal averaged scattering matrix expansion coefficients, total field"),
                  "    n         11            44            12            34           22p           22m"]
            for nn in range(c["s00"].shape[0]):
                L.append(iw(nn, 5) + es(c["s00"][nn, 0, 0], 14, 6) + es(c["s00"][nn, 3, 3], 14, 6)
                         + es(0.5 * (c["s02"][nn, 1, 0] + c["s02"][nn, 0, 1]), 14, 6)
                         + es(0.5 * (c["s02"][nn, 3, 2] + c["s02"][nn, 2, 3]), 14, 6)
                         + es(c["sp22"][nn, 1, 1], 14, 6) + es(c["sm22"][nn, 1, 1], 14, 6))
        if random:
            hdr = "    n         11            44            12            34           22            33"
            for title, key in (("orientation averaged scattering matrix expansion coefficients", "sm_coef"),
                               ("orientation averaged coherent scattering matrix expansion coefficients", "smcf_coef")):
                c = out[key]   # (2T+1, 4, 4) [n][i][j]
                L += [label(title), hdr]
                for nn in range(c.shape[0]):
                    L.append(iw(nn, 5) + es(c[nn, 0, 0], 14, 6) + es(c[nn, 3, 3], 14, 6) + es(c[nn, 0, 1], 14, 6)
                             + es(c[nn, 2, 3], 14, 6) + es(c[nn, 1, 1], 14, 6) + es(c[nn, 2, 2], 14, 6))
    return L


def write_output(path, runs_out, append=False):
    """Write (or append) the run-variable and result blocks of every run."""
    with open(path, "a" if append else "w") as f:
        for run, out in runs_out:
            for rec in run_variables(run, out) + calculation_results(run, out):
                f.write(rec + "\n")
