"""MSTM input files on this path: read the reference's input deck
(keyword line, value line; `sphere_data` ... `end_of_sphere_data`;
`new_run` between runs, `end_of_options` at the end, `loop_variable`
sweeps; `!` comments; Fortran literals such as
`1.d-15`, `(1.6d0,0.d0)`, `t` / `f`), as variable_list_operation and
inputdata read it (mstm-input-37.f90:148-933), and run the options of the
solver path through the library:

  fixed orientation   fixedorsoln + qtotcalc (+ scattering_matrix_calculation
                      with 181 polar angles when calculate_scattering_matrix)
  random_orientation  tmatrix_solution + ranorientscatmatrix (+ the scattering
                      matrix at 181 angles)
  fft_translation_option  the FFT translation for clusters of at least
                      min_fft_nsphere spheres (input:1114)

Spheres inside other spheres are detected by the library (host spheres) and
solved with their couplings.  Options outside this path (plane boundaries,
periodic lattices, near fields, Gaussian beams, random configurations, ...)
are rejected with a clear error rather than ignored.

    python -m mstm_b200.inputfile run.inp [--precision fp64|mixed]
"""
import math
import time
import re
import sys

import numpy as np

REF_PI = 3.1415927410125732   # pi as the reference stores it (a default-real literal)

# option -> (type, default); types: i int, r real, c complex, l logical, a string
OPTIONS = {
    "output_file": ("a", "mstm_output.dat"),
    "number_spheres": ("i", 0),
    "sphere_data_input_file": ("a", ""),
    "length_scale_factor": ("r", 1.0),
    "ref_index_scale_factor": ("r", 1.0),
    "medium_ref_index": ("c", 1.0 + 0.0j),
    "medium_re_ref_index": ("r", None),
    "medium_im_ref_index": ("r", None),
    "mie_epsilon": ("r", 1.0e-6),
    "translation_epsilon": ("r", 1.0e-5),
    "solution_epsilon": ("r", 1.0e-6),
    "max_iterations": ("i", 10000),
    "max_t_matrix_order": ("i", 100),
    "random_orientation": ("l", False),
    "t_matrix_convergence_epsilon": ("r", 1.0e-6),
    "fft_translation_option": ("l", False),
    "min_fft_nsphere": ("i", 200),
    "node_order": ("i", -1),
    "neighbor_node_model": ("i", 2),
    "cell_volume_fraction": ("r", 0.0),
    "d_cell": ("r", None),
    "incident_beta_deg": ("r", 0.0),
    "incident_alpha_deg": ("r", 0.0),
    "calculate_scattering_matrix": ("l", True),
    "azimuthal_average": ("l", False),
    "scattering_map_increment": ("r", 1.0),
    "print_sphere_data": ("l", True),
    "normalize_s11": ("l", True),
    "store_translation_matrix": ("l", True),
    "solution_method": ("a", "iterative"),
    "t_matrix_output_file": ("a", ""),
    "append_output_file": ("l", False),
    # accepted; their output blocks are not written (see output.py)
    "calculate_up_down_scattering": ("l", True),
    "print_timings": ("l", True),
    "number_configurations": ("i", 0),   # used only with configuration_average (rejected)
}
# options accepted only at values that keep the run on this path
RESTRICTED = {
    "number_plane_boundaries": ("i", 0),
    "periodic_lattice": ("l", False),
    "calculate_near_field": ("l", False),
    "gaussian_beam_constant": ("r", 0.0),
    "random_configuration": ("l", False),
    "random_configuration_host": ("l", False),
    "configuration_average": ("l", False),
    "incidence_average": ("l", False),
    "incident_frame": ("l", False),
    "scattering_map_model": ("i", 0),
    "single_origin_expansion": ("l", True),
    "numerical_azimuthal_average": ("l", False),
    "interaction_radius": ("r", 1.0e10),
    "normalize_solution_error": ("l", True),
}


def _real(s):
    return float(s.strip().lower().replace("d", "e"))


def _complex(s):
    s = s.strip()
    m = re.fullmatch(r"\(\s*([^,]+)\s*,\s*([^)]+)\s*\)", s)
    if m:
        return complex(_real(m.group(1)), _real(m.group(2)))
    return complex(_real(s), 0.0)


def _logical(s):
    v = s.strip().lower().strip(".")
    if v in ("t", "true"):
        return True
    if v in ("f", "false"):
        return False
    raise ValueError(f"not a logical: {s!r}")


def _convert(kind, s):
    s = s.strip()
    if kind == "i":
        return int(_real(s))
    if kind == "r":
        return _real(s)
    if kind == "c":
        return _complex(s)
    if kind == "l":
        return _logical(s)
    return s


def _split_items(line):
    """Fortran list-directed items: commas or blanks separate, parentheses group."""
    out, cur, depth = [], "", 0
    for ch in line:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if depth == 0 and (ch == "," or ch.isspace()):
            if cur:
                out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur:
        out.append(cur)
    return out


def parse_sphere_line(line):
    """x, y, z, r, then the index as one complex item or as re, im (default 1)."""
    it = _split_items(line)
    if len(it) < 4:
        raise ValueError(f"sphere line needs x, y, z, radius: {line!r}")
    x, y, z, r = (_real(v) for v in it[:4])
    if len(it) == 4:
        ri = 1.0 + 0.0j
    elif len(it) == 5:
        ri = _complex(it[4])
    else:
        ri = complex(_real(it[4]), _real(it[5]))
    return x, y, z, r, ri


def _loop_values(kind, start, stop, step, limit=100000):
    """The values nested_loop (mstm-main-3.f90:110-179) gives a loop variable:
    start, start+step, ... while |v - start| does not exceed |stop - start| by
    more than 1e-6; returns (values, the value the variable is left with)."""
    dist = (lambda a, b: abs(a - b))
    maxdif = dist(stop, start)
    if step == 0:
        raise ValueError("loop_variable with a zero step")
    vals, v = [], start
    while True:
        vals.append(v)
        v = v + step
        if dist(v, start) - maxdif > 1.0e-6:
            return vals, v
        if len(vals) >= limit:
            raise ValueError("loop_variable gives more than %d runs" % limit)


def parse(text):
    """The runs of an input deck, each a dict of options plus `spheres` (the
    sphere_data lines).  As inputdata reads it (mstm-input-37.f90:736-933):
    `new_run` ends a run and the next one starts from the same settings;
    `end_of_options` ends the input (anything after it is not read);
    `loop_variable name` + `start, stop, step` repeats the run over the
    values (nested loops in the order declared, the first outermost; the
    variable keeps the value past the end, as the reference leaves it);
    `run_file` names the run log."""
    lines = [ln.rstrip("\n") for ln in text.splitlines()]
    runs, cur = [], {k: v for k, (t, v) in OPTIONS.items()}
    cur["_specified"] = ()
    cur.update({k: v for k, (t, v) in RESTRICTED.items()})
    cur["run_file"] = ""
    spheres = []
    loops = []
    i = 0

    def nextval():
        nonlocal i
        while i < len(lines):
            v = lines[i].strip()
            i += 1
            if v and v[0] not in "!%":
                return v
        raise ValueError("unexpected end of input file")

    def finish_run():
        nonlocal loops
        base = dict(cur, spheres=list(spheres))
        combos = [dict()]
        for name, kind, start, stop, step in loops:
            vals, after = _loop_values(kind, start, stop, step)
            combos = [dict(c, **{name: v}) for c in combos for v in vals]
            cur[name] = after
        for c in combos:
            r = dict(base, **c)
            if c:
                r["_loop"] = dict(c)
            runs.append(r)
        loops = []

    ended = False
    while i < len(lines):
        key = lines[i].strip().lower()
        i += 1
        if not key or key[0] in "!%":
            continue
        if key == "new_run":
            finish_run()
            continue
        if key == "end_of_options":
            finish_run()
            ended = True
            break
        if key == "run_file":
            cur["run_file"] = nextval()
            continue
        if key == "loop_variable":
            name = nextval().lower()
            if name == "sphere_number":
                raise NotImplementedError("loop_variable over a per-sphere quantity is outside this path")
            if name not in OPTIONS or OPTIONS[name][0] not in "irc":
                raise NotImplementedError(f"loop_variable {name!r}: not a numeric option of this path")
            kind = OPTIONS[name][0]
            it = _split_items(nextval())
            if len(it) < 3:
                raise ValueError(f"loop_variable {name}: needs start, stop, step")
            start, stop, step = (_convert(kind, v) for v in it[:3])
            loops.append((name, kind, start, stop, step))
            cur["_specified"] = tuple(sorted(set(cur.get("_specified", ())) | {name}))
            continue
        if key == "sphere_data":
            spheres = []
            while i < len(lines):
                v = lines[i].strip()
                i += 1
                if v.lower() in ("end_of_sphere_data",):
                    break
                if v.lower() == "end_of_options":
                    i -= 1
                    break
                if not v or v[0] in "!%":
                    continue
                spheres.append(parse_sphere_line(v))
            continue
        if key in OPTIONS:
            cur[key] = _convert(OPTIONS[key][0], nextval())
            cur["_specified"] = tuple(sorted(set(cur.get("_specified", ())) | {key}))
        elif key in RESTRICTED:
            cur[key] = _convert(RESTRICTED[key][0], nextval())
        else:
            raise NotImplementedError(f"input option {key!r} is outside the multiple-sphere solve this library replaces")
    if not ended:
        finish_run()   # a file without end_of_options ends as if it had one (mstm-main-3.f90:47)
    return runs


def check_supported(run):
    for k, (t, ok) in RESTRICTED.items():
        if run[k] != ok:
            raise NotImplementedError(f"{k} = {run[k]!r} is outside the multiple-sphere solve this library replaces")
    if run["solution_method"].strip().lower()[:1] not in ("i", ""):
        raise NotImplementedError("only the iterative solution method is on this path")


def cluster_arrays(run):
    """Positions and radii scaled by length_scale_factor, indices by
    ref_index_scale_factor; the sphere count limited to number_spheres."""
    sp = run["spheres"]
    if run["sphere_data_input_file"]:
        with open(run["sphere_data_input_file"]) as f:
            sp = [parse_sphere_line(ln) for ln in f if ln.strip() and ln.strip()[0] not in "!%"]
    n = run["number_spheres"] if run["number_spheres"] > 0 else len(sp)
    sp = sp[:n]
    if len(sp) < n:
        raise ValueError(f"number_spheres {n} but {len(sp)} sphere lines")
    a = np.array([[s[0], s[1], s[2], s[3]] for s in sp], np.float64) * run["length_scale_factor"]
    ri = np.array([s[4] for s in sp], np.complex128) * run["ref_index_scale_factor"]
    return a[:, :3].copy(), a[:, 3].copy(), ri


def medium_index(run):
    m = complex(run["medium_ref_index"])
    if run["medium_re_ref_index"] is not None:
        m = complex(run["medium_re_ref_index"], m.imag)
    if run["medium_im_ref_index"] is not None:
        m = complex(m.real, run["medium_im_ref_index"])
    return m


def incidence(run, medium):
    """(alpha, sin beta, direction) as main_calling_program forms them (input:1311-1328)."""
    beta = run["incident_beta_deg"]
    direction = 1 if beta <= 90.0 else 2
    sinc = math.sin(beta * REF_PI / 180.0) / medium.real
    return run["incident_alpha_deg"] * REF_PI / 180.0, sinc, direction


def execute(run, precision="fp64"):
    """Run one deck entry on the GPU; returns a dict of results.  The
    scattering-matrix directions follow main_calling_program
    (input:1300-1363): udim = floor(180.00001/scattering_map_increment) steps
    over 0..180 degrees for random orientation and for the azimuth-averaged
    fixed-orientation matrix, -180..180 in the plane of incidence otherwise."""
    from . import api
    check_supported(run)
    udim = int(math.floor(180.00001 / run["scattering_map_increment"]))
    nangles = udim + 1
    pos, rad, ri = cluster_arrays(run)
    med = medium_index(run)
    g = api.SphereCluster(pos, rad, ri, mie_epsilon=run["mie_epsilon"], precision=precision, medium_index=med)
    out = dict(number_spheres=len(rad), neqns=g.number_eqns, vol_radius=g.vol_radius, medium=med,
               max_mie_order=int(g.sphere_order.max()), run_number=run.get("_run_number", 1))
    _, mqe, mqa = g.miecoefcalc()
    host, nh = g.host_spheres()
    if nh > 0:
        out["host"] = host
    from .output import mean_mie
    out["mean_mie"] = mean_mie(rad, mqe, mqa, host if nh > 0 else None)
    t0 = time.perf_counter()
    try:
        if run["fft_translation_option"] and len(rad) >= run["min_fft_nsphere"]:
            d = run["d_cell"] if run["d_cell"] is not None else 0.0
            out["fft_grid"] = g.fft_setup(cell_volume_fraction=run["cell_volume_fraction"], d_cell=d,
                                          node_order=run["node_order"], neighbor_node_model=run["neighbor_node_model"])
        if run["random_orientation"]:
            T = g.t_matrix_order(trans_eps=run["translation_epsilon"], max_t_order=run["max_t_matrix_order"])
            r = g.tmatrix_solution(T, solution_eps=run["solution_epsilon"], convergence_eps=run["t_matrix_convergence_epsilon"],
                                   max_iterations=run["max_iterations"])
            out.update(solution_time=time.perf_counter() - t0, iterations_max=r["maxiter"], error_max=r["maxerr"],
                       t_matrix_order_estimate=T, sphere_qeff_unpol=np.asarray(r["sphere_qeff"]).T.copy())
            u = r["order"]
            nb = 2 * u * (u + 2)
            tm = np.asfortranarray(r["tmat"][:nb, :nb])
            out.update(kind="random_orientation", t_matrix_order=u, qtot=r["qtot"], sphere_qeff=r["sphere_qeff"],
                       maxiter=r["maxiter"], maxerr=r["maxerr"], istat=r["istat"])
            if run["t_matrix_output_file"]:
                from .tmatrix_file import write_tmatrix_file
                write_tmatrix_file(run["t_matrix_output_file"], r["tmat"], T, u)
            if run["calculate_scattering_matrix"]:
                ro = g.ranorientscatmatrix(tm, u, nangles=nangles)
                out.update(theta=np.linspace(0.0, 180.0, nangles), smat=ro["smat"], sm_coef=ro["sm"], smcf_coef=ro["smcf"],
                           coherent_ratio=ro["coherent"], g_asym=ro["sm"][1, 0, 0] / (3.0 * ro["sm"][0, 0, 0]))
        else:
            alpha, sinc, direction = incidence(run, med)
            r = g.fixedorsoln(eps=run["solution_epsilon"], niter=run["max_iterations"], alpha=alpha, sinc=sinc, direction=direction)
            out.update(kind="fixed_orientation", qtot=r["qtot"], qeff=r["qeff"], iterations=r["iterations"], maxerr=r["maxerr"],
                       istat=r["istat"], amnp=r["amnp"], sinc=sinc, direction=direction, solution_time=time.perf_counter() - t0,
                       iterations_max=r["maxiter"], error_max=r["maxerr"], sphere_qeff_unpol=np.asarray(r["qeff"])[:, 0, :].T.copy())
            if run["calculate_scattering_matrix"]:
                sc = g.scattering(r["amnp"], trans_eps=run["translation_epsilon"], max_t_order=run["max_t_matrix_order"],
                                  nangles=nangles)
                out.update(g_asym=sc["g"], t_matrix_order=sc["t_matrix_order"])
                if run["azimuthal_average"]:
                    out.update(theta=np.linspace(0.0, 180.0, nangles), smat=sc["smat"],
                               gsf=g.gsf_coefficients(sc["amnp0"], sc["t_matrix_order"]))
                else:
                    theta, sm = g.scattering_plane(sc["amnp0"], sc["t_matrix_order"], increment=run["scattering_map_increment"],
                                                   alpha=alpha)
                    out.update(theta=theta, smat=sm, amnp0=sc["amnp0"])
    finally:
        g.close()
    return out


def report(out):
    """Text summary of one run (efficiencies, asymmetry parameter, scattering matrix)."""
    L = [f"number of spheres {out['number_spheres']}, equations {out['neqns']}, volume-equivalent radius {out['vol_radius']:.6f}"]
    if "fft_grid" in out:
        fg = out["fft_grid"]
        L.append(f"fft translation: cell_dim {fg['cell_dim']}, d_cell {fg['d_cell']:.5f}, node order {fg['node_order']}, "
                 f"near pairs {fg['near_pairs']}")
    q = np.asarray(out["qtot"])
    if out["kind"] == "fixed_orientation":
        L.append(f"fixed orientation: iterations {out['iterations']}, max error {out['maxerr']:.3e}, status {out['istat']}")
        L.append("efficiencies (ext, abs, sca) for unpolarized, parallel, perpendicular incidence:")
        for k, nm in enumerate(("unpolarized", "par", "perp")):
            L.append(f"  {nm:12s} {q[0, k]:.8e} {q[1, k]:.8e} {q[2, k]:.8e}")
    else:
        L.append(f"random orientation: T-matrix order {out['t_matrix_order']}, max iterations {out['maxiter']}, status {out['istat']}")
        L.append(f"orientation-averaged efficiencies (ext, abs, sca): {q[0]:.8e} {q[1]:.8e} {q[2]:.8e}")
    if "smat" in out:
        L.append(f"asymmetry parameter {out['g_asym']:.8f}")
        L.append("scattering matrix (theta, S11, S12, S33, S34):")
        sm, theta = out["smat"], out["theta"]
        n = sm.shape[0]
        for i in range(0, n, max(1, (n - 1) // 18)):
            L.append(f"  {theta[i]:7.2f} {sm[i, 0, 0]:.6e} {sm[i, 0, 1]:.6e} {sm[i, 2, 2]:.6e} {sm[i, 2, 3]:.6e}")
    return "\n".join(L)


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="run an MSTM input file on the B200 solver")
    ap.add_argument("input")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    a = ap.parse_args(argv)
    with open(a.input) as f:
        runs = parse(f.read())
    from .output import output_header, write_output
    # run numbers restart, and a file starts with the header, whenever the
    # output file changes (mstm-main-3.f90:63-80)
    old, number = None, 0
    for run in runs:
        first = run["output_file"] != old
        if first:
            old, number = run["output_file"], 0
        number += 1
        run = dict(run, _run_number=number)
        out = execute(run, a.precision)
        print(report(out))
        if first:
            with open(run["output_file"], "a" if run["append_output_file"] else "w") as f:
                f.write("\n".join(output_header(a.input)) + "\n")
        # the run's blocks in the reference's layout (print_run_variables +
        # print_calculation_results)
        write_output(run["output_file"], [(run, out)], append=True)


if __name__ == "__main__":
    main(sys.argv[1:])
