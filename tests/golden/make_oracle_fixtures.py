"""Freeze the oracle's FP64 results on the benchmark workloads at full size.

The oracle (oracle/, a C restatement of MSTM's solver path) is run here, on
the CPU, on the same seeded configurations the benchmark solves on the GPU;
its outputs are stored under tests/golden/ so that the GPU tests and the
benchmark can state the error of every result against it without running
it again (a full solve takes minutes of CPU time).

Cases (all to the squared-norm criterion ||r||^2/||b||^2 < 1e-12 of
cbicg, mstm-solver-8.f90:763-767, 920-924):
  fractal500       500-monomer PCA aggregate (x = 2, m = 1.6+0.05i, Df 1.8,
                   kf 1.3, seed 2), fixedorsoln (solver:350-569), then
                   fosmexpansion / fosmcalc (scatprops:1750-1951) at 181 angles;
  cylinder_fft     RSA cylinder (aspect 1, fv 0.25, x = 1, m = 1.31, seed 3)
                   on the FFT translation path (fft:72-974; d_cell 4, node
                   order -1 + ceiling(d_cell), neighbour model 2);
  tmatrix100       100 spheres, x = 1.5, m = 1.6+0.005i, RSA in a sphere at
                   fv 0.20 (seed 4): tmatrix_solution (solver:22-332) with
                   t_matrix_convergence 1e-6, then ranorientscatmatrix
                   (scatprops:1963-2592);
  ensemble_tmatrix the two smallest configurations of the 256-configuration
                   T-matrix ensemble (50-400 spheres, seed 4), as tmatrix100;
  host1000         a host sphere (m = 1.33) holding 1000 inclusions (x = 0.5,
                   m = 1.6+0.05i, RSA at fv 0.15, seed 7; host radius the RSA
                   bounding radius): fixedorsoln with host spheres
                   (findhostspheres, external_to_internal_expansion,
                   modules:5230-5276, 6533-6608), orders from mie_epsilon 1e-6.

Stored per case: efficiencies (totals and per sphere), iteration counts,
per-sphere norms of the solution and the full blocks of a few spheres,
the scattering-matrix outputs, and for T matrices the column norms, the
diagonal and the first columns.  Large arrays are kept out (the full
solution of fractal500 is 3.2 MB).

Run:  python tests/golden/make_oracle_fixtures.py [--threads N] [--only case ...]
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

EPS = 1.0e-12
NANG = 181
KEEP_SPHERES = 4        # spheres whose full solution blocks are kept
KEEP_COLUMNS = 16       # leading T-matrix columns kept in full


def _sphere_norms(o, amnp):
    off = o.offset
    return np.array([[np.linalg.norm(amnp[off[i]:off[i + 1], p]) for p in range(amnp.shape[1])] for i in range(o.n)])


def fixed_case(name, pos, x, m, threads, fft=None):
    from oracle import oracle as O
    from mstm_b200 import configs as C
    n = len(pos)
    L = C.truncation_order(x)
    t0 = time.time()
    o = O.Oracle(pos, np.full(n, x), np.full(n, m), mie_eps=-L, store_matrix=True, nthreads=threads)
    grid = None
    if fft is not None:
        grid = o.fft_setup(**fft)
    r = o.fixedorsoln(eps=EPS, niter=10000)
    t1 = time.time()
    s = o.scattering(r["amnp"], nangles=NANG)
    amnp = r["amnp"]
    out = dict(pos=np.asarray(pos), x=x, m=m, order=L, eps=EPS, qtot=r["qtot"], qeff=r["qeff"], maxiter=r["maxiter"], iterations=np.array(r["iterations"]),
               maxerr=r["maxerr"], status=r["status"], sphere_norms=_sphere_norms(o, amnp),
               amnp_head=amnp[:o.offset[KEEP_SPHERES], :], g=s["g"], smat=s["smat"], t_matrix_order=s["t_matrix_order"],
               amnp0=s["amnp0"], solve_s=t1 - t0, threads=threads)
    if grid is not None:
        out.update(cell_dim=np.array(grid["cell_dim"]), d_cell=grid["d_cell"], node_order=grid["node_order"],
                   near_pairs=grid["npairs"])
    o.close()
    np.savez_compressed(os.path.join(HERE, "oracle_%s.npz" % name), **out)
    print("%s: N=%d Qext %.12f iterations %d, %.0f s" % (name, n, r["qtot"][0, 0], r["maxiter"], t1 - t0), flush=True)


def host_case(name, w, threads):
    from oracle import oracle as O
    t0 = time.time()
    o = O.Oracle(w["pos"], w["radius"], w["ref_index"], mie_eps=1.0e-6, store_matrix=True, nthreads=threads)
    r = o.fixedorsoln(eps=EPS, niter=10000)
    t1 = time.time()
    amnp = r["amnp"]
    out = dict(pos=np.asarray(w["pos"]), radius=w["radius"], ref_index=w["ref_index"], mie_eps=1.0e-6, eps=EPS, order=o.order,
               offset=o.offset, qtot=r["qtot"], qeff=r["qeff"], maxiter=r["maxiter"], iterations=np.array(r["iterations"]),
               maxerr=r["maxerr"], status=r["status"], sphere_norms=_sphere_norms(o, amnp), amnp_head=amnp[:o.offset[KEEP_SPHERES], :],
               solve_s=t1 - t0, threads=threads)
    o.close()
    np.savez_compressed(os.path.join(HERE, "oracle_%s.npz" % name), **out)
    print("%s: N=%d Qext %.12f iterations %s, %.0f s" % (name, len(w["radius"]), r["qtot"][0, 0], r["iterations"], t1 - t0), flush=True)


def tmatrix_case(name, pos, x, m, threads):
    from oracle import oracle as O
    from mstm_b200 import configs as C
    n = len(pos)
    L = C.truncation_order(x)
    t0 = time.time()
    o = O.Oracle(pos, np.full(n, x), np.full(n, m), mie_eps=-L, store_matrix=True, nthreads=threads)
    r = o.tmatrix_solution(solution_eps=EPS, convergence_eps=1.0e-6)
    t1 = time.time()
    u = r["order"]
    nb = 2 * u * (u + 2)
    tm = np.asfortranarray(r["tmat"][:nb, :nb])
    xv = o.vol_radius()
    qe, qs = O.tmatrix_qext_qsca(u, tm, xv)
    ro = O.ranorientscatmatrix(u, tm, nangles=NANG)
    out = dict(pos=np.asarray(pos), x=x, m=m, order=L, eps=EPS, t_matrix_order=r["tmo"], order_used=u, qtot=r["qtot"],
               sphere_qeff=r["sphere_qeff"], maxiter=r["maxiter"], maxerr=r["maxerr"], status=r["status"],
               col_norms=np.linalg.norm(tm, axis=0), diag=np.diag(tm).copy(), cols_head=tm[:, :KEEP_COLUMNS].copy(),
               qext_t=qe, qsca_t=qs, sm=ro["sm"], smcf=ro["smcf"], smat=ro["smat"], solve_s=t1 - t0, threads=threads)
    o.close()
    np.savez_compressed(os.path.join(HERE, "oracle_%s.npz" % name), **out)
    print("%s: N=%d order %d/%d Qext %.12f, %.0f s" % (name, n, u, r["tmo"], r["qtot"][0], t1 - t0), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", nargs="*", default=None)
    a = ap.parse_args()
    from mstm_b200 import configs as C
    want = (lambda k: a.only is None or k in a.only)
    if want("fractal500"):
        w = C.workload("fractal500")
        fixed_case("fractal500", w["pos"], 2.0, 1.6 + 0.05j, a.threads)
    if want("tmatrix100"):
        pos, _ = C.rsa_sphere(100, 1.5, 0.20, seed=4)
        tmatrix_case("tmatrix100", pos, 1.5, 1.6 + 0.005j, a.threads)
    if want("ensemble_tmatrix"):
        from mstm_b200 import ensemble as EN
        cfgs = EN.ensemble_configs(256, seed=4, nmin=50, nmax=400)
        small = sorted(range(len(cfgs)), key=lambda k: (cfgs[k]["n"], k))[:2]
        for k in small:
            tmatrix_case("ensemble_tmatrix_c%d" % k, cfgs[k]["pos"], 1.5, 1.6 + 0.005j, a.threads)
    if want("host1000"):
        host_case("host1000", C.host_inclusions(1000, 0.5, 0.15, seed=7), a.threads)
    if want("cylinder_fft"):
        pos, _ = C.rsa_cylinder(5000, 1.0, 0.25, 1.0, seed=3)
        fixed_case("cylinder_fft", pos, 1.0, 1.31 + 0j, a.threads, fft=dict(d_cell=4.0))


if __name__ == "__main__":
    main()
