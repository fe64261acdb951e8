"""Benchmark: fixed-orientation solves per second of MSTM's multiple-sphere
interaction solve on B200.

Workload (one step = one solve): a seeded particle-cluster fractal aggregate,
500 touching monomers, x = 2.0, m = 1.6+0.05i, Df = 1.8, kf = 1.3, incidence
along +z, both polarisations, direct pair translation, sphere order L = 9
(neqns = 99,000, 124,750 pairs).  A solve = pair-operator generation (FP64,
and FP32 for the tuned arm: every fixed-orientation solve regenerates them, as
the reference's initial_run does) + incident coefficients + both
polarisations solved to ||r||/||b|| < 1e-6 (MSTM solution_epsilon = 1e-12 in
its squared-norm test) + efficiencies (`value`); the end-to-end number
(`e2e`) adds, every step, the positions copied in from pinned host memory and
the solution and efficiencies copied back.

Arms:
  default            tuned path (mixed precision: FP32 GMRES cycles from FP64
                     true residuals, both polarisations in each pass), with
                     the plain FP64 drop-in path (the reference's BiCG step for
                     step) measured beside it;
  --impl reference   the CPU restatement of the reference (oracle/) on all host
                     cores: one complete FP64 solve of the same configuration
                     per timed step (its own BiCG iterations to the same
                     criterion).

Timing: CUDA events on the stream the library launches on, W untimed warm-up
solves, K timed solves; operators (2 GB FP64 + 1 GB FP32) exceed the 126 MB L2,
so every pass streams from HBM.  Under torchrun each rank solves its own
configuration (replicas, no data-path collective) and rank 0 reports the
maximum time over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

EPS = 1.0e-12          # squared-norm criterion: ||r||/||b|| < 1e-6
# DRAM bytes per byte of row records and vectors of the FP32 row-kernel
# translation pass of 2 columns, from the ncu capture of the 200-sphere
# aggregate (189.06 MB of 185.0 MB)
TRAFFIC_PER_ALG_BYTE = 189.06 / 185.0
NITER = 10000
WORKLOAD = "fractal500"
METRIC = "solves/s at 1e-6 residual (fractal aggregate N=500, x=2, both polarisations)"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(dist, x, device):
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(ws, steps, ms_total_max):
    """Whole-job throughput: the solves of all ranks over the slowest rank's time."""
    return ws * steps * 1000.0 / ms_total_max


def bench_config(ws):
    """The workload both arms time (the same dict in both lines)."""
    return {"workload": "fractal aggregate, 500 touching monomers, x=2.0, m=1.6+0.05i, Df=1.8, kf=1.3, "
                        "L=9, +z incidence, both polarisations",
            "neqns": 99000, "pairs": 124750, "residual": "||r||/||b|| < 1e-6 (squared-norm eps 1e-12)",
            "parallelism": "replicas" if ws > 1 else "single GPU",
            "l2": "operators (2 GB FP64 / 1 GB FP32) exceed the 126 MB L2; no flush needed"}


def oracle_fixture(name):
    """The oracle's frozen FP64 results for a workload (tests/golden, made by
    tests/golden/make_oracle_fixtures.py), or None."""
    path = os.path.join(ROOT, "tests", "golden", "oracle_%s.npz" % name)
    if not os.path.exists(path):
        return None
    return dict(np.load(path))


def rel_err(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


def errors_vs_oracle(qtot, smat, g, f):
    """Relative errors of a fixed-orientation result against the oracle's:
    each efficiency (unpolarised) and the 3 x 3 table, the 181-angle
    scattering matrix (of S11's largest value) and the asymmetry parameter.
    Qabs is compared relative to Qext (non-absorbing spheres have Qabs at
    rounding level, where a relative error means nothing)."""
    out = {"qext": abs(qtot[0, 0] / f["qtot"][0, 0] - 1), "qabs_of_qext": abs(qtot[1, 0] - f["qtot"][1, 0]) / abs(f["qtot"][0, 0]),
           "qsca": abs(qtot[2, 0] / f["qtot"][2, 0] - 1), "qtot_3x3": rel_err(qtot, f["qtot"])}
    if smat is not None:
        out["smat_of_s11max"] = float(np.abs(smat - f["smat"]).max() / np.abs(f["smat"][:, 0, 0]).max())
        out["g"] = abs(g / f["g"] - 1)
    return {k: float("%.3g" % v) for k, v in out.items()}


def workload_for_rank(rank):
    from mstm_b200 import configs as C
    w = C.workload(WORKLOAD)
    if rank > 0:
        w = dict(w)
        w["pos"] = C.pca_aggregate(500, w["x"], 1.8, 1.3, seed=2 + 1000 * rank)
    return w


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import torch
    from mstm_b200 import _lib, api
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = init_dist(ws, "nccl")
    L = _lib.lib()
    w = workload_for_rank(rank)
    stream = torch.cuda.current_stream(dev)

    def make(prec):
        g = api.SphereCluster(w["pos"], w["radius"], w["ref_index"], mie_epsilon=-w["order"], precision=prec,
                              device=local)
        _lib.check(L.mstmg_set_stream(g.ctx, ctypes.c_void_p(stream.cuda_stream)), "set_stream")
        return g

    ne = None
    results = {}
    for prec in ("mixed", "fp64"):
        g = make(prec)
        ne = g.number_eqns
        amnp = torch.zeros(2 * ne * 2, dtype=torch.float64, device=dev)
        qeff = torch.zeros(9 * g.number_spheres, dtype=torch.float64, device=dev)
        qtot = torch.zeros(9, dtype=torch.float64, device=dev)
        me, mi = ctypes.c_double(0.0), ctypes.c_int(0)

        def solve():
            st = L.mstmg_fixed_orientation(g.ctx, 0.0, 0.0, 1, EPS, NITER, ctypes.c_void_p(amnp.data_ptr()),
                                           ctypes.c_void_p(qeff.data_ptr()), ctypes.c_void_p(qtot.data_ptr()),
                                           ctypes.byref(me), ctypes.byref(mi))
            _lib.check(st, "fixed_orientation")
            return st

        for _ in range(args.warmup):
            solve()
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        clocks = ClockSampler(local)
        if prec == "mixed" and rank == 0:
            clocks.start()
        _lib.check(L.mstmg_set_timing(g.ctx, 1), "timing")
        l0 = L.mstmg_kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            st = solve()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        launches = L.mstmg_kernel_launches() - l0
        ms = e0.elapsed_time(e1)
        ck = clocks.stop() if (prec == "mixed" and rank == 0) else None
        k64, n64, k32, n32 = ctypes.c_double(0), ctypes.c_int(0), ctypes.c_double(0), ctypes.c_int(0)
        _lib.check(L.mstmg_kernel_time(g.ctx, ctypes.byref(k64), ctypes.byref(n64), ctypes.byref(k32), ctypes.byref(n32)),
                   "kernel_time")
        _lib.check(L.mstmg_set_timing(g.ctx, 0), "timing")
        stats = g.last_stats()
        ms_max = max_over_ranks(dist, ms, dev)
        q = qtot.cpu().numpy().reshape(3, 3, order="F")
        vs_oracle = None
        fx = oracle_fixture(WORKLOAD) if rank == 0 else None
        if fx is not None:
            sol = amnp.cpu().numpy().view(np.complex128).reshape(2, ne).T
            sc = g.scattering(np.asfortranarray(sol))
            vs_oracle = errors_vs_oracle(q, sc["smat"], sc["g"], fx)
        results[prec] = dict(ms_total=ms_max, ms_per_step=ms_max / args.steps, istat=st, maxerr=me.value, stats=stats,
                             qtot=q, launches=launches, k64=(k64.value, n64.value), k32=(k32.value, n32.value), clocks=ck,
                             bytes64=g.operator_bytes("fp64"), bytes32=g.operator_bytes("mixed"), nrhs_hint=None,
                             vs_oracle=vs_oracle)
        if prec == "mixed":
            # end to end through the public C ABI with host buffers: new
            # positions copied in from pinned host memory, results read back
            pos_h = torch.from_numpy(np.ascontiguousarray(w["pos"], dtype=np.float64)).pin_memory()
            amnp_h = torch.zeros(2 * ne * 2, dtype=torch.float64).pin_memory()
            qeff_h = torch.zeros(9 * g.number_spheres, dtype=torch.float64).pin_memory()
            qtot_h = torch.zeros(9, dtype=torch.float64).pin_memory()

            def solve_e2e():
                _lib.check(L.mstmg_ctx_set_positions(g.ctx, ctypes.c_void_p(pos_h.data_ptr())), "set_positions")
                _lib.check(L.mstmg_fixed_orientation(g.ctx, 0.0, 0.0, 1, EPS, NITER, ctypes.c_void_p(amnp_h.data_ptr()),
                                                     ctypes.c_void_p(qeff_h.data_ptr()), ctypes.c_void_p(qtot_h.data_ptr()),
                                                     ctypes.byref(me), ctypes.byref(mi)), "fixed_orientation")

            solve_e2e()
            torch.cuda.synchronize(dev)
            if dist is not None:
                dist.barrier()
            e0.record(stream)
            for _ in range(args.steps):
                solve_e2e()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms_e2e = max_over_ranks(dist, e0.elapsed_time(e1), dev)
            results["e2e"] = dict(ms=ms_e2e, h2d=pos_h.numel() * 8,
                                  d2h=(amnp_h.numel() + qeff_h.numel() + qtot_h.numel()) * 8)
        g.close()

    extras = run_extras(args, dev, stream) if (rank == 0 and ws == 1 and not args.no_extras) else None
    if rank == 0:
        line = report_line(args, ws, results, ne)
        if extras:
            line["other_workloads"] = extras
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_sample(threads=os.cpu_count() or 1)
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_extras(args, dev, stream):
    """Secondary workloads of the same path, each timed with CUDA events on the
    library's stream after one untimed warm-up: the FFT-translation cluster
    (5000 spheres in a cylinder, cell edge 4), one configuration of the
    T-matrix ensemble (100 spheres, x = 1.5), and the small 20-sphere cluster."""
    import torch
    from mstm_b200 import _lib, api
    from mstm_b200 import configs as C
    L = _lib.lib()
    out = {}

    def timed(fn, reps):
        """median over `reps` calls (one untimed call first), each bracketed by
        CUDA events on the library's stream"""
        fn()
        torch.cuda.synchronize(dev)
        r, ts = None, []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = fn()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts), r

    def cluster(pos, x, m, prec):
        n = len(pos)
        g = api.SphereCluster(pos, np.full(n, x), np.full(n, m), mie_epsilon=-C.truncation_order(x), precision=prec)
        _lib.check(L.mstmg_set_stream(g.ctx, ctypes.c_void_p(stream.cuda_stream)), "set_stream")
        return g

    # FFT translation cluster
    pos = C.rsa_cylinder(5000, 1.0, 0.25, 1.0, seed=3)
    pos = pos[0] if isinstance(pos, tuple) else pos
    row = {"workload": "5000 spheres, x=1.0, m=1.31, RSA in a cylinder (aspect 1) at fv 0.25, FFT translation, d_cell 4",
           "metric": "solves/s at 1e-6 residual (both polarisations)"}
    fx = oracle_fixture("cylinder_fft")
    for prec in ("mixed", "fp64"):
        g = cluster(pos, 1.0, 1.31 + 0j, prec)
        grid = g.fft_setup(d_cell=4.0)
        ms, r = timed(lambda: g.fixedorsoln(eps=EPS, niter=NITER), 2)
        row[prec] = {"solves_per_s": round(1000.0 / ms, 3), "ms": round(ms, 2), "qext": r["qtot"][0, 0], "iterations": r["iterations"]}
        if fx is not None:
            sc = g.scattering(r["amnp"])
            row[prec]["vs_oracle"] = errors_vs_oracle(r["qtot"], sc["smat"], sc["g"], fx)
        if prec == "mixed":
            # the matvec against the FFT path's algorithmic bytes: near-pair
            # operators (FP32) + the kernel spectra (complex64, read once) +
            # the node grids (written and read by the forward and inverse
            # transforms) + x read and y written, for the two columns of an
            # Arnoldi pass
            ms_pass = g.time_translation("mixed", 2, 10)
            near = g.operator_bytes("fp64")[0] / 2.0   # the near pairs' folded FP32 operator values (row records add padding)
            cdim, no = grid["cell_dim"], grid["node_order"]
            nodes = (2 * cdim[0]) * (2 * cdim[1]) * (2 * cdim[2])
            nbn = no * (no + 2)
            spectra = nodes * nbn * nbn * 2 * 8
            grids = 2 * 2 * nodes * nbn * 2 * 2 * 8
            vecs = 2 * g.number_eqns * 8 * 2
            alg = near + spectra + grids + vecs
            row["matvec"] = {"ms_per_pass_2_columns": round(ms_pass, 4), "algorithmic_bytes": alg,
                             "bytes": {"near_pair_operators": near, "kernel_spectra": spectra, "node_grids": grids, "vectors": vecs},
                             "achieved_gbs": round(alg / ms_pass / 1e6, 1), "frac_of_measured_hbm": round(alg / ms_pass / 1e6 / hbm_peak(), 4)}
        row["grid"] = grid
        g.close()
    row["qext_rel_diff"] = abs(row["mixed"]["qext"] / row["fp64"]["qext"] - 1)
    out["fft_cylinder5000"] = row
    # one T-matrix configuration of the ensemble
    pos, _ = C.rsa_sphere(100, 1.5, 0.20, seed=4)
    row = {"workload": "100 spheres, x=1.5, m=1.6+0.005i, RSA in a sphere at fv 0.20: cluster T matrix, "
                       "all 2Lc(Lc+2) columns to residual 1e-6 (solution_eps 1e-12), t_matrix_convergence 1e-6",
           "metric": "T matrices/s"}
    fx = oracle_fixture("tmatrix100")
    for prec, tcore in (("mixed", 0), ("mixed", -1), ("fp64", 0)):
        key = prec if (prec == "fp64" or tcore == 0) else "mixed_rotation_kernels"
        n = len(pos)
        g = api.SphereCluster(pos, np.full(n, 1.5), np.full(n, 1.6 + 0.005j), mie_epsilon=-C.truncation_order(1.5),
                              precision=prec, tensor_core=tcore)
        _lib.check(L.mstmg_set_stream(g.ctx, ctypes.c_void_p(stream.cuda_stream)), "set_stream")
        T = g.t_matrix_order()
        ms, r = timed(lambda: g.tmatrix_solution(T, solution_eps=1e-12, convergence_eps=1e-6), 1 if prec == "fp64" else 3)
        row[key] = {"tmatrices_per_s": round(1000.0 / ms, 4), "ms": round(ms, 1), "order": r["order"], "t_matrix_order": T,
                    "columns": 2 * r["order"] * (r["order"] + 2), "qext": r["qtot"][0], "maxiter": r["maxiter"]}
        if fx is not None:
            u = r["order"]
            nb = 2 * u * (u + 2)
            tm = np.asfortranarray(r["tmat"][:nb, :nb])
            ro = g.ranorientscatmatrix(tm, u)
            row[key]["vs_oracle"] = {
                "qext": float("%.3g" % abs(r["qtot"][0] / fx["qtot"][0] - 1)),
                "qsca": float("%.3g" % abs(r["qtot"][2] / fx["qtot"][2] - 1)),
                "tmat_col_norms": float("%.3g" % rel_err(np.linalg.norm(tm, axis=0), fx["col_norms"])),
                "ranorient_smat_of_s11max": float("%.3g" % (np.abs(ro["smat"] - fx["smat"]).max() / np.abs(fx["smat"][:, 0, 0]).max())),
                "order_used_equal": bool(u == int(fx["order_used"]))}
        if key == "mixed":
            # the tensor-core pass alone: its launches timed with CUDA events in one more solve
            _lib.check(L.mstmg_set_timing(g.ctx, 1), "timing")
            g.tmatrix_solution(T, solution_eps=1e-12, convergence_eps=1e-6)
            tms, tn = ctypes.c_double(0), ctypes.c_int(0)
            _lib.check(L.mstmg_kernel_time_tc(g.ctx, ctypes.byref(tms), ctypes.byref(tn)), "kernel_time_tc")
            _lib.check(L.mstmg_set_timing(g.ctx, 0), "timing")
            row[key]["tensor_core_passes"] = {"launches": tn.value, "ms_total": round(tms.value, 2),
                                              "ms_per_pass": round(tms.value / max(1, tn.value), 4)}
        g.close()
    row["qext_rel_diff"] = abs(row["mixed"]["qext"] / row["fp64"]["qext"] - 1)
    row["speedup_tensor_cores"] = round(row["mixed_rotation_kernels"]["ms"] / row["mixed"]["ms"], 2)
    out["tmatrix_cluster100"] = row
    # host spheres: one host sphere holding 1000 inclusions, the FP64 BiCG
    # (the solver the reference runs), against the oracle's frozen solve and
    # the oracle itself timed on this host's cores
    w = C.host_inclusions(1000, 0.5, 0.15, seed=7)
    row = {"workload": "a host sphere (m=1.33, radius %.3f, the RSA bounding radius) holding 1000 inclusions (x=0.5, "
                       "m=1.6+0.05i, RSA at fv 0.15, seed 7): fixed orientation, both polarisations to residual 1e-6, "
                       "FP64 BiCG and mixed GMRES, orders from mie_epsilon 1e-6" % w["radius"][0],
           "metric": "solves/s"}
    g = api.SphereCluster(w["pos"], w["radius"], w["ref_index"], mie_epsilon=1e-6, precision="fp64")
    _lib.check(L.mstmg_set_stream(g.ctx, ctypes.c_void_p(stream.cuda_stream)), "set_stream")
    ms, r = timed(lambda: g.fixedorsoln(eps=EPS, niter=NITER), 3)
    hosts, nh = g.host_spheres()
    row["fp64"] = {"solves_per_s": round(1000.0 / ms, 3), "ms": round(ms, 2), "qext": r["qtot"][0, 0], "iterations": r["iterations"],
                   "unknowns": g.number_eqns, "pairs_same_host": L.mstmg_npairs(g.ctx), "spheres_with_a_host": nh,
                   "ms_per_translation_pass_2_columns": round(g.time_translation("fp64", 2, 10), 4)}
    # the pass against HBM: the stored FP64 records (same-host pairs and the
    # host-to-inclusion regular translations) and the two columns in and out
    rec = g.operator_bytes("fp64")[0]
    alg = rec + 2 * 2 * g.number_eqns * 16
    pms = row["fp64"]["ms_per_translation_pass_2_columns"]
    row["fp64"]["pass_roofline"] = {"kernel": "translate_kernel<double, 64, 4> (order-generic, same-host pairs) + the host pairs' launch",
                                    "algorithmic_bytes": alg, "achieved_gbs": round(alg / pms / 1e6, 1),
                                    "frac_of_measured_hbm": round(alg / pms / 1e6 / hbm_peak(), 4),
                                    "bound": "instruction issue (profiles/translate_generic_fp64_host300.md)"}
    fx = oracle_fixture("host1000")
    if fx is not None:
        row["fp64"]["vs_oracle"] = {"qext": float("%.3g" % abs(r["qtot"][0, 0] / fx["qtot"][0, 0] - 1)),
                                    "qabs": float("%.3g" % abs(r["qtot"][1, 0] / fx["qtot"][1, 0] - 1)),
                                    "qeff_all": float("%.3g" % rel_err(r["qeff"], fx["qeff"])),
                                    "iterations_equal": bool(list(r["iterations"]) == list(fx["iterations"]))}
    g.close()
    # the mixed solve (FP32 GMRES passes, the host couplings in FP32, FP64 true residuals)
    g = api.SphereCluster(w["pos"], w["radius"], w["ref_index"], mie_epsilon=1e-6, precision="mixed")
    _lib.check(L.mstmg_set_stream(g.ctx, ctypes.c_void_p(stream.cuda_stream)), "set_stream")
    ms_m, rm = timed(lambda: g.fixedorsoln(eps=EPS, niter=NITER), 3)
    row["mixed"] = {"solves_per_s": round(1000.0 / ms_m, 3), "ms": round(ms_m, 2), "qext": rm["qtot"][0, 0],
                    "iterations_gmres_step_pairs": rm["iterations"],
                    "ms_per_translation_pass_2_columns": round(g.time_translation("mixed", 2, 10), 4)}
    if fx is not None:
        row["mixed"]["vs_oracle"] = {"qext": float("%.3g" % abs(rm["qtot"][0, 0] / fx["qtot"][0, 0] - 1)),
                                     "qabs_of_qext": float("%.3g" % abs((rm["qtot"][1, 0] - fx["qtot"][1, 0]) / fx["qtot"][0, 0])),
                                     "qeff_all_of_max": float("%.3g" % (np.abs(rm["qeff"] - fx["qeff"]).max() / np.abs(fx["qeff"]).max()))}
    g.close()
    import multiprocessing
    threads = multiprocessing.cpu_count()
    t0 = time.time()
    o = _oracle_for_host(w, threads)
    ro = o.fixedorsoln(eps=EPS, niter=NITER)
    o.close()
    row["oracle_cpu"] = {"s": round(time.time() - t0, 2), "threads": threads, "iterations": ro["iterations"],
                         "what": "the oracle's full FP64 solve (operators, BiCG, efficiencies) on this host's cores"}
    row["speedup_vs_oracle_cpu"] = {"fp64": round(row["oracle_cpu"]["s"] * 1000.0 / ms, 1),
                                    "mixed": round(row["oracle_cpu"]["s"] * 1000.0 / ms_m, 1)}
    out["host_spheres1000"] = row
    # the 20-sphere cluster (the reference's CPU-sized case)
    w = C.workload("cluster20")
    row = {"workload": "20 spheres, x=1.0, m=1.5+0.01i, RSA in a sphere at fv 0.10, both polarisations",
           "metric": "solves/s at 1e-6 residual"}
    for prec in ("mixed", "fp64"):
        g = cluster(w["pos"], 1.0, 1.5 + 0.01j, prec)
        ms, r = timed(lambda: g.fixedorsoln(eps=EPS, niter=NITER), 5)
        row[prec] = {"solves_per_s": round(1000.0 / ms, 2), "ms": round(ms, 3), "qext": r["qtot"][0, 0]}
        g.close()
    out["cluster20"] = row
    # learned warm start: the network trained on the solver's own solutions of
    # 20,000 seeded configurations (mstm_b200/data/warmstart_net.npz, made by
    # `python -m mstm_b200.warmstart --train 20000 --eval 1000`, whose held-out
    # results it carries), evaluated here live on the first 100 configurations
    # of the same held-out stream (seed 6)
    from mstm_b200 import warmstart as WS
    wpath = os.path.join(ROOT, "mstm_b200", "data", "warmstart_net.npz")
    if os.path.exists(wpath):
        net, meta = WS.load_net(wpath, dev)
        held = WS.solve_samples(WS.draw_configs(100, 6, workers=8))
        live = WS.evaluate(net, held)
        ws = {"n_train": meta.get("n_train"), "n_eval": meta.get("n_eval"), "epochs": meta.get("epochs"),
              "study": {k: meta[k] for k in meta if k.startswith("fallback_")},
              "live_n_eval": len(held), "live": live}
    else:
        ws = WS.study(n_train=120, n_eval=8, epochs=60, device=dev, log=None)
    ws["workload"] = ("held-out configurations of 100-300 spheres, x in [0.5, 2], m random, fv in [0.05, 0.3], "
                      "+z incidence, mixed precision to 1e-6 residual; network trained on the solver's own solutions; "
                      "iterations in GMRES step pairs over both polarisations, wall time including the network's inference")
    out["warm_start"] = ws
    # the orientation-averaged ensemble: configurations of 50-400 spheres
    # (x = 1.5, seed 4), each a cluster T matrix (tensor-core passes) and its
    # random-orientation averages; 8 of the 256 configurations, every 32nd by
    # size, so the sample spans the size range
    from mstm_b200 import ensemble as EN
    cfgs = EN.ensemble_configs(256, seed=4, nmin=50, nmax=400)
    by_size = sorted(range(len(cfgs)), key=lambda k: (cfgs[k]["n"], k))
    subset = [cfgs[k] for k in by_size[16::32]]
    EN.solve_one(cfgs[by_size[0]], "mixed", solution_eps=1e-12)   # warm-up (module load, first allocations)
    torch.cuda.synchronize(dev)
    tuner = EN.Autotuner(reps=2)
    ens = EN.solve_ensemble(subset, precision="mixed", workers=1, tuner=tuner, solution_eps=1e-12)
    s11 = ens["smat"][:, 0, 0]
    row = {"workload": "orientation-averaged ensemble: 256 seeded configurations of 50-400 spheres (uniform), x=1.5, "
                       "m=1.6+0.005i, RSA in a sphere at fv 0.20; timed here: 8 of them, every 32nd by size (%s spheres); "
                       "per configuration the cluster T matrix to residual 1e-6 (tensor-core passes) and its random-orientation "
                       "Qext/Qsca and scattering matrix" % [c["n"] for c in subset],
           "metric": "T matrices/s (wall clock, one after the other)",
           "tmatrices_per_s": round(ens["tmatrices_per_s"], 4), "wall_s": round(ens["wall_s"], 2),
           "orders": [r["order"] for r in ens["per_config"]], "qext_mean": ens["qext"], "qsca_mean": ens["qsca"],
           "s11_mean_every_10deg": [float("%.6g" % v) for v in s11[::10]], "tuning_s": round(ens["tune_s"], 2),
           "autotuner_chose": [dict(size=l["key"][0], best=l["best"], ms=round(l["best_ms"], 3)) for l in tuner.log]}
    errs = {}
    for k in by_size[:2]:   # the two smallest configurations against the oracle's frozen T matrices
        fx = oracle_fixture("ensemble_tmatrix_c%d" % k)
        if fx is None:
            continue
        r = EN.solve_one(cfgs[k], "mixed", solution_eps=1e-12)
        errs["c%d" % k] = {"n": cfgs[k]["n"], "qext": float("%.3g" % abs(r["qtot"][0] / fx["qtot"][0] - 1)),
                           "qsca": float("%.3g" % abs(r["qtot"][2] / fx["qtot"][2] - 1)),
                           "smat_of_s11max": float("%.3g" % (np.abs(r["smat"] - fx["smat"]).max() / np.abs(fx["smat"][:, 0, 0]).max())),
                           "order_used_equal": bool(r["order"] == int(fx["order_used"]))}
    row["vs_oracle"] = errs
    out["ensemble_tmatrix_cfg4"] = row
    # many small fixed-orientation configurations: one at a time against four streams
    rng = np.random.default_rng(11)
    small = [C.rsa_sphere(int(rng.integers(15, 41)), 1.0, 0.10, seed=300 + k)[0] for k in range(48)]
    EN.solve_fixed_ensemble(small[:4], 1.0, 1.5 + 0.01j, workers=1)

    def median_run(workers):
        # wall-clock rate of a sub-second run: the median of three runs (host
        # scheduling alone moves single runs by 2x here)
        runs = sorted((EN.solve_fixed_ensemble(small, 1.0, 1.5 + 0.01j, workers=workers) for _ in range(3)),
                      key=lambda f: f["solves_per_s"])
        return runs[1]

    f1 = median_run(1)
    f4 = median_run(4)
    EN.solve_fixed_ensemble_batched(small[:4], 1.0, 1.5 + 0.01j)
    fb = EN.solve_fixed_ensemble_batched(small, 1.0, 1.5 + 0.01j, reps=3)
    out["ensemble_fixed_small"] = {
        "workload": "48 configurations, 15-40 spheres (seeded), x=1.0, m=1.5+0.01i, RSA at fv 0.10: fixed orientation, "
                    "both polarisations to residual 1e-6 (mixed precision)",
        "metric": "solves/s (median of 3 runs)", "one_at_a_time": round(f1["solves_per_s"], 1), "four_streams": round(f4["solves_per_s"], 1),
        "one_ensemble_context": round(fb["solves_per_s"], 1),
        "qext_rel_diff": abs(f4["qext_mean"] / f1["qext_mean"] - 1),
        "qext_rel_diff_one_context": abs(fb["qext_mean"] / f1["qext_mean"] - 1)}
    return out


def hbm_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        return 6650.0


def report_line(args, ws, R, ne):
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    m = R["mixed"]
    p = R["fp64"]
    value = job_value(ws, args.steps, m["ms_total"])
    plain = job_value(ws, args.steps, p["ms_total"])
    # dominant kernel: the FP32 translation pass of the tuned path
    ms32, n32 = m["k32"]
    stored32, canon32 = m["bytes32"]   # FP32 row-record bytes (as stored), and the reference layout's bytes at 4 B per real
    folded32 = m["bytes64"][0] / 2.0   # the folded operator values at 4 B each, without the row records' padding
    # algorithmic bytes per launch, as the canonical matvec bytes define them
    # (the reference layout's stored operator at 4 B per real, read once, +
    # x read + y written; one column per active polarisation: the tuned
    # path's Arnoldi passes carry 2 columns while both polarisations are
    # active, iterations count Arnoldi steps in pairs).  The kernel itself
    # reads the operator folded by the Wigner and axial symmetries, in row
    # records (stored32: padding and a phase table on top), which is its DRAM
    # traffic; the same pass against the folded values is reported beside.
    it = m["stats"]["iterations"]
    n32p = max(1, m["stats"]["passes32"])
    avg_cols = min(2.0, 2.0 * sum(it) / n32p) if sum(it) > 0 else 2.0
    vec_bytes = 2.0 * ne * 8 * avg_cols
    alg = canon32 + vec_bytes
    dur = ms32 / max(1, n32)
    achieved = alg / (dur * 1e-3) / 1e9 if n32 else None
    folded_gbs = (folded32 + vec_bytes) / (dur * 1e-3) / 1e9 if n32 else None
    ms64, n64 = p["k64"]
    stored64, _ = p["bytes64"]
    dur64 = ms64 / max(1, n64)
    ach64 = (stored64 + 2.0 * ne * 16 * 2) / (dur64 * 1e-3) / 1e9 if n64 else None
    e2e = R["e2e"]
    line = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "solves/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(m["ms_per_step"], 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64 GMRES cycles + c128 true residuals (tuned); c128 BiCG (plain)",
        "data": "synthetic: seeded PCA fractal aggregate (no dataset)",
        "config": bench_config(ws),
        "plain_fp64": {"value": round(plain, 4), "ms_per_step": round(p["ms_per_step"], 3),
                       "iterations": p["stats"]["iterations"], "translation_gbs": round(ach64, 1) if ach64 else None,
                       "translation_frac": round(ach64 / hbm, 4) if ach64 else None},
        "speedup_vs_plain_fp64": round(value / plain, 3),
        "tuned": {"iterations": it, "outer": m["stats"]["outer"], "passes64": m["stats"]["passes64"],
                  "passes32": m["stats"]["passes32"], "qext": m["qtot"][0, 0], "qext_plain": p["qtot"][0, 0],
                  "qext_rel_diff": abs(m["qtot"][0, 0] / p["qtot"][0, 0] - 1)},
        "roofline": {"kernel": "translate_rows_kernel<9, 2, 0> (FP32 pair translation pass, row kernel)", "bound": "hbm",
                     "achieved": round(achieved, 1) if achieved else None, "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4) if achieved else None,
                     "traffic": round(TRAFFIC_PER_ALG_BYTE * (stored32 + vec_bytes)),
                     "row_record_bytes": stored32,
                     "traffic_source": "ncu dram__bytes_read+write of this kernel on the 200-sphere aggregate "
                                       "(profiles/translate_rows_fp32_fractal200.md: 1.02x the row records and vectors "
                                       "read and written), scaled to this workload's row records",
                     "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": alg,
                     "algorithmic_bytes_source": "canonical matvec bytes (reference operator layout at 4 B per real, "
                                                 "read once, + x and y): the kernel reads the symmetry-folded operator, "
                                                 "so its traffic is below this",
                     "launch_ms": round(dur, 4), "launches": n32,
                     "folded_bytes_per_launch": folded32 + vec_bytes,
                     "folded_gbs": round(folded_gbs, 1) if folded_gbs else None,
                     "frac_of_folded_bytes": round(folded_gbs / hbm, 4) if folded_gbs else None},
        "e2e": {"value": round(ws * 1000.0 * args.steps / e2e["ms"], 4), "unit": "solves/s",
                "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]},
        "gpu_launches": int(m["launches"]),
    }
    if m.get("vs_oracle") or p.get("vs_oracle"):
        line["vs_oracle"] = {"workload": WORKLOAD + " (oracle FP64, same seeded configuration, tests/golden)",
                             "tuned": m.get("vs_oracle"), "plain_fp64": p.get("vs_oracle"),
                             "tolerance": "plain 1e-9 relative; tuned 1e-6 on efficiencies, 1e-4 on the scattering matrix"}
    if m["clocks"]:
        line["clocks"] = m["clocks"]
    return line


# ---------------------------------------------------------------------------
# CPU: the oracle (restatement of the reference) on the host cores
# ---------------------------------------------------------------------------
def _oracle_for_host(w, threads):
    from oracle import oracle as O
    return O.Oracle(w["pos"], w["radius"], w["ref_index"], mie_eps=1e-6, store_matrix=True, nthreads=threads)


def _oracle_for(name, threads, store=True):
    from mstm_b200 import configs as C
    from oracle import oracle as O
    w = C.workload(name)
    return O.Oracle(w["pos"], w["radius"], w["ref_index"], mie_eps=-w["order"], store_matrix=store, nthreads=threads)


def cpu_full_solve(name, threads):
    """One complete FP64 oracle solve (operator generation, both
    polarisations to the reference's criterion, efficiencies), as the
    reference's fixedorsoln runs it: seconds, and the iteration counts."""
    o = _oracle_for(name, threads)
    t0 = time.perf_counter()
    r = o.fixedorsoln(eps=EPS, niter=NITER)
    dt = time.perf_counter() - t0
    o.close()
    return dt, r["iterations"], r["status"]


def cpu_sample_solve_time(threads, iters_total, sample_iters=3, store=True):
    """Operator generation + `sample_iters` BiCG iterations of one
    polarisation with the oracle, scaled to a full solve of `iters_total`
    iterations (both polarisations).  store=False: the operators are
    recomputed in every pass (store_translation_matrix = .false., the
    reference's default)."""
    o = _oracle_for(WORKLOAD, threads, store)
    f = o.planewave()
    pnp = o.multmie(np.ascontiguousarray(f[:, 0]))
    t0 = time.perf_counter()
    o.sphereinteraction(pnp, initial_run=True)   # generates and stores the operators, + one pass
    t1 = time.perf_counter()
    o.cbicg(pnp, pnp, niter=sample_iters, eps=0.0, initialize=False)
    t2 = time.perf_counter()
    setup = t1 - t0
    per_iter = (t2 - t1) / (sample_iters + 1.0 / 2.0)   # cbicg's initial residual is one half-width pass
    o.close()
    return setup + per_iter * iters_total, setup, per_iter


def cpu_baseline_sample(threads):
    """The GPU arm's CPU baseline, a bounded sample: on fractal500, operator
    generation + 3 BiCG iterations on all host threads (and + 1 iteration on
    one thread, and + 1 iteration with the operators recomputed in every
    pass), scaled by the iteration count of the oracle's own solve of this
    configuration (tests/golden); beside it, complete oracle solves of the
    20-sphere cluster (the reference's CPU-sized case) on all threads and on
    one."""
    fx = oracle_fixture(WORKLOAD)
    iters = [int(v) for v in fx["iterations"]] if fx is not None else [79, 78]
    try:
        tot, setup, per_iter = cpu_sample_solve_time(threads, sum(iters))
        tot1, setup1, per_iter1 = cpu_sample_solve_time(1, sum(iters), sample_iters=1)
        totn, setupn, per_itern = cpu_sample_solve_time(threads, sum(iters), sample_iters=1, store=False)
        c20, it20, _ = cpu_full_solve("cluster20", threads)
        c20_1, _, _ = cpu_full_solve("cluster20", 1)
    except Exception as e:  # the baseline never blocks the GPU line
        return {"value": None, "unit": "solves/s", "cores": threads, "kind": "port", "sample": "failed: %s" % e}
    return {"value": round(1.0 / tot, 6), "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": "oracle (C restatement of MSTM, OpenMP over pairs, stored operators) on fractal500: operator "
                      "generation + 3 BiCG iterations timed (%.2f s + %.3f s/iteration), scaled to the %d iterations "
                      "of the oracle's own solve (%s)" % (setup, per_iter, sum(iters), iters),
            "one_core": {"value": round(1.0 / tot1, 7), "setup_s": round(setup1, 2), "s_per_iteration": round(per_iter1, 3)},
            "operators_not_stored": {"value": round(1.0 / totn, 7), "s_per_iteration": round(per_itern, 3),
                                     "note": "store_translation_matrix = .false. (the reference's default): operators "
                                             "recomputed in every pass, all threads, 1 iteration timed and scaled"},
            "cluster20_full_solve": {"solves_per_s": round(1.0 / c20, 3), "solves_per_s_one_core": round(1.0 / c20_1, 3),
                                     "iterations": it20, "note": "20 spheres, x=1, both polarisations to 1e-6, complete"}}


def run_reference(args):
    """The reference arm: complete FP64 solves of the benchmark configuration
    by the oracle (the C restatement of MSTM's fixedorsoln: stored operators
    as store_translation_matrix = .true., the reference's BiCG to its own
    criterion and its own iteration count, efficiencies) on all host
    threads, one solve per timed step.  The warm-up steps are bounded
    samples (operator generation + one BiCG iteration), which bring the
    threads, pages and caches to the state the timed solves run in."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample_solve_time(threads, 0, sample_iters=1)
    times, its = [], None
    for _ in range(args.steps):
        dt, its, st = cpu_full_solve(WORKLOAD, threads)
        times.append(dt)
    mean = sum(times) / len(times)
    v = 1.0 / mean
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 6), "unit": "solves/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(mean * 1000, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic: seeded PCA fractal aggregate (no dataset)",
            "config": bench_config(ws),
            "cpu_baseline": {"value": round(v, 6), "unit": "solves/s", "cores": threads, "kind": "port",
                             "sample": "per timed step one complete oracle solve of fractal500 (operator generation, both "
                                       "polarisations to ||r||^2/||b||^2 < 1e-12: %s BiCG iterations, efficiencies); "
                                       "warm-up steps: operator generation + 1 iteration; the Fortran reference cannot be "
                                       "built here (no Fortran compiler)" % its,
                             "solve_s": [round(t, 2) for t in times]},
            "e2e": {"value": round(v, 6), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_translation_case(args):
    """Operator generation + `--translation-passes` translation passes of one
    workload, timed with CUDA events (the case the ncu captures use)."""
    from mstm_b200 import api, configs as C
    if args.workload.startswith("tmcluster"):   # the T-matrix clusters: x = 1.5, RSA at fv 0.20, seed 4
        n = int(args.workload[len("tmcluster"):])
        pos, _ = C.rsa_sphere(n, 1.5, 0.20, seed=4)
        w = dict(pos=pos, radius=np.full(n, 1.5), ref_index=np.full(n, 1.6 + 0.005j), order=C.truncation_order(1.5))
    else:
        w = C.workload(args.workload)
    prec = "mixed" if args.precision == "tc" else args.precision
    g = api.SphereCluster(w["pos"], w["radius"], w["ref_index"], mie_epsilon=-w["order"], precision=prec,
                          fp32_chunk=args.fp32_chunk, tile_ctas_per_sm=args.ctas_per_sm, tile_pairs=args.tile_pairs)
    ms = g.time_translation(args.precision, args.nrhs, args.translation_passes)
    sb, cb = g.operator_bytes(prec)
    print(json.dumps({"workload": args.workload, "precision": args.precision, "nrhs": args.nrhs, "fp32_chunk": args.fp32_chunk,
                      "ctas_per_sm": args.ctas_per_sm, "tile_pairs": args.tile_pairs, "ms_per_pass": ms, "operator_bytes": sb, "operator_gbs": sb / ms / 1e6}))
    g.close()


def run_tmatrix_case(args):
    """One cluster T matrix of the seeded `--tmatrix-case`-sphere cluster
    (x = 1.5, m = 1.6+0.005i, RSA at fv 0.20, residual 1e-6), after one
    untimed solve (the case the T-matrix launch-list capture uses)."""
    import time
    from mstm_b200 import _lib, api, configs as C
    n = args.tmatrix_case
    pos, _ = C.rsa_sphere(n, 1.5, 0.20, seed=4)
    g = api.SphereCluster(pos, np.full(n, 1.5), np.full(n, 1.6 + 0.005j), mie_epsilon=-C.truncation_order(1.5),
                          precision=args.precision, tensor_core=args.tensor_core)
    T = g.t_matrix_order()
    g.tmatrix_solution(T, solution_eps=1e-12, convergence_eps=1e-6)
    L = _lib.lib()
    l0 = L.mstmg_kernel_launches()
    t0 = time.perf_counter()
    r = g.tmatrix_solution(T, solution_eps=1e-12, convergence_eps=1e-6)
    dt = time.perf_counter() - t0
    print(json.dumps({"spheres": n, "precision": args.precision, "tensor_core": args.tensor_core, "t_matrix_order": T,
                      "order": r["order"], "s": dt, "launches": L.mstmg_kernel_launches() - l0, "maxiter": r["maxiter"],
                      "outer": r["outer"], "qext": r["qtot"][0]}))
    g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--translation-passes", type=int, default=0,
                    help="profiling case: only run this many translation passes (no solve)")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "tc"])
    ap.add_argument("--fp32-chunk", type=int, default=0, help="profiling case: FP32 column chunk (2 or 4; 0 default)")
    ap.add_argument("--ctas-per-sm", type=int, default=0, help="profiling case: tiled kernel CTAs per SM (0 default)")
    ap.add_argument("--tile-pairs", type=int, default=0, help="profiling case: 0 the FP32 row kernel (default), 1 or 2 the rotation-tiled kernel with that many pairs per step")
    ap.add_argument("--nrhs", type=int, default=4)
    ap.add_argument("--tmatrix-case", type=int, default=0, help="profiling case: one T matrix of this many spheres")
    ap.add_argument("--tensor-core", type=int, default=0, help="profiling case: 0 tensor-core passes where they apply, -1 never")
    args = ap.parse_args()
    if args.translation_passes:
        run_translation_case(args)
    elif args.tmatrix_case:
        run_tmatrix_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
