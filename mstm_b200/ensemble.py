"""Ensembles of random configurations (the random-orientation workflow of
main_calling_program, mstm-input-37.f90:1411-1448, repeated over
configurations): each configuration's cluster T matrix (tmatrix_solution),
its orientation-averaged efficiencies and scattering matrix
(ranorientscatmatrix), and the ensemble means.

Configurations of uneven size are solved concurrently: worker threads each
drive their own contexts, and every context launches on its own CUDA stream,
so small configurations fill the GPU together (the C calls release the
interpreter lock).  Kernel settings are chosen per size class by `Autotuner`,
which times one many-column translation pass -- the operation that dominates
a T-matrix solve -- under each candidate setting and keeps the fastest.

`solve_fixed_ensemble` does the same for fixed-orientation solves
(fixedorsoln with both polarisations) of many small configurations, whose
solves are bound by launch and synchronisation latency rather than by the
GPU's arithmetic, so that concurrent streams overlap one another's gaps.
"""
import ctypes
import threading
import time

import numpy as np

from . import _lib
from . import api
from . import configs as C


def ensemble_configs(count, seed=4, nmin=50, nmax=400, x=1.5, m=1.6 + 0.005j, fv=0.20):
    """Seeded ensemble: sphere counts uniform in [nmin, nmax], identical spheres
    of size parameter x and index m, RSA in a bounding sphere at volume fraction fv."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        pos, _ = C.rsa_sphere(n, x, fv, seed=int(rng.integers(0, 2 ** 31 - 1)))
        out.append(dict(pos=np.asarray(pos, np.float64), x=x, m=m, n=n, order=C.truncation_order(x)))
    return out


class Autotuner:
    """Per size class (sphere count rounded to 50, sphere order, precision), the
    pass that serves the many-column solves: the tensor-core pass (dense TF32
    hi/lo operators), or the rotation kernels with their CTAs per SM, FP32
    column chunk and kernel family (tiled or order-generic), chosen by timing
    one translation pass over the column count of a T-matrix group."""

    CANDIDATES = [dict(tensor_core=0)] + \
                 [dict(tensor_core=-1, tile_ctas_per_sm=c, fp32_chunk=k, generic_kernel=0) for c in (0, 2) for k in (2, 4)] + \
                 [dict(tensor_core=-1, tile_ctas_per_sm=0, fp32_chunk=0, generic_kernel=1)]

    def __init__(self, reps=3):
        self.reps = reps
        self.table = {}
        self.lock = threading.Lock()
        self.log = []

    @staticmethod
    def size_class(n):
        return int(50 * round(n / 50.0))

    def choose(self, cfg, precision, columns):
        key = (self.size_class(len(cfg["pos"])), cfg["order"], precision, columns)
        with self.lock:
            if key in self.table:
                return self.table[key]
        L = _lib.lib()
        best, best_ms, trials = None, float("inf"), []
        n = len(cfg["pos"])
        for cand in self.CANDIDATES:
            g = api.SphereCluster(cfg["pos"], np.full(n, cfg["x"]), np.full(n, cfg["m"]), mie_epsilon=-cfg["order"],
                                  precision=precision, **cand)
            ms = ctypes.c_double(0.0)
            prec = 0 if precision == "fp64" else (2 if cand.get("tensor_core", -1) == 0 else 1)
            rc = L.mstmg_time_translation(g.ctx, prec, columns, self.reps, ctypes.byref(ms))
            err = L.mstmg_last_error().decode() if rc != 0 else ""
            g.close()
            if rc != 0:
                trials.append((dict(cand), None, f"status {rc}: {err}"))
                continue
            trials.append((dict(cand), ms.value, ""))
            if ms.value < best_ms:
                best, best_ms = dict(cand), ms.value
        with self.lock:
            if best is not None:
                self.table[key] = best
            self.log.append(dict(key=key, trials=trials, best=best, best_ms=best_ms))
        return best


def solve_one(cfg, precision="mixed", settings=None, solution_eps=1e-6, convergence_eps=1e-6, nangles=181, trans_eps=1e-5):
    """T matrix, orientation-averaged efficiencies and scattering matrix of one configuration."""
    n = len(cfg["pos"])
    g = api.SphereCluster(cfg["pos"], np.full(n, cfg["x"]), np.full(n, cfg["m"]), mie_epsilon=-cfg["order"], precision=precision,
                          **(settings or {}))
    T = g.t_matrix_order(trans_eps=trans_eps)
    r = g.tmatrix_solution(T, solution_eps=solution_eps, convergence_eps=convergence_eps)
    u = r["order"]
    nb = 2 * u * (u + 2)
    tm = np.asfortranarray(r["tmat"][:nb, :nb])
    ro = g.ranorientscatmatrix(tm, u, nangles=nangles)
    qe, qs = g.tmatrix_qext_qsca(tm, u)
    g.close()
    return dict(n=n, t_matrix_order=T, order=u, qtot=r["qtot"], qext_t=qe, qsca_t=qs, smat=ro["smat"], coherent=ro["coherent"],
                maxiter=r["maxiter"], istat=r["istat"])


def solve_ensemble(cfgs, precision="mixed", workers=4, tuner=None, **kw):
    """Solve every configuration (largest first, over `workers` threads) and
    return per-configuration results, ensemble means and throughput."""
    order = sorted(range(len(cfgs)), key=lambda k: -len(cfgs[k]["pos"]))
    results = [None] * len(cfgs)
    tune_cols = 128   # columns of one tensor-core tile, about a T-matrix order group
    t_tune = time.time()
    if tuner is not None:
        # one representative per size class, timed alone before any solve runs
        seen = set()
        for k in order:
            key = (Autotuner.size_class(len(cfgs[k]["pos"])), cfgs[k]["order"])
            if key not in seen:
                seen.add(key)
                tuner.choose(cfgs[k], precision, tune_cols)
    t_tune = time.time() - t_tune
    errors = []
    nxt = [0]
    lock = threading.Lock()

    def worker():
        while True:
            with lock:
                if nxt[0] >= len(order):
                    return
                k = order[nxt[0]]
                nxt[0] += 1
            cfg = cfgs[k]
            try:
                settings = tuner.choose(cfg, precision, tune_cols) if tuner is not None else None
                results[k] = solve_one(cfg, precision, settings, **kw)
            except Exception as e:   # reported after the join
                errors.append((k, repr(e)))

    t0 = time.time()
    threads = [threading.Thread(target=worker) for _ in range(max(1, workers))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.time() - t0
    if errors:
        raise RuntimeError(f"ensemble: {len(errors)} configurations failed, first: {errors[0]}")
    q = np.array([r["qtot"] for r in results])
    smat = np.mean([r["smat"] for r in results], axis=0)
    return dict(per_config=results, qext=float(q[:, 0].mean()), qabs=float(q[:, 1].mean()), qsca=float(q[:, 2].mean()),
                smat=smat, wall_s=wall, tune_s=t_tune, tmatrices_per_s=len(cfgs) / wall)


def solve_fixed_ensemble(positions, x, m, precision="mixed", workers=4, solution_eps=1e-12, max_iterations=4000,
                         mie_epsilon=None):
    """Fixed-orientation solves (both polarisations, +z incidence) of a list of
    configurations (each an (N, 3) array of positions, spheres of size
    parameter x and index m), `workers` at a time on their own streams.
    Returns dict(per_config: qtot (3, 3) and iterations, qext_mean, wall_s,
    solves_per_s).  More than about 4 workers stops paying: measured on a B200
    with 48 clusters of 15-40 spheres, 1/2/4 workers gave 289/474/663
    solves/s and 8 workers fell to 60."""
    me = -C.truncation_order(x) if mie_epsilon is None else mie_epsilon
    ctxs = [api.SphereCluster(p, np.full(len(p), x), np.full(len(p), m), mie_epsilon=me, precision=precision) for p in positions]
    results = [None] * len(ctxs)
    errors = []
    nxt = [0]
    lock = threading.Lock()

    def worker():
        while True:
            with lock:
                if nxt[0] >= len(ctxs):
                    return
                k = nxt[0]
                nxt[0] += 1
            try:
                r = ctxs[k].fixedorsoln(eps=solution_eps, niter=max_iterations)
                results[k] = dict(qtot=r["qtot"], iterations=r["iterations"], istat=r["istat"])
            except Exception as e:   # reported after the join
                errors.append((k, repr(e)))

    t0 = time.time()
    threads = [threading.Thread(target=worker) for _ in range(max(1, workers))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.time() - t0
    for g in ctxs:
        g.close()
    if errors:
        raise RuntimeError(f"fixed ensemble: {len(errors)} configurations failed, first: {errors[0]}")
    q = np.array([r["qtot"][0, 0] for r in results])
    return dict(per_config=results, qext_mean=float(q.mean()), wall_s=wall, solves_per_s=len(ctxs) / wall)


def solve_fixed_ensemble_batched(positions, x, m, solution_eps=1e-12, max_iterations=4000, mie_epsilon=None, reps=1):
    """The configurations of solve_fixed_ensemble as ONE ensemble context
    (api.SphereEnsemble): no pairs between configurations, every Arnoldi step
    one translation pass over all of them, each configuration's two
    polarisations stopping on their own criterion.  Same return dict;
    wall_s is the solve call alone (the context is built before it), the
    median of `reps` calls."""
    me = -C.truncation_order(x) if mie_epsilon is None else mie_epsilon
    ens = api.SphereEnsemble([(p, np.full(len(p), x), m) for p in positions], mie_epsilon=me)
    walls = []
    try:
        for _ in range(max(1, reps)):
            t0 = time.time()
            r = ens.fixedorsoln(eps=solution_eps, niter=max_iterations)
            walls.append(time.time() - t0)
    finally:
        ens.close()
    wall = sorted(walls)[len(walls) // 2]
    results = [dict(qtot=r["qtot"][k], iterations=r["iterations"][k].tolist(), istat=int(r["istat"])) for k in range(len(positions))]
    q = np.array([rk["qtot"][0, 0] for rk in results])
    return dict(per_config=results, qext_mean=float(q.mean()), wall_s=wall, solves_per_s=len(positions) / wall)


def shard_configs(sizes, world):
    """Split configurations over `world` ranks with balanced work: largest
    first, each to the rank with the least work so far (a solve's pass work
    grows as N^2 pairs).  Returns one sorted index list per rank."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for k in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(k)
        load[r] += float(sizes[k]) ** 2
    return [sorted(p) for p in parts]


def reduce_means(qtots, dist=None, device="cpu"):
    """Ensemble means of Qext, Qabs, Qsca (unpolarised) over all ranks: each
    rank's sums and count, one all-reduce (SUM) when a process group is
    given.  qtots: this rank's (3, 3) efficiency arrays."""
    import torch
    s = np.zeros(4)
    for q in qtots:
        s[:3] += [q[0, 0], q[1, 0], q[2, 0]]
        s[3] += 1.0
    t = torch.tensor(s, dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t)
    s = t.cpu().numpy()
    n = max(s[3], 1.0)
    return dict(qext_mean=s[0] / n, qabs_mean=s[1] / n, qsca_mean=s[2] / n, count=int(s[3]))


def solve_fixed_ensemble_sharded(positions, x, m, rank=0, world=1, dist=None, device="cpu", solve=None, **kw):
    """An ensemble split over ranks (one GPU each, no exchange during the
    solves): this rank solves its share (shard_configs) with `solve`
    (default solve_fixed_ensemble_batched: one ensemble context), then one
    all-reduce gives every rank the ensemble means.  Returns dict(indices,
    per_config of this rank, and the means of reduce_means)."""
    solve = solve_fixed_ensemble_batched if solve is None else solve
    idx = shard_configs([len(p) for p in positions], world)[rank]
    local = solve([positions[k] for k in idx], x, m, **kw) if idx else dict(per_config=[])
    out = reduce_means([r["qtot"] for r in local["per_config"]], dist, device)
    out.update(indices=idx, per_config=local["per_config"])
    return out
