"""The N > 1 path of bench.py on CPU: world-size-2 gloo ranks exercise the
replica logic (each rank its own seeded configuration, no data-path
collective) and the max-over-ranks timing that the GPU run uses under
torchrun with NCCL."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank), LOCAL_RANK=str(rank))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    w_, r_, l_ = bench.dist_env()
    dist = bench.init_dist(w_, "gloo")
    # the slowest rank sets the job time
    t = bench.max_over_ranks(dist, 10.0 + 5.0 * rank, "cpu")
    # replicas: each rank's own configuration (positions differ, sizes agree)
    w = bench.workload_for_rank(rank)
    h = float(np.sum(np.abs(w["pos"])))   # the aggregates are centred: compare spreads
    import torch
    hs = [torch.zeros(1, dtype=torch.float64) for _ in range(ws)]
    dist.all_gather(hs, torch.tensor([h], dtype=torch.float64))
    # a small solve per rank on the CPU oracle, timed and reduced like the bench
    from oracle.oracle import Oracle
    from mstm_b200 import configs as C
    pos, _ = C.rsa_sphere(6, 1.0, 0.1, seed=10 + rank)
    o = Oracle(pos, [1.0] * 6, [1.5 + 0.01j] * 6, mie_eps=-5)
    import time
    t0 = time.perf_counter()
    r = o.fixedorsoln(eps=1e-10)
    ms = (time.perf_counter() - t0) * 1e3
    ms_max = bench.max_over_ranks(dist, ms, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put(dict(rank=rank, t=t, hashes=[float(x.item()) for x in hs], n=len(w["pos"]), ms=ms, ms_max=ms_max,
               qext=float(r["qtot"][0, 0]), value=bench.job_value(ws, 1, ms_max)))


def test_two_gloo_ranks_replicas_and_max_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ws, port = 2, _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort(key=lambda d: d["rank"])
    assert all(d["t"] == 15.0 for d in out)                      # MAX over ranks
    assert out[0]["hashes"] == out[1]["hashes"]                  # every rank saw both
    assert out[0]["hashes"][0] != out[0]["hashes"][1]            # distinct configurations
    assert out[0]["n"] == out[1]["n"] == 500
    ms_max = max(d["ms"] for d in out)
    assert all(abs(d["ms_max"] - ms_max) < 1e-9 for d in out)
    # whole-job throughput: all ranks' solves over the slowest rank's time
    assert abs(out[0]["value"] - 2 * 1000.0 / ms_max) < 1e-9 * out[0]["value"]
    assert out[0]["qext"] != out[1]["qext"]
