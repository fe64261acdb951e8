"""Ensembles split over ranks on CPU: world-size-2 gloo ranks each solve their
share of the configurations (the FP64 oracle stands in for a rank's GPU
solve) and one all-reduce gives every rank the ensemble means."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_solve(positions, x, m, **kw):
    from oracle.oracle import Oracle
    out = []
    for p in positions:
        o = Oracle(p, [x] * len(p), [m] * len(p), mie_eps=-4)
        r = o.fixedorsoln(eps=1e-10)
        out.append(dict(qtot=r["qtot"], iterations=[r["maxiter"]] * 2, istat=r["status"]))
        o.close()
    return dict(per_config=out)


def _configs():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from mstm_b200 import configs as C
    return [C.rsa_sphere(n, 0.8, 0.1, seed=40 + k)[0] for k, n in enumerate((3, 6, 4, 5, 2))]


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from mstm_b200 import ensemble as E
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    r = E.solve_fixed_ensemble_sharded(_configs(), 0.8, 1.5 + 0.01j, rank=rank, world=ws, dist=dist, solve=_oracle_solve)
    dist.barrier()
    dist.destroy_process_group()
    q.put(dict(rank=rank, indices=r["indices"], qext_mean=r["qext_mean"], qsca_mean=r["qsca_mean"], count=r["count"]))


def test_shard_configs_balances_and_covers():
    from mstm_b200 import ensemble as E
    sizes = [50, 400, 120, 300, 80, 250, 60]
    parts = E.shard_configs(sizes, 3)
    assert sorted(k for p in parts for k in p) == list(range(len(sizes)))
    loads = [sum(sizes[k] ** 2 for k in p) for p in parts]
    assert max(loads) <= 400 ** 2 + 1   # no rank carries more than the largest configuration's share
    assert E.shard_configs([5, 5], 4)[2:] == [[], []]


def test_two_gloo_ranks_ensemble_means():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ws, port = 2, _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=240) for _ in range(ws)], key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(out[0]["indices"] + out[1]["indices"]) == [0, 1, 2, 3, 4]
    assert not set(out[0]["indices"]) & set(out[1]["indices"])
    ref = _oracle_solve(_configs(), 0.8, 1.5 + 0.01j)["per_config"]
    qext = np.mean([r["qtot"][0, 0] for r in ref])
    qsca = np.mean([r["qtot"][2, 0] for r in ref])
    for d in out:
        assert d["count"] == 5
        assert abs(d["qext_mean"] / qext - 1) < 1e-12 and abs(d["qsca_mean"] / qsca - 1) < 1e-12
