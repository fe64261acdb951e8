"""Single-cluster sharding over ranks (mstm_b200.shard, mstmg_set_pair_shard).

CPU (gloo, world size 2): the reference's BiCG driven on interactions summed
over the ranks, each rank holding one part of a dense operator, reaches the
dense solution and the single-rank iterates.  GPU: the shards of a cluster's
tiles sum to the whole translation pass (FP64 to 1e-12 and FP32 to 2e-6 of
the largest output; on the FFT path too, shard 0 adding the far field) and
to the whole Mie-multiplied interaction, plain and conjugate-transpose
columns; a BiCG on two shard contexts summed in one
process gives the library's FP64 fixed-orientation solve (its iterations,
efficiencies to 1e-9); the solvers refuse a sharded context.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from mstm_b200 import configs as C


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _dense_case(n=40, seed=3):
    rng = np.random.default_rng(seed)
    K = 0.3 * (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) / np.sqrt(n)
    b = rng.normal(size=n) + 1j * rng.normal(size=n)
    # the ranks' parts: K = K0 + K1, split entry by entry
    mask = rng.random((n, n)) < 0.5
    return K, b, [np.where(mask, K, 0), np.where(mask, 0, K)]


def _local_dense(Kr):
    Kt = torch.as_tensor(Kr)

    def f(X, con_tran, initial_run):
        Y = torch.empty_like(X)
        for r, ct in enumerate(con_tran):
            Y[r] = (Kt.conj().T @ X[r]) if ct else (Kt @ X[r])
        return Y
    return f


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    from mstm_b200 import shard
    K, b, parts = _dense_case()
    f = shard.summed(_local_dense(parts[rank]))
    bt = torch.as_tensor(b)
    x, it, err, st = shard.cbicg(f, bt, bt.clone(), 1e-20, 200)
    q.put((rank, x.numpy(), it, err, st))
    dist.barrier()
    dist.destroy_process_group()


def test_cbicg_on_interactions_summed_over_two_gloo_ranks():
    from mstm_b200 import shard
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict((r, (x, it, err, st)) for r, x, it, err, st in (q.get(timeout=120) for _ in range(ws)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    K, b, _ = _dense_case()
    xd = np.linalg.solve(np.eye(len(b)) - K, b)
    one = shard.cbicg(_local_dense(K), torch.as_tensor(b), torch.as_tensor(b).clone(), 1e-20, 200)
    for r in range(ws):
        x, it, err, st = res[r]
        assert st == 0 and err < 1e-20
        assert np.abs(x - xd).max() <= 1e-9 * np.abs(xd).max()
        assert it == one[1] and np.abs(x - one[0].numpy()).max() <= 1e-12 * np.abs(xd).max()
    assert np.array_equal(res[0][0], res[1][0])   # every rank holds the same iterate


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _fractal(name="fractal60"):
    w = C.workload(name)
    return w["pos"], w["radius"], w["ref_index"], -float(w["order"])


@pytest.mark.gpu
@pytest.mark.parametrize("nshards", [2, 3])
def test_shards_sum_to_the_whole_pass(nshards):
    from mstm_b200 import api
    pos, rad, ri, em = _fractal()
    whole = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="mixed")
    parts = []
    for s in range(nshards):
        g = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="mixed")
        g.set_pair_shard(s, nshards)
        parts.append(g)
    rng = np.random.default_rng(nshards)
    x = rng.normal(size=(whole.number_eqns, 2)) + 1j * rng.normal(size=(whole.number_eqns, 2))
    for prec, tol in (("fp64", 1e-12), ("fp32", 2e-6)):
        y = whole.translation_pass(x, [0, 1], prec)
        ys = sum(g.translation_pass(x, [0, 1], prec) for g in parts)
        assert np.abs(ys - y).max() <= tol * np.abs(y).max(), prec
    y = whole.sphereinteraction(x, con_tran=[0, 1], mie_mult=[1, 1])
    ys = sum(g.sphereinteraction(x, con_tran=[0, 1], mie_mult=[1, 1]) for g in parts)
    assert np.abs(ys - y).max() <= 1e-12 * np.abs(y).max()
    # one shard back to the whole set
    parts[0].set_pair_shard(0, 1)
    y0 = whole.translation_pass(x, [0, 1], "fp64")
    assert np.abs(parts[0].translation_pass(x, [0, 1], "fp64") - y0).max() <= 1e-14 * np.abs(y0).max()
    for g in parts + [whole]:
        g.close()


@pytest.mark.gpu
def test_bicg_over_two_shards_in_one_process_matches_the_library():
    from mstm_b200 import api, shard
    pos, rad, ri, em = _fractal()
    ref = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="fp64")
    r = ref.fixedorsoln(eps=1e-12, niter=2000)
    ws = []
    for s in range(2):
        sc = shard.ShardedCluster(pos, rad, ri, mie_epsilon=em)   # world size 1 here
        sc.g.set_pair_shard(s, 2)
        ws.append(sc)
    summed = lambda X, ct, init: ws[0]._local(X, ct, init) + ws[1]._local(X, ct, init)
    pnp = torch.as_tensor(np.ascontiguousarray(ref.fixed_orientation_rhs().T), device=ws[0].device)
    amnp = np.zeros((ref.number_eqns, 2), np.complex128, order="F")
    its = []
    for p in range(2):
        x, it, err, st = shard.cbicg(summed, pnp[p], pnp[p].clone(), 1e-12, 2000, initialize=(p == 0))
        assert st == 0 and err < 1e-12
        its.append(it)
        amnp[:, p] = x.cpu().numpy()
    assert abs(its[0] - r["iterations"][0]) <= 1 and abs(its[1] - r["iterations"][1]) <= 1
    q = ref.efficiencies(amnp)
    assert np.allclose(q["qtot"], r["qtot"], rtol=1e-9)
    # the same through the class on one rank
    one = shard.ShardedCluster(pos, rad, ri, mie_epsilon=em)
    r1 = one.fixedorsoln(eps=1e-12, niter=2000)
    assert r1["istat"] == 0 and r1["iterations"] == r["iterations"]
    assert np.allclose(r1["qtot"], r["qtot"], rtol=1e-9)
    for g in ws + [one]:
        g.close()
    ref.close()


@pytest.mark.gpu
def test_sharded_context_refuses_the_solvers():
    from mstm_b200 import api
    from mstm_b200._lib import MstmgError
    pos, rad, ri, em = _fractal()
    g = api.SphereCluster(pos, rad, ri, mie_epsilon=em, precision="mixed")
    g.set_pair_shard(1, 2)
    with pytest.raises(MstmgError):
        g.fixedorsoln(eps=1e-6)
    with pytest.raises(MstmgError):
        g.tmatrix_solution(g.t_matrix_order())
    x = np.ones((g.number_eqns, 16), np.complex128)
    with pytest.raises(MstmgError):
        g.translation_pass(x, None, "tc")
    with pytest.raises(MstmgError):
        g.set_pair_shard(2, 2)
    g.close()


@pytest.mark.gpu
def test_fft_shards_sum_to_the_whole_pass():
    """On the FFT path the near-pair tiles are dealt to the shards and shard 0
    adds the far field: the shards still sum to the whole pass."""
    from mstm_b200 import api
    cyl, _ = C.rsa_cylinder(300, 1.0, 0.25, 1.0, seed=3)
    n = len(cyl)
    mk = lambda: api.SphereCluster(cyl, np.full(n, 1.0), np.full(n, 1.31 + 0j), mie_epsilon=-7, precision="mixed")
    whole = mk()
    whole.fft_setup(d_cell=4.0)
    parts = []
    for s in range(2):
        g = mk()
        g.fft_setup(d_cell=4.0)
        g.set_pair_shard(s, 2)
        parts.append(g)
    rng = np.random.default_rng(11)
    x = rng.normal(size=(whole.number_eqns, 2)) + 1j * rng.normal(size=(whole.number_eqns, 2))
    for prec, tol in (("fp64", 1e-12), ("fp32", 2e-6)):
        y = whole.translation_pass(x, [0, 1], prec)
        ys = parts[0].translation_pass(x, [0, 1], prec) + parts[1].translation_pass(x, [0, 1], prec)
        assert np.abs(ys - y).max() <= tol * np.abs(y).max(), prec
    for g in parts + [whole]:
        g.close()
