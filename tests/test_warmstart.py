"""Learned warm start: the device network kernels against the CPU restatement
(oracle/warmstart_ref.py), and what the trained network gains over the
reference's Mie-solution start."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws():
    import torch
    from mstm_b200 import warmstart as W
    return W, torch.device("cuda", 0)


def _tiny_samples(W, n_cfg=2, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n_cfg):
        cfg = W.sample_config(rng)
        n = 24 + 6 * c
        cfg["pos"] = cfg["pos"][:n]
        X = rng.standard_normal((n, W.NF)).astype(np.float32)
        t = (0.1 * rng.standard_normal((n, W.NOUT))).astype(np.float32)
        mask = (rng.random((n, W.NOUT)) < 0.8).astype(np.float32)
        out.append(dict(cfg=cfg, X=X, target=t, mask=mask))
    return out


def test_knn_kernel_matches_cpu(ws):
    W, dev = ws
    from oracle import warmstart_ref as R
    s = _tiny_samples(W, 3, seed=1)
    nbr, start = W.knn_device(s, dev)
    for c, (a, b) in enumerate(zip(start[:-1], start[1:])):
        ref = R.knn(s[c]["cfg"]["pos"], W.K_NN)
        assert np.array_equal(nbr[a:b] - a, ref)


@pytest.mark.parametrize("bf16", [False, True])
def test_gradients_match_cpu_restatement(ws, bf16):
    """Loss and every parameter gradient of one forward/backward pass: FP32
    weights agree with the FP64 restatement to FP32 rounding; BF16 weights to
    the BF16 rounding of the weights."""
    W, dev = ws
    from oracle import warmstart_ref as R
    s = _tiny_samples(W, 2, seed=2)
    net = W.WarmStartNet(dev, seed=3, bf16=bf16)
    gr = W.batch_graph(s, dev)
    y, cache = net.forward(gr)
    loss, dy = net.loss_grad(y, gr["target"], gr["mask"], gr["msum"])
    net.backward(gr, cache, dy)
    P = {}
    for name, (o, shp) in net.off.items():
        src = net.pb if (bf16 and not name.endswith("_b")) else net.p
        P[name] = src[o:o + int(np.prod(shp))].float().cpu().numpy().astype(np.float64).reshape(shp)
    # biases are always FP32 in the device pass
    for name in P:
        if name.endswith("_b"):
            o, shp = net.off[name]
            P[name] = net.p[o:o + int(np.prod(shp))].cpu().numpy().astype(np.float64).reshape(shp)
    X = gr["X"].cpu().numpy().astype(np.float64)
    ef = gr["ef"].cpu().numpy().astype(np.float64)
    dst = gr["dst"].cpu().numpy()
    src_ = gr["src"].cpu().numpy()
    lr, G = R.forward_backward(P, X, ef, dst, src_, gr["target"].cpu().numpy().astype(np.float64),
                               gr["mask"].cpu().numpy().astype(np.float64))
    tol = 2e-3 if not bf16 else 2e-2
    assert abs(float(loss.item()) / lr - 1) < tol
    g = net.g.cpu().numpy()
    for name, (o, shp) in net.off.items():
        gd = g[o:o + int(np.prod(shp))].reshape(shp)
        gc = G[name]
        assert np.linalg.norm(gd - gc) <= tol * max(np.linalg.norm(gc), 1e-12), name


def test_trained_guess_beats_mie_start(ws):
    """Train on configurations the solver itself solved, then start held-out
    configurations from the predicted guess: the initial relative residual is
    well below that of the reference's Mie-solution start, the converged
    efficiencies are the same, and the iteration count is no worse."""
    W, dev = ws
    rng = np.random.default_rng(11)

    def cfgs(k):
        out = []
        for _ in range(k):
            c = W.sample_config(rng)
            n = int(rng.integers(100, 161))
            c["pos"] = c["pos"][:n]
            out.append(c)
        return out

    train = [W.make_sample(c) for c in cfgs(64)]
    held = [W.make_sample(c) for c in cfgs(6)]
    net = W.WarmStartNet(dev, seed=0)
    hist = W.train(net, train, epochs=60, batch=8, lr=2e-3)
    assert hist[-1] < 0.7 * hist[0]
    res_plain, res_warm, it_plain, it_warm = [], [], 0, 0
    for s in held:
        x0 = W.predict_guess(net, s)
        # solved to ||r||/||b|| < 1e-8 so that the two solutions agree to well below 1e-6
        rw = W.solve_with_guess(s["cfg"], x0, eps=1e-16, precision="fp64", fallback=10.0)
        rp = W.solve_with_guess(s["cfg"], s["a0"], eps=1e-16, precision="fp64", fallback=10.0)
        assert rw["used"] == [1, 1]
        res_plain += rp["guess_residual"]
        res_warm += rw["guess_residual"]
        it_plain += sum(rp["iterations"])
        it_warm += sum(rw["iterations"])
        assert np.allclose(rw["qtot"], rp["qtot"], rtol=1e-6)
    assert np.mean(res_warm) < 0.75 * np.mean(res_plain)
    assert it_warm <= it_plain * 1.05


def test_fallback_to_mie_start(ws):
    """A guess whose initial residual exceeds the threshold is replaced by the
    Mie-solution start: the solve then matches the plain one exactly."""
    W, dev = ws
    rng = np.random.default_rng(3)
    c = W.sample_config(rng)
    c["pos"] = c["pos"][:120]
    s = W.make_sample(c)
    bad = s["a0"] * 50.0
    rw = W.solve_with_guess(s["cfg"], bad, eps=1e-12, precision="fp64", fallback=0.1)
    rp = W.solve_with_guess(s["cfg"], s["a0"], eps=1e-12, precision="fp64", fallback=10.0)
    assert rw["used"] == [0, 0] and min(rw["guess_residual"]) > 0.1
    assert rw["iterations"] == rp["iterations"]
    assert np.allclose(rw["qtot"], rp["qtot"], rtol=1e-12)


def test_ensemble_samples_match_single_solves(ws):
    """The study's training samples from ensemble solves (configurations of
    one order together) carry the same Mie start and, to the solution
    tolerance, the same targets as one-at-a-time solves."""
    from mstm_b200 import configs as C
    W, _ = ws
    cfgs = W.draw_configs(4, 17)
    cfgs[1] = dict(cfgs[1], order=cfgs[0]["order"], x=cfgs[0]["x"])   # two of one order share an ensemble
    cfgs[1]["pos"] = C.rsa_sphere_batched(len(cfgs[1]["pos"]), cfgs[1]["x"], cfgs[1]["fv"], seed=3)[0]
    batched = W.solve_samples(cfgs, eps=1e-12)
    for cfg, b in zip(cfgs, batched):
        s = W.make_sample(cfg, eps=1e-12)
        assert np.abs(b["a0"] - s["a0"]).max() <= 1e-12 * np.abs(s["a0"]).max()
        assert np.array_equal(b["mask"], s["mask"]) and np.allclose(b["X"], s["X"])
        scale = np.abs(s["target"]).max()
        assert np.abs(b["target"] - s["target"]).max() <= 1e-4 * scale


def test_saved_network_reloads_and_evaluates(ws, tmp_path):
    """The network trained at scale (mstm_b200/data/warmstart_net.npz) loads,
    its guesses on held-out configurations start below the Mie start's
    residual, and a save / load round trip keeps the weights."""
    import os
    W, dev = ws
    path = os.path.join(os.path.dirname(W.__file__), "data", "warmstart_net.npz")
    net, meta = W.load_net(path, dev)
    assert meta["n_train"] == 20000 and meta["n_eval"] == 1000
    held = W.solve_samples(W.draw_configs(4, 6, workers=0))
    ev = W.evaluate(net, held, fallbacks=(1.0,))
    r = ev["fallback_1"]
    assert r["polarisations"] == 8 and r["mean_initial_residual_warm"] < r["mean_initial_residual_mie"]
    W.save_net(net, str(tmp_path / "n.npz"), meta=meta)
    net2, meta2 = W.load_net(str(tmp_path / "n.npz"), dev)
    assert np.array_equal(net2.state(), net.state()) and meta2 == meta
