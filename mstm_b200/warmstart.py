"""Learned warm start for the fixed-orientation solve (no counterpart in MSTM).

A message-passing network over each sphere's k nearest neighbours predicts the
sphere's interaction correction Delta a_i = a_i - a_i^0 to its isolated-sphere
solution a_i^0 = Mie_i f_i (the reference's BiCG initial guess, fixedorsoln,
mstm-solver-8.f90:482-483).  The BiCG then starts from a^0 + Delta a; a
polarisation whose initial relative residual ||r||/||b|| exceeds `fallback`
(default 1, the residual of a zero start) starts from a^0 as the reference
does (mstmg_fixed_orientation_guess), so the converged residual, not the
network, decides the answer.

Network (sizes as in the cluster-ensemble study this targets):
  node features (41): x, Re m, log10 Im m, volume fraction, N/300, and the
      LR-basis Mie matrix entries A(1,1), A(2,1) (re, im) for n = 1..9;
  edge features (10) for the edge j -> i: (r_j - r_i)/x_i, |r_j - r_i|/x_i,
      cos and sin of (z_j - z_i) (the relative phase of the +z incident
      wave), x_j, Re m_j, log10 Im m_j, x_j/x_i;
  encoder  h = SiLU(X We + be)                               (41 -> 128)
  3 layers m_e = SiLU([h_i, h_j, e_ij] Wm + bm)                (265 -> 128)
           h_i <- h_i + SiLU(h_i Wu1 + (sum_e m_e) Wu2 + bu)   (128+128 -> 128)
  head     y = h Wo + bo                                       (128 -> 792)
  output: both polarisations' exciting-field corrections
      e_i = Mie_i^{-1} Delta a_i in the sphere's incident-phase frame
      (times e^{-i z_i}), order-9 block layout, re/im; Delta a_i = Mie_i e_i.
Weights are BF16 copies of FP32 masters; every product accumulates in FP32.
All arithmetic runs in the library's kernels (warmstart.cu); torch provides
device memory only.
"""
import ctypes
import math

import numpy as np

from . import _lib
from . import api
from . import configs as C

LMAX = 9
NBH = LMAX * (LMAX + 2)          # one mode of an order-9 block
NOUT = 2 * 2 * 2 * NBH           # polarisations x modes x (re, im)
NF = 5 + 4 * LMAX
EF = 10
K_NN = 12
HID = 128
LAYERS = 3


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _aidx(m, n, p, L):
    return (m + (L + 2) * (n - 1) if m >= 0 else (n + 1) + (L + 2) * (-m - 1)) + (L + 2) * L * p


def block_map(L):
    """Indices of an order-L sphere block inside the order-9 block (both modes)."""
    src, dst = [], []
    for p in range(2):
        for n in range(1, L + 1):
            for m in range(-n, n + 1):
                src.append(_aidx(m, n, p, L))
                dst.append(_aidx(m, n, p, LMAX))
    return np.array(src), np.array(dst)


# ---------------------------------------------------------------------------
# configurations and features
# ---------------------------------------------------------------------------
def sample_config(rng):
    """One configuration of the warm-start study: 100-300 spheres, x in [0.5, 2],
    Re m in [1.3, 1.7], Im m log-uniform in [1e-4, 0.1], volume fraction in
    [0.05, 0.30], RSA in a bounding sphere."""
    n = int(rng.integers(100, 301))
    x = float(rng.uniform(0.5, 2.0))
    m = complex(rng.uniform(1.3, 1.7), 10.0 ** rng.uniform(-4.0, -1.0))
    fv = float(rng.uniform(0.05, 0.30))
    pos, _ = C.rsa_sphere(n, x, fv, seed=int(rng.integers(0, 2 ** 31 - 1)))
    return dict(pos=np.asarray(pos, np.float64), x=x, m=m, fv=fv, order=C.truncation_order(x))


def node_features(cfg, an):
    """an: the context's LR Mie matrices, (2,2,L) complex per sphere, identical spheres."""
    n, L = len(cfg["pos"]), cfg["order"]
    f = np.zeros((n, NF), np.float32)
    f[:, 0] = cfg["x"]
    f[:, 1] = cfg["m"].real
    f[:, 2] = math.log10(cfg["m"].imag)
    f[:, 3] = cfg["fv"]
    f[:, 4] = n / 300.0
    for k in range(min(L, LMAX)):
        a11, a21 = an[4 * k], an[4 * k + 1]
        f[:, 5 + 4 * k:9 + 4 * k] = [a11.real, a11.imag, a21.real, a21.imag]
    return f


def edge_features(cfg, nbr):
    """nbr: (n, K) neighbour indices (local); edges j -> i for every i, in order."""
    pos, x, m = cfg["pos"], cfg["x"], cfg["m"]
    n = len(pos)
    i = np.repeat(np.arange(n), nbr.shape[1])
    j = nbr.reshape(-1)
    d = (pos[j] - pos[i]) / x
    dz = pos[j, 2] - pos[i, 2]
    e = np.zeros((len(i), EF), np.float32)
    e[:, 0:3] = d
    e[:, 3] = np.linalg.norm(d, axis=1)
    e[:, 4] = np.cos(dz)
    e[:, 5] = np.sin(dz)
    e[:, 6] = x
    e[:, 7] = m.real
    e[:, 8] = math.log10(m.imag)
    e[:, 9] = 1.0
    return i, j, e


def solver_pair(cfg, precision="mixed"):
    n = len(cfg["pos"])
    return api.SphereCluster(cfg["pos"], np.full(n, cfg["x"]), np.full(n, cfg["m"]), mie_epsilon=-cfg["order"],
                             precision=precision)


def _mie_blocks(an, L):
    """(L, 2, 2) LR Mie matrices A_n(s, t) of one sphere and their inverses."""
    A = np.asarray(an[:4 * L]).reshape(L, 2, 2).transpose(0, 2, 1)   # stored column-major per n
    return A, np.linalg.inv(A)


def _order_of_slots(L):
    """Degree n of every slot of one mode of an order-L block."""
    n_of = np.zeros(L * (L + 2), np.int64)
    for n in range(1, L + 1):
        for m in range(-n, n + 1):
            n_of[_aidx(m, n, 0, L)] = n
    return n_of


def _apply_blocks(B, v, L):
    """Per slot (m, n): the two modes of v (..., 2 L(L+2)) times B_n (L, 2, 2)."""
    h = L * (L + 2)
    n_of = _order_of_slots(L) - 1
    v0, v1 = v[..., :h], v[..., h:]
    out = np.empty_like(v)
    out[..., :h] = B[n_of, 0, 0] * v0 + B[n_of, 0, 1] * v1
    out[..., h:] = B[n_of, 1, 0] * v0 + B[n_of, 1, 1] * v1
    return out


def make_sample(cfg, eps=1e-10):
    """Solve the configuration (mixed precision, the solver's own answer) and
    return features and the targets: the correction of each sphere's exciting
    field, e_i = Mie_i^{-1} (a_i - a_i^0), in its incident-phase frame.  (The
    network predicts e, not a - a^0: high-order coefficients of a are tiny and
    any absolute error there is amplified by the high-order translation terms,
    while Mie_i e_i scales the error of e down with them.)"""
    g = solver_pair(cfg)
    an = g.miecoefcalc()[0]
    L = cfg["order"]
    a0 = g.fixedorsoln(eps=eps, niter=0)["amnp"]
    a = g.fixedorsoln(eps=eps)["amnp"]
    g.close()
    n = len(cfg["pos"])
    nb = 2 * L * (L + 2)
    src, dst = block_map(L)
    _, Ainv = _mie_blocks(an, L)
    phase = np.exp(-1j * cfg["pos"][:, 2])
    t = np.zeros((n, NOUT), np.float32)
    mask = np.zeros((n, NOUT), np.float32)
    for pol in range(2):
        d = (a[:, pol] - a0[:, pol]).reshape(n, nb) * phase[:, None]
        e = _apply_blocks(Ainv, d, L)
        for c_ in range(2):
            cols = pol * 4 * NBH + 2 * dst + c_
            t[:, cols] = (e.real if c_ == 0 else e.imag)[:, src]
            mask[:, cols] = 1.0
    return dict(cfg=cfg, X=node_features(cfg, an), target=t, mask=mask, a0=a0, an=np.asarray(an[:4 * L]))


# ---------------------------------------------------------------------------
# the network
# ---------------------------------------------------------------------------
class WarmStartNet:
    def __init__(self, device, seed=0, bf16=True, hidden=HID, layers=LAYERS):
        import torch
        self.torch = torch
        self.dev = device
        self.H = hidden
        self.layers = layers
        self.bf16 = bf16
        self.L = _lib.lib()
        H = hidden
        shapes = [("enc_w", (NF, H)), ("enc_b", (H,))]
        for t in range(layers):
            shapes += [(f"m{t}_w", (2 * H + EF, H)), (f"m{t}_b", (H,)), (f"u{t}_w1", (H, H)), (f"u{t}_w2", (H, H)),
                       (f"u{t}_b", (H,))]
        shapes += [("out_w", (H, NOUT)), ("out_b", (NOUT,))]
        self.shapes = shapes
        sizes = [int(np.prod(s)) for _, s in shapes]
        self.n = int(sum(sizes))
        rng = np.random.default_rng(seed)
        flat = np.zeros(self.n, np.float32)
        self.off = {}
        o = 0
        for (name, s), sz in zip(shapes, sizes):
            self.off[name] = (o, s)
            if name.endswith("_b"):
                pass
            else:
                fan = s[0]
                scale = (0.1 if name == "out_w" else 1.0) / math.sqrt(fan)
                flat[o:o + sz] = rng.standard_normal(sz).astype(np.float32) * scale
            o += sz
        self.p = torch.from_numpy(flat).to(device)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.pb = torch.zeros(self.n, dtype=torch.bfloat16, device=device)
        self.step_no = 0
        self.msum = None
        self.scale = None   # per-output target scale (fit_scale), set by train()
        self.stream = torch.cuda.current_stream(device).cuda_stream
        self._ck(self.L.mstmg_nn_to_bf16(self.n, _vp(self.p), _vp(self.pb), self.stream))

    # parameter views
    def w(self, name, grad=False, low=False):
        o, s = self.off[name]
        src = self.g if grad else (self.pb if (low and self.bf16) else self.p)
        return src[o:o + int(np.prod(s))].view(*s)

    def _ck(self, rc):
        if rc != 0:
            raise RuntimeError(f"warm-start kernel failed ({rc}): {self.L.mstmg_last_error().decode()}")

    def _gemm(self, A, Bname, C_, transB=False, accumulate=False):
        """C = A @ W (transB: A @ W^T); W in BF16 when enabled."""
        W = self.w(Bname, low=True)
        K_, N_ = (W.shape[0], W.shape[1]) if not transB else (W.shape[1], W.shape[0])
        M = A.shape[0]
        self._ck(self.L.mstmg_nn_gemm(M, N_, K_, _vp(A), A.shape[1], 0, _vp(W), W.shape[1], int(transB),
                                      int(self.bf16), _vp(C_), C_.shape[1], int(accumulate), self.stream))

    def _wgrad(self, A, dZ, name, accumulate=False):
        """dW = A^T dZ (FP32)."""
        G = self.w(name, grad=True)
        self._ck(self.L.mstmg_nn_gemm(A.shape[1], dZ.shape[1], A.shape[0], _vp(A), A.shape[1], 1, _vp(dZ), dZ.shape[1], 0, 0,
                                      _vp(G), G.shape[1], int(accumulate), self.stream))

    def _bias_act(self, Z, bname, act):
        Y = self.torch.empty_like(Z)
        self._ck(self.L.mstmg_nn_bias_act(Z.shape[0], Z.shape[1], _vp(Z), _vp(self.w(bname)), _vp(Y), act, self.stream))
        return Y

    def _act_back(self, Z, bname, dY, act):
        dZ = self.torch.empty_like(Z)
        self._ck(self.L.mstmg_nn_act_back(Z.shape[0], Z.shape[1], _vp(Z), _vp(self.w(bname)), _vp(dY), _vp(dZ), act, self.stream))
        self._ck(self.L.mstmg_nn_colsum(Z.shape[0], Z.shape[1], _vp(dZ), _vp(self.w(bname, grad=True)), self.stream))
        return dZ

    def forward(self, gr):
        """gr: dict(X (Nn,NF), ef (E,EF), dst, src (E,) int32) on the device."""
        torch = self.torch
        Nn, E, H = gr["X"].shape[0], gr["ef"].shape[0], self.H
        cache = {}
        Z0 = torch.empty(Nn, H, device=self.dev)
        self._gemm(gr["X"], "enc_w", Z0)
        h = self._bias_act(Z0, "enc_b", 1)
        cache["Z0"] = Z0
        for t in range(self.layers):
            Ze = torch.empty(E, 2 * H + EF, device=self.dev)
            self._ck(self.L.mstmg_nn_edge_concat(E, H, EF, _vp(gr["dst"]), _vp(gr["src"]), _vp(h), _vp(gr["ef"]), _vp(Ze), self.stream))
            Zm = torch.empty(E, H, device=self.dev)
            self._gemm(Ze, f"m{t}_w", Zm)
            Mm = self._bias_act(Zm, f"m{t}_b", 1)
            agg = torch.zeros(Nn, H, device=self.dev)
            self._ck(self.L.mstmg_nn_scatter_add(E, H, _vp(gr["dst"]), _vp(Mm), _vp(agg), self.stream))
            Zu = torch.empty(Nn, H, device=self.dev)
            self._gemm(h, f"u{t}_w1", Zu)
            self._gemm(agg, f"u{t}_w2", Zu, accumulate=True)
            dh = self._bias_act(Zu, f"u{t}_b", 1)
            cache[t] = dict(h=h, Ze=Ze, Zm=Zm, agg=agg, Zu=Zu)
            self._ck(self.L.mstmg_nn_axpy(dh.numel(), 1.0, _vp(h), _vp(dh), self.stream))   # residual: h + SiLU(...)
            h = dh
        Zo = torch.empty(Nn, NOUT, device=self.dev)
        self._gemm(h, "out_w", Zo)
        y = self._bias_act(Zo, "out_b", 0)
        cache["hL"] = h
        cache["Zo"] = Zo
        return y, cache

    def backward(self, gr, cache, dy):
        torch = self.torch
        Nn, E, H = gr["X"].shape[0], gr["ef"].shape[0], self.H
        self.g.zero_()
        dZo = self._act_back(cache["Zo"], "out_b", dy, 0)
        self._wgrad(cache["hL"], dZo, "out_w")
        dh = torch.empty(Nn, H, device=self.dev)
        self._gemm(dZo, "out_w", dh, transB=True)
        for t in reversed(range(self.layers)):
            c = cache[t]
            dZu = self._act_back(c["Zu"], f"u{t}_b", dh, 1)
            self._wgrad(c["h"], dZu, f"u{t}_w1")
            self._wgrad(c["agg"], dZu, f"u{t}_w2")
            dh_prev = dh   # the residual path, then the update's input gradient added in place
            self._gemm(dZu, f"u{t}_w1", dh_prev, transB=True, accumulate=True)
            dagg = torch.empty(Nn, H, device=self.dev)
            self._gemm(dZu, f"u{t}_w2", dagg, transB=True)
            dM = torch.empty(E, H, device=self.dev)
            self._ck(self.L.mstmg_nn_gather(E, H, _vp(gr["dst"]), _vp(dagg), _vp(dM), 0, self.stream))
            dZm = self._act_back(c["Zm"], f"m{t}_b", dM, 1)
            self._wgrad(c["Ze"], dZm, f"m{t}_w")
            dZe = torch.empty(E, 2 * H + EF, device=self.dev)
            self._gemm(dZm, f"m{t}_w", dZe, transB=True)
            self._ck(self.L.mstmg_nn_edge_concat_back(E, H, EF, _vp(gr["dst"]), _vp(gr["src"]), _vp(dZe), _vp(dh_prev), self.stream))
            dh = dh_prev
        dZ0 = self._act_back(cache["Z0"], "enc_b", dh, 1)
        self._wgrad(gr["X"], dZ0, "enc_w")

    def loss_grad(self, y, target, mask, msum_=None):
        torch = self.torch
        dy = torch.empty_like(y)
        loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        msum = float(self.msum if msum_ is None else msum_)
        self._ck(self.L.mstmg_nn_mse(y.numel(), _vp(y), _vp(target), _vp(mask), msum, _vp(dy), _vp(loss), self.stream))
        return loss, dy

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_no += 1
        self._ck(self.L.mstmg_nn_adam(self.n, _vp(self.p), _vp(self.g), _vp(self.m), _vp(self.v), _vp(self.pb) if self.bf16 else None,
                                      lr, b1, b2, eps, self.step_no, self.stream))

    def state(self):
        return self.p.detach().cpu().numpy().copy()

    def load(self, flat):
        self.p.copy_(self.torch.from_numpy(np.asarray(flat, np.float32)).to(self.dev))
        self._ck(self.L.mstmg_nn_to_bf16(self.n, _vp(self.p), _vp(self.pb), self.stream))


# ---------------------------------------------------------------------------
# graphs, training, inference
# ---------------------------------------------------------------------------
def knn_device(samples, device, k=K_NN):
    """k nearest neighbours of every sphere (library kernel), per configuration."""
    import torch
    L = _lib.lib()
    pos = np.concatenate([s["cfg"]["pos"] for s in samples])
    counts = [len(s["cfg"]["pos"]) for s in samples]
    start = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    scfg = np.repeat(np.arange(len(samples)), counts).astype(np.int32)
    dp = torch.from_numpy(pos).to(device)
    ds = torch.from_numpy(start).to(device)
    dc = torch.from_numpy(scfg).to(device)
    nbr = torch.empty(len(pos) * k, dtype=torch.int32, device=device)
    st = torch.cuda.current_stream(device).cuda_stream
    rc = L.mstmg_nn_knn(len(pos), k, _vp(ds), _vp(dc), _vp(dp), _vp(nbr), st)
    if rc != 0:
        raise RuntimeError("knn kernel failed")
    return nbr.view(len(pos), k).cpu().numpy(), start


def batch_graph(samples, device, with_target=True):
    import torch
    nbr_all, start = knn_device(samples, device)
    X, ef, dst, src, T, M = [], [], [], [], [], []
    for s, (a, b) in zip(samples, zip(start[:-1], start[1:])):
        nbr = nbr_all[a:b] - a
        i, j, e = edge_features(s["cfg"], nbr)
        X.append(s["X"])
        ef.append(e)
        dst.append(i + a)
        src.append(j + a)
        if with_target:
            T.append(s["target"])
            M.append(s["mask"])
    gr = dict(X=torch.from_numpy(np.concatenate(X)).to(device), ef=torch.from_numpy(np.concatenate(ef)).to(device),
              dst=torch.from_numpy(np.concatenate(dst).astype(np.int32)).to(device),
              src=torch.from_numpy(np.concatenate(src).astype(np.int32)).to(device), start=start)
    if with_target:
        mk_ = np.concatenate(M)
        gr["target"] = torch.from_numpy(np.concatenate(T)).to(device)
        gr["mask"] = torch.from_numpy(mk_).to(device)
        gr["msum"] = float(mk_.sum())
    return gr


def _slot_orders():
    """Degree n of every output column (order-9 layout, both polarisations, re/im)."""
    n_of = _order_of_slots(LMAX)
    cols = np.zeros(NOUT, np.int64)
    for pol in range(2):
        for p in range(2):
            for q in range(NBH):
                for c_ in range(2):
                    cols[pol * 4 * NBH + 2 * (q + p * NBH) + c_] = n_of[q]
    return cols


def fit_scale(samples):
    """RMS of the targets per degree n over the training set: the network
    predicts targets divided by it, so every degree weighs alike in the loss."""
    cols = _slot_orders()
    num = np.zeros(LMAX + 1)
    den = np.zeros(LMAX + 1)
    for s in samples:
        t2 = (s["target"] ** 2 * s["mask"]).sum(axis=0)
        mk = s["mask"].sum(axis=0)
        np.add.at(num, cols, t2)
        np.add.at(den, cols, mk)
    rms = np.sqrt(num / np.maximum(den, 1.0))
    rms[rms == 0] = 1.0
    return rms[cols].astype(np.float32)


def train(net, samples, epochs=20, batch=8, lr=1e-3, seed=0, log=None):
    rng = np.random.default_rng(seed)
    net.scale = fit_scale(samples)
    samples = [dict(s, target=(s["target"] / net.scale).astype(np.float32)) for s in samples]
    graphs = [batch_graph(samples[i:i + batch], net.dev) for i in range(0, len(samples), batch)]
    hist = []
    for ep in range(epochs):
        order = rng.permutation(len(graphs))
        tot = 0.0
        for b in order:
            gr = graphs[b]
            y, cache = net.forward(gr)
            loss, dy = net.loss_grad(y, gr["target"], gr["mask"], gr["msum"])
            net.backward(gr, cache, dy)
            net.adam(lr=lr)
            tot += float(loss.item())
        hist.append(tot / len(graphs))
        if log:
            log(f"epoch {ep} loss {hist[-1]:.4e}")
    return hist


def predict_guess(net, sample):
    """x0 = a^0 + e^{i z} Delta a_pred for one configuration (neqns x 2)."""
    gr = batch_graph([sample], net.dev, with_target=False)
    y, _ = net.forward(gr)
    y = y.cpu().numpy()
    if getattr(net, "scale", None) is not None:
        y = y * net.scale
    cfg = sample["cfg"]
    n, L = len(cfg["pos"]), cfg["order"]
    nb = 2 * L * (L + 2)
    src, dst = block_map(L)
    A, _ = _mie_blocks(sample["an"], L)
    phase = np.exp(1j * cfg["pos"][:, 2])
    x0 = np.array(sample["a0"], np.complex128, copy=True)
    for pol in range(2):
        re = y[:, pol * 4 * NBH + 2 * dst]
        im = y[:, pol * 4 * NBH + 2 * dst + 1]
        e = np.zeros((n, nb), np.complex128)
        e[:, src] = re + 1j * im
        x0[:, pol] += (_apply_blocks(A, e, L) * phase[:, None]).reshape(-1)
    return x0


def solve_with_guess(cfg, x0, eps=1e-12, precision="mixed", fallback=1.0):
    """Fixed-orientation solve from x0 (falls back per polarisation to the Mie start)."""
    g = solver_pair(cfg, precision)
    L = _lib.lib()
    ne = g.number_eqns
    x0 = np.asfortranarray(x0, np.complex128)
    amnp = np.zeros((ne, 2), np.complex128, order="F")
    qeff = np.zeros(9 * g.number_spheres)
    qtot = np.zeros(9)
    used = np.zeros(2, np.int32)
    res = np.zeros(2)
    me, mi = ctypes.c_double(0.0), ctypes.c_int(0)
    st = L.mstmg_fixed_orientation_guess(g.ctx, 0.0, 0.0, 1, eps, 10000, api._ptr(x0), fallback, api._ptr(used), api._ptr(res),
                                         api._ptr(amnp), api._ptr(qeff), api._ptr(qtot), ctypes.byref(me), ctypes.byref(mi))
    _lib.check(st, "fixed_orientation_guess")
    stats = g.last_stats()
    g.close()
    return dict(amnp=amnp, qtot=qtot.reshape(3, 3, order="F"), used=used.tolist(), guess_residual=res.tolist(), **stats)


# ---------------------------------------------------------------------------
# the study at scale: configurations solved in ensembles, graphs kept on the GPU
# ---------------------------------------------------------------------------
def _draw_params(rng, n):
    """The parameters of n configurations as sample_config draws them (the
    positions come later, from their own seeds)."""
    out = []
    for _ in range(n):
        nn = int(rng.integers(100, 301))
        x = float(rng.uniform(0.5, 2.0))
        m = complex(rng.uniform(1.3, 1.7), 10.0 ** rng.uniform(-4.0, -1.0))
        fv = float(rng.uniform(0.05, 0.30))
        out.append(dict(n=nn, x=x, m=m, fv=fv, seed=int(rng.integers(0, 2 ** 31 - 1)), order=C.truncation_order(x)))
    return out


def _rsa_positions(p):
    pos, _ = C.rsa_sphere_batched(p["n"], p["x"], p["fv"], seed=p["seed"])
    return np.asarray(pos, np.float64)


def draw_configs(n, seed, workers=0):
    """n configurations of the study (100-300 spheres, x in [0.5, 2], Re m in
    [1.3, 1.7], Im m log-uniform in [1e-4, 0.1], fv in [0.05, 0.30], RSA in a
    bounding sphere with batched candidates), the positions made by a process
    pool (spawned, so it can start after CUDA) when workers > 1."""
    params = _draw_params(np.random.default_rng(seed), n)
    if workers > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(workers) as pool:
            pos = pool.map(_rsa_positions, params, chunksize=16)
    else:
        pos = [_rsa_positions(p) for p in params]
    return [dict(pos=q, x=p["x"], m=p["m"], fv=p["fv"], order=p["order"]) for p, q in zip(params, pos)]


def solve_samples(cfgs, eps=1e-10, batch=32):
    """Training samples of many configurations: the solver's own solutions,
    configurations of one sphere order solved together in ensemble contexts
    (mstmg_ensemble_fixed_orientation), the Mie start a^0 = Mie f and the
    targets formed as make_sample forms them."""
    L_ = _lib.lib()
    by_order = {}
    for k, cfg in enumerate(cfgs):
        by_order.setdefault(cfg["order"], []).append(k)
    out = [None] * len(cfgs)
    for L, idx in sorted(by_order.items()):
        nb = 2 * L * (L + 2)
        src, dst = block_map(L)
        for b0 in range(0, len(idx), batch):
            chunk = idx[b0:b0 + batch]
            ens = api.SphereEnsemble([(cfgs[k]["pos"], np.full(len(cfgs[k]["pos"]), cfgs[k]["x"]), cfgs[k]["m"]) for k in chunk],
                                     mie_epsilon=-L)
            r = ens.fixedorsoln(eps=eps)
            an_all = ens.miecoefcalc()[0]
            pw = np.zeros((ens.number_eqns, 2), np.complex128, order="F")
            _lib.check(L_.mstmg_planewave(ens.ctx, 0.0, 0.0, 1, api._ptr(pw)), "planewave")
            off, start = ens.sphere_offset, ens.config_start
            for c, k in enumerate(chunk):
                cfg = cfgs[k]
                n = len(cfg["pos"])
                i0 = start[c]
                an = np.asarray(an_all[4 * L * i0:4 * L * (i0 + 1)])
                A, Ainv = _mie_blocks(an, L)
                rows = slice(off[start[c]], off[start[c + 1]])
                a = r["amnp"][rows]
                f = pw[rows]
                a0 = np.zeros_like(a)
                for pol in range(2):
                    a0[:, pol] = _apply_blocks(A, f[:, pol].reshape(n, nb), L).reshape(-1)
                phase = np.exp(-1j * cfg["pos"][:, 2])
                t = np.zeros((n, NOUT), np.float32)
                mask = np.zeros((n, NOUT), np.float32)
                for pol in range(2):
                    e = _apply_blocks(Ainv, (a[:, pol] - a0[:, pol]).reshape(n, nb) * phase[:, None], L)
                    for c_ in range(2):
                        cols = pol * 4 * NBH + 2 * dst + c_
                        t[:, cols] = (e.real if c_ == 0 else e.imag)[:, src]
                        mask[:, cols] = 1.0
                out[k] = dict(cfg=cfg, X=node_features(cfg, an), target=t, mask=mask, a0=np.asfortranarray(a0), an=an)
            ens.close()
    return out


def save_net(net, path, meta=None):
    """The trained weights (FP32 masters), the target scale and a description."""
    import json
    np.savez_compressed(path, params=net.state(), scale=net.scale, hidden=net.H, layers=net.layers,
                        meta=json.dumps(meta or {}))


def load_net(path, device):
    import json
    d = np.load(path)
    net = WarmStartNet(device, seed=0, hidden=int(d["hidden"]), layers=int(d["layers"]))
    net.load(d["params"])
    net.scale = d["scale"]
    return net, json.loads(str(d["meta"]))


def evaluate(net, held, fallbacks=(1.0, 0.1), eps=1e-12, precision="mixed"):
    """Held-out configurations: solver iterations and wall time (the guess's
    network inference included) to ||r||/||b|| < 1e-6 from the network's guess
    under each fallback threshold, against the reference's Mie start.  The
    variants of one configuration run back to back in an order that rotates
    from one configuration to the next, after an untimed run of each, so that
    warm-up and clock drift fall on all of them alike."""
    import time
    import torch
    res = {}
    variants = ["mie"] + list(fallbacks)
    t = {v: 0.0 for v in variants}
    it = {v: 0 for v in variants}
    nfb = {v: 0 for v in variants}
    r0 = {v: [] for v in variants}

    def run(s, v, x0, t_inf):
        t0 = time.perf_counter()
        if v == "mie":
            rp = solve_with_guess(s["cfg"], s["a0"], eps=eps, precision=precision, fallback=10.0)
        else:
            rp = solve_with_guess(s["cfg"], x0, eps=eps, precision=precision, fallback=v)
        return rp, time.perf_counter() - t0 + (0.0 if v == "mie" else t_inf)

    for k, s in enumerate(held):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x0 = predict_guess(net, s)
        torch.cuda.synchronize()
        t_inf = time.perf_counter() - t0
        if k == 0:
            for v in variants:
                run(s, v, x0, t_inf)   # untimed
        for v in variants[k % len(variants):] + variants[:k % len(variants)]:
            rp, dt = run(s, v, x0, t_inf)
            t[v] += dt
            it[v] += sum(rp["iterations"])
            r0[v] += rp["guess_residual"]
            if v != "mie":
                nfb[v] += 2 - sum(rp["used"])
    for fb in fallbacks:
        res["fallback_%g" % fb] = dict(fallback=fb, iterations_warm=it[fb], iterations_mie_start=it["mie"],
                                      iteration_ratio=round(it[fb] / max(1, it["mie"]), 4), wall_s_warm=round(t[fb], 2),
                                      wall_s_mie_start=round(t["mie"], 2), wall_ratio=round(t[fb] / max(1e-9, t["mie"]), 4),
                                      mean_initial_residual_warm=float(np.mean(r0[fb])),
                                      mean_initial_residual_mie=float(np.mean(r0["mie"])), fallbacks=nfb[fb],
                                      polarisations=2 * len(held))
    return res


def study_at_scale(n_train=20000, n_eval=1000, epochs=20, batch=16, lr=2e-3, train_seed=5, eval_seed=6, workers=16, device=None,
                   save=None, log=print):
    """The warm-start study as specified: n_train configurations drawn with
    seed 5 and solved by the library (ensembles of one sphere order), the
    network trained on them on the GPU with the library's kernels, n_eval
    held-out configurations drawn with seed 6 evaluated against the Mie start
    with the 1.0 and 0.1 fallback thresholds."""
    import time
    import torch
    dev = device or torch.device("cuda", 0)
    t0 = time.time()
    tr_cfgs = draw_configs(n_train, train_seed, workers)
    ev_cfgs = draw_configs(n_eval, eval_seed, workers)
    t_draw = time.time() - t0
    t0 = time.time()
    graphs, scale_src, ntr = [], [], 0
    net = WarmStartNet(dev, seed=0)
    for b0 in range(0, n_train, 512):
        samples = solve_samples(tr_cfgs[b0:b0 + 512])
        if net.scale is None:
            net.scale = fit_scale(samples)
        for i in range(0, len(samples), batch):
            part = [dict(s, target=(s["target"] / net.scale).astype(np.float32)) for s in samples[i:i + batch]]
            graphs.append(batch_graph(part, dev))
        ntr += len(samples)
        if log:
            log("solved %d / %d training configurations (%.0f s)" % (ntr, n_train, time.time() - t0))
    held = solve_samples(ev_cfgs)
    torch.cuda.synchronize(dev)
    t_gen = time.time() - t0
    rng = np.random.default_rng(0)
    t0 = time.time()
    hist = []
    for ep in range(epochs):
        tot = 0.0
        for b in rng.permutation(len(graphs)):
            gr = graphs[b]
            y, cache = net.forward(gr)
            loss, dy = net.loss_grad(y, gr["target"], gr["mask"], gr["msum"])
            net.backward(gr, cache, dy)
            net.adam(lr=lr * (0.5 if ep >= epochs // 2 else 1.0))
            tot += float(loss.item())
        hist.append(tot / len(graphs))
        if log:
            log("epoch %d loss %.4e" % (ep, hist[-1]))
    torch.cuda.synchronize(dev)
    t_train = time.time() - t0
    del graphs
    t0 = time.time()
    ev = evaluate(net, held)
    t_eval = time.time() - t0
    out = dict(n_train=n_train, n_eval=n_eval, epochs=epochs, batch=batch, draw_s=round(t_draw, 1), gen_s=round(t_gen, 1),
               train_s=round(t_train, 1), eval_s=round(t_eval, 1), loss_first=hist[0], loss_last=hist[-1], **ev)
    if save:
        save_net(net, save, meta=out)
    if log:
        log(out)
    return out


def study(n_train=200, n_eval=16, epochs=60, seed=5, device=None, fallback=1.0, log=print):
    """Generate, train, evaluate: the warm-start study on configurations drawn
    as sample_config draws them.  Returns a summary dict (iterations and
    initial residuals with and without the guess, timing, fallbacks)."""
    import time
    import torch
    dev = device or torch.device("cuda", 0)
    rng = np.random.default_rng(seed)
    t0 = time.time()
    train_set = [make_sample(sample_config(rng)) for _ in range(n_train)]
    held = [make_sample(sample_config(rng)) for _ in range(n_eval)]
    t_gen = time.time() - t0
    net = WarmStartNet(dev, seed=0)
    t0 = time.time()
    hist = train(net, train_set, epochs=epochs, batch=8, lr=2e-3)
    torch.cuda.synchronize(dev)
    t_train = time.time() - t0
    out = dict(n_train=n_train, n_eval=n_eval, epochs=epochs, gen_s=round(t_gen, 1), train_s=round(t_train, 1),
               loss_first=hist[0], loss_last=hist[-1])
    for fb_name, fb in (("with_fallback", fallback), ("guess_always", 10.0)):
        it_p = it_w = nfb = 0
        rp_l, rw_l = [], []
        for s in held:
            x0 = predict_guess(net, s)
            rw = solve_with_guess(s["cfg"], x0, eps=1e-12, precision="mixed", fallback=fb)
            rp = solve_with_guess(s["cfg"], s["a0"], eps=1e-12, precision="mixed", fallback=10.0)
            it_p += sum(rp["iterations"])
            it_w += sum(rw["iterations"])
            nfb += 2 - sum(rw["used"])
            rp_l += rp["guess_residual"]
            rw_l += rw["guess_residual"]
        out[fb_name] = dict(fallback=fb, iterations_mie_start=it_p, iterations_warm=it_w, iteration_ratio=round(it_w / it_p, 4),
                            mean_initial_residual_mie=float(np.mean(rp_l)), mean_initial_residual_warm=float(np.mean(rw_l)),
                            fallbacks=nfb)
    if log:
        log(out)
    return out


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train and evaluate the learned warm start")
    ap.add_argument("--train", type=int, default=20000)
    ap.add_argument("--eval", type=int, default=1000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--workers", type=int, default=16)
    ap.add_argument("--save", default=None, help="write the trained network here (.npz)")
    a = ap.parse_args()
    print(json.dumps(study_at_scale(a.train, a.eval, a.epochs, workers=a.workers, save=a.save,
                                    log=lambda m: print(m, flush=True))))
