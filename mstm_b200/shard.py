"""One sphere cluster sharded over the ranks of a torch.distributed group.

MSTM parallelises a single cluster by dealing the sphere pairs round-robin
to the ranks of its MPI group and summing every rank's part of the
translation with an allreduce (the task loop of external_to_external_expansion,
december2023/mstm-modules-33.f90:6466-6474, and the reduction in
mstm-scatprops-26.f90:152-156); the BiCG iteration around it runs on every
rank alike (mstm-solver-8.f90:654-949).  Here each rank's context keeps one
shard of the tiles of pairs (mstmg_set_pair_shard), `interaction` sums the
ranks' parts with `all_reduce` (NCCL between GPUs, gloo on CPU), and
`cbicg` is the reference's iteration on the summed products, with every
vector replicated on every rank.
"""
import ctypes

import numpy as np
import torch

from . import _lib, api


def _dotc(a, b):
    """Fortran dot_product(a, b) = sum(conj(a) b)."""
    return torch.vdot(a, b)


def cbicg(interaction, pnp, x, eps, niter, initialize=True):
    """MSTM's complex biconjugate gradient (cbicg, mstm-solver-8.f90:654-949,
    normalize_solution_error true) for (I - M H) x = pnp.

    interaction(X, con_tran, initial_run) returns (M H) X for the columns of
    X (rows of the (k, neqns) tensor), column r a conjugate-transpose
    product where con_tran[r] is 1, as sphereinteraction does.  x is the
    initial guess (updated in place).  Returns (x, iterations, error, status):
    status 2 for the reference's breakdown (a zero denominator)."""
    if float(torch.abs(_dotc(pnp, pnp))) == 0.0:
        return x, 0, 0.0, 0
    enorm = float(_dotc(pnp, pnp).real)
    cr = interaction(x[None, :], [0], initialize)[0]
    cr = pnp - x + cr
    cq = torch.conj(cr)
    cw = cq.clone()
    cp = cr.clone()
    csk = torch.sum(cr * cr)   # dot_product(conjg(cr), cr): no conjugate
    err, it = 0.0, 0
    if float(torch.abs(csk)) == 0.0:
        return x, 0, 0.0, 0
    status = 0
    for it in range(1, niter + 1):
        out = interaction(torch.stack([cp, cw]), [0, 1], False)
        cap = cp - out[0]
        caw = cw - out[1]
        cak = _dotc(cw, cap)
        if float(torch.abs(cak)) == 0.0:
            status = 2
            break
        cak = csk / cak
        x += cak * cp
        cr = cr - cak * cap
        cq = cq - torch.conj(cak) * caw
        csk2 = _dotc(cq, cr)
        err = float(_dotc(cr, cr).real) / enorm
        if err < eps or float(torch.abs(csk)) == 0.0:
            break
        cbk = csk2 / csk
        csk = csk2
        cp = cr + cbk * cp
        cw = cq + torch.conj(cbk) * cw
    return x, it, err, status


def summed(local, group=None):
    """interaction(X, con_tran, initial_run) whose result is the sum over the
    ranks of `group` of local(X, con_tran, initial_run) (an all_reduce of
    the real and imaginary parts; every rank gets the whole product)."""
    import torch.distributed as dist

    def f(X, con_tran, initial_run):
        Y = local(X, con_tran, initial_run)
        if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
            dist.all_reduce(torch.view_as_real(Y), group=group)
        return Y
    return f


class ShardedCluster:
    """A SphereCluster (FP64) whose pair translations are split over the ranks
    of `group` (the default group; one rank per GPU).  Every rank builds the
    same cluster; rank r translates the tiles t with t % world == r.
    fixedorsoln() solves both polarisations with the reference's BiCG on the
    summed interactions and returns what SphereCluster.fixedorsoln returns."""

    def __init__(self, positions, radii, ref_index, group=None, mie_epsilon=1.0e-6, device=None, **kw):
        import torch.distributed as dist
        self.group = group
        on = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if on else 0
        self.world = dist.get_world_size(group) if on else 1
        dev = torch.cuda.current_device() if device is None else int(device)
        self.device = torch.device("cuda", dev)
        self.g = api.SphereCluster(positions, radii, ref_index, mie_epsilon=mie_epsilon, precision="fp64", device=dev, **kw)
        if self.world > 1:
            self.g.set_pair_shard(self.rank, self.world)
        self.neqns = self.g.number_eqns
        self.interaction = summed(self._local, group)

    def _local(self, X, con_tran, initial_run):
        X = X.contiguous()
        Y = torch.empty_like(X)
        k = X.shape[0]
        ct = np.ascontiguousarray(np.asarray(con_tran, np.int32))
        mm = np.ones(k, np.int32)
        torch.cuda.synchronize(self.device)
        _lib.check(self.g._L.mstmg_interaction(self.g.ctx, k, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(Y.data_ptr()),
                                               api._ptr(ct), api._ptr(mm), int(initial_run)), "sphereinteraction")
        return Y

    def fixedorsoln(self, eps=1.0e-6, niter=10000, alpha=0.0, sinc=0.0, direction=1):
        pnp = torch.as_tensor(np.ascontiguousarray(self.g.fixed_orientation_rhs(alpha, sinc, direction).T), device=self.device)
        amnp = np.zeros((self.neqns, 2), np.complex128, order="F")
        its, errs, st = [0, 0], [0.0, 0.0], 0
        for p in range(2):
            x = pnp[p].clone()   # the Mie solution start (mstm-solver-8.f90:482-483)
            x, its[p], errs[p], s = cbicg(self.interaction, pnp[p], x, eps, niter, initialize=(p == 0))
            st = max(st, 1 if s == 2 else 0)
            amnp[:, p] = x.cpu().numpy()
        if its[1] > niter or errs[1] > eps:
            st = 1
        q = self.g.efficiencies(amnp, alpha, sinc, direction)
        return dict(amnp=amnp, qeff=q["qeff"], qtot=q["qtot"], maxerr=errs[1], maxiter=its[1], istat=st, iterations=its)

    def close(self):
        self.g.close()
