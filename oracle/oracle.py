"""ctypes front end of the CPU oracle (oracle/libmstm_oracle.so).

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA product; only
tests/, __graft_entry__.smoke() and the CPU legs of bench.py import it.  The
C restatement it wraps follows MSTM's Fortran routines line by line (see the
citations in mstm_oracle.c).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmstm_oracle.so")
_lib = None

c_int = ctypes.c_int
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
P = ctypes.POINTER


def build():
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.restype = c_void_p
        L.orc_create.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_double, c_int, c_int]
        L.orc_destroy.argtypes = [c_void_p]
        L.orc_neqns.argtypes = [c_void_p]
        L.orc_neqns.restype = c_int
        L.orc_orders.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        L.orc_mie_coefs.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
        L.orc_sphereinteraction.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int]
        L.orc_sphereinteraction_ex.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int]
        L.orc_hosts.argtypes = [c_void_p, c_void_p]
        L.orc_hosts.restype = c_int
        L.orc_host_mie_coefs.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        L.orc_cbicg.argtypes = [c_void_p, c_int, c_double, c_void_p, c_void_p, c_int, P(c_int), P(c_double)]
        L.orc_cbicg.restype = c_int
        L.orc_planewave.argtypes = [c_void_p, c_double, c_double, c_int, c_void_p]
        L.orc_fixedorsoln.argtypes = [c_void_p, c_double, c_double, c_int, c_double, c_int, c_void_p, c_void_p,
                                      P(c_double), P(c_int), c_int]
        L.orc_fixedorsoln.restype = c_int
        L.orc_qtotcalc.argtypes = [c_void_p, c_void_p, c_void_p]
        L.orc_last_iterations.argtypes = [c_void_p, c_void_p]
        L.orc_vol_radius.argtypes = [c_void_p]
        L.orc_vol_radius.restype = c_double
        L.orc_x_rotcoef.argtypes = [c_double, c_int, c_int, c_void_p]
        L.orc_x_vcfunc.argtypes = [c_int, c_int, c_int, c_int, c_void_p]
        L.orc_x_atcdim.argtypes = [c_int, c_int]
        L.orc_x_atcdim.restype = c_int
        L.orc_x_moffset.argtypes = [c_int, c_int, c_int]
        L.orc_x_moffset.restype = c_int
        L.orc_x_axial.argtypes = [c_int, c_double, c_double, c_double, c_int, c_int, c_void_p]
        L.orc_x_mieoa.argtypes = [c_double, c_double, c_double, c_double, P(c_int), P(c_double), P(c_double),
                                  P(c_double), c_void_p, c_void_p]
        L.orc_x_translate_rot.argtypes = [c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_int, c_int]
        L.orc_x_gentranmatrix.argtypes = [c_int, c_int, c_void_p, c_int, c_void_p]
        L.orc_x_cspherebessel.argtypes = [c_int, c_double, c_double, c_void_p, c_void_p]
        L.orc_x_crichankel.argtypes = [c_int, c_double, c_double, c_void_p]
        L.orc_x_direct_solve.argtypes = [c_void_p, c_void_p, c_void_p]
        L.orc_x_multmie.argtypes = [c_void_p, c_int, c_void_p, c_void_p]
        L.orc_x_qeff.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        L.orc_tranordertest.argtypes = [c_double, c_double, c_int, c_double]
        L.orc_tranordertest.restype = c_int
        L.orc_t_matrix_order.argtypes = [c_void_p, c_double, c_int, c_void_p, c_void_p]
        L.orc_t_matrix_order.restype = c_int
        L.orc_merge_to_common_origin.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]
        L.orc_fosmexpansion.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
        L.orc_fosmcalc.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_void_p]
        L.orc_distribute_from_common_origin.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p]
        L.orc_tmatrix_solution.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_double, c_double, c_int, c_void_p,
                                           c_void_p, P(c_int), P(c_int), P(c_double)]
        L.orc_tmatrix_solution.restype = c_int
        L.orc_tmatrix_symmetrize.argtypes = [c_int, c_void_p, c_void_p]
        L.orc_tmatrix_qext_qsca.argtypes = [c_int, c_void_p, c_double, P(c_double), P(c_double)]
        L.orc_ranorientscatmatrix.argtypes = [c_int, c_void_p, c_double, c_void_p, c_void_p]
        L.orc_fft_setup.argtypes = [c_void_p, c_double, c_double, c_int, c_int, c_void_p, P(c_double)]
        L.orc_fft_setup.restype = c_int
        L.orc_fft_near_pairs.argtypes = [c_void_p, c_void_p, c_void_p]
        L.orc_fft_near_pairs.restype = c_int
        L.orc_ranorienscatmatrixcalc.argtypes = [c_double, c_void_p, c_int, c_void_p]
        L.orc_scatteringmatrix.argtypes = [c_int, c_void_p, c_double, c_double, c_int, c_double, c_void_p, c_void_p]
        L.orc_incident_plane_scattering.argtypes = [c_int, c_void_p, c_int, c_int, c_double, c_double, c_double, c_int,
                                                    c_double, c_void_p]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(c_void_p)


class Oracle:
    """FP64 CPU restatement of one MSTM sphere cluster (free space, medium index 1;
    spheres may lie inside others, as the reference's host spheres).

    positions (N,3), radii (N,), ref_index (N,) complex; mie_eps as the
    reference's ``mie_epsilon`` (negative -L forces order L).
    """

    def __init__(self, positions, radii, ref_index, mie_eps=-7.0, store_matrix=True, nthreads=1):
        self.L = lib()
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        rad = np.ascontiguousarray(np.asarray(radii, dtype=np.float64))
        ri = np.asarray(ref_index, dtype=np.complex128)
        if ri.ndim == 0:
            ri = np.full(len(rad), ri)
        ri2 = np.ascontiguousarray(np.stack([ri.real, ri.imag], axis=1))
        self.n = len(rad)
        self.pos, self.rad = pos, rad
        self.ctx = self.L.orc_create(self.n, _p(pos), _p(rad), _p(ri2), float(mie_eps), int(store_matrix),
                                     int(nthreads))
        self.neqns = self.L.orc_neqns(self.ctx)
        self.order = np.zeros(self.n, np.int32)
        self.offset = np.zeros(self.n + 1, np.int32)
        self.mie_offset = np.zeros(self.n + 1, np.int32)
        self.L.orc_orders(self.ctx, _p(self.order), _p(self.offset), _p(self.mie_offset))

    def close(self):
        if self.ctx:
            self.L.orc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mie(self):
        nt = int(self.mie_offset[-1])
        an = np.zeros(nt, np.complex128)
        ai = np.zeros(nt, np.complex128)
        qe = np.zeros(self.n)
        qa = np.zeros(self.n)
        self.L.orc_mie_coefs(self.ctx, _p(an), _p(ai), _p(qe), _p(qa))
        return an, ai, qe, qa

    def sphereinteraction(self, ain, con_tran=None, mie_mult=None, initial_run=False, skip_external=False):
        ain = np.asfortranarray(np.asarray(ain, np.complex128).reshape(self.neqns, -1, order="F"))
        nrhs = ain.shape[1]
        out = np.zeros((self.neqns, nrhs), np.complex128, order="F")
        ct = np.array(con_tran if con_tran is not None else [0] * nrhs, np.int32)
        mm = np.array(mie_mult if mie_mult is not None else [1] * nrhs, np.int32)
        self.L.orc_sphereinteraction_ex(self.ctx, nrhs, _p(ain), _p(out), _p(ct), _p(mm), int(initial_run),
                                        int(skip_external))
        return out

    def hosts(self):
        """(host of each sphere, -1 for none; number of spheres with a host)"""
        h = np.zeros(self.n, np.int32)
        nh = self.L.orc_hosts(self.ctx, _p(h))
        return h, nh

    def host_mie(self):
        """The D, U, V coefficients of the host spheres (zero for the others)."""
        nt = int(self.mie_offset[-1])
        d, u, v = (np.zeros(nt, np.complex128) for _ in range(3))
        self.L.orc_host_mie_coefs(self.ctx, _p(d), _p(u), _p(v))
        return d, u, v

    def cbicg(self, pnp, x0, niter=10000, eps=1e-6, initialize=True):
        pnp = np.ascontiguousarray(pnp, np.complex128)
        x = np.array(x0, np.complex128, copy=True)
        it = c_int(0)
        err = c_double(0.0)
        rc = self.L.orc_cbicg(self.ctx, niter, eps, _p(pnp), _p(x), int(initialize), ctypes.byref(it),
                              ctypes.byref(err))
        return x, it.value, err.value, rc

    def planewave(self, alpha=0.0, sinc=0.0, direction=1):
        out = np.zeros((self.neqns, 2), np.complex128, order="F")
        self.L.orc_planewave(self.ctx, alpha, sinc, direction, _p(out))
        return out

    def fixedorsoln(self, eps=1e-6, niter=10000, alpha=0.0, sinc=0.0, direction=1, direct=False):
        amnp = np.zeros((self.neqns, 2), np.complex128, order="F")
        qeff = np.zeros((3, 3, self.n), np.float64, order="F")
        maxerr = c_double(0.0)
        maxiter = c_int(0)
        st = self.L.orc_fixedorsoln(self.ctx, alpha, sinc, direction, eps, niter, _p(amnp), _p(qeff),
                                    ctypes.byref(maxerr), ctypes.byref(maxiter), int(direct))
        qtot = np.zeros((3, 3), np.float64, order="F")
        self.L.orc_qtotcalc(self.ctx, _p(qeff), _p(qtot))
        iters = np.zeros(2, np.int32)
        self.L.orc_last_iterations(self.ctx, _p(iters))
        return dict(amnp=amnp, qeff=qeff, qtot=qtot, status=st, maxerr=maxerr.value, maxiter=maxiter.value,
                    iterations=iters.tolist())

    def direct_solve(self, pnp):
        pnp = np.ascontiguousarray(pnp, np.complex128)
        out = np.zeros(self.neqns, np.complex128)
        self.L.orc_x_direct_solve(self.ctx, _p(pnp), _p(out))
        return out

    def multmie(self, x, idir=1):
        x = np.ascontiguousarray(x, np.complex128)
        out = np.zeros(self.neqns, np.complex128)
        self.L.orc_x_multmie(self.ctx, idir, _p(x), _p(out))
        return out

    def vol_radius(self):
        return self.L.orc_vol_radius(self.ctx)

    def t_matrix_order(self, trans_eps=1.0e-5, maxt=100):
        origin = np.zeros(3)
        to = np.zeros(self.n, np.int32)
        nt = self.L.orc_t_matrix_order(self.ctx, trans_eps, maxt, _p(origin), _p(to))
        return nt, origin, to

    def merge_to_common_origin(self, amnp, nodrt, origin, trans_order):
        """amnp: (neqns, npol) -> (nb(nodrt), npol) common-origin TE/TM coefficients."""
        amnp = np.asfortranarray(amnp, np.complex128)
        nb = 2 * nodrt * (nodrt + 2)
        out = np.zeros((nb, amnp.shape[1]), np.complex128, order="F")
        to = np.ascontiguousarray(trans_order, np.int32)
        r0 = np.ascontiguousarray(origin, np.float64)
        for p in range(amnp.shape[1]):
            col = np.ascontiguousarray(amnp[:, p])
            o = np.zeros(nb, np.complex128)
            self.L.orc_merge_to_common_origin(self.ctx, nodrt, _p(col), _p(r0), _p(to), _p(o))
            out[:, p] = o
        return out

    def fft_setup(self, cell_volume_fraction=0.2, d_cell=0.0, node_order=-1, neighbor_node_model=2):
        """Switch to the FFT translation (fft_translation-5.f90): near pairs direct,
        the rest through cell nodes.  Returns dict(cell_dim, d_cell, node_order, npairs)."""
        cd = np.zeros(3, np.int32)
        dc = c_double(0.0)
        no = self.L.orc_fft_setup(self.ctx, cell_volume_fraction, d_cell, node_order, neighbor_node_model, _p(cd),
                                  ctypes.byref(dc))
        npair = self.L.orc_fft_near_pairs(self.ctx, None, None)
        return dict(cell_dim=cd.tolist(), d_cell=dc.value, node_order=no, npairs=npair)

    def distribute_from_common_origin(self, amnp0, nodrt, origin):
        """amnp0: (nb(nodrt), nrhs) LR common-origin coefficients -> (neqns, nrhs) regular expansions about each sphere."""
        amnp0 = np.asfortranarray(amnp0, np.complex128)
        out = np.zeros((self.neqns, amnp0.shape[1]), np.complex128, order="F")
        r0 = np.ascontiguousarray(origin, np.float64)
        for p in range(amnp0.shape[1]):
            col = np.ascontiguousarray(amnp0[:, p])
            o = np.zeros(self.neqns, np.complex128)
            self.L.orc_distribute_from_common_origin(self.ctx, nodrt, _p(col), _p(r0), _p(o))
            out[:, p] = o
        return out

    def tmatrix_solution(self, tmo=None, trans_eps=1.0e-5, maxt=100, solution_eps=1.0e-6, convergence_eps=1.0e-6,
                         max_iterations=10000):
        """tmatrix_solution: dict(tmat (nblkt, nblkt), order, sphere_qeff (3, N), qtot (ext, abs, sca),
        status, maxiter, maxerr, origin, trans_order)."""
        nt, origin, to = self.t_matrix_order(trans_eps, maxt)
        if tmo is None:
            tmo = nt
        nblkt = 2 * tmo * (tmo + 2)
        tmat = np.zeros((nblkt, nblkt), np.complex128, order="F")
        sq = np.zeros((3, self.n), np.float64, order="F")
        used, mi, me = c_int(0), c_int(0), c_double(0.0)
        st = self.L.orc_tmatrix_solution(self.ctx, tmo, _p(np.ascontiguousarray(to, np.int32)), _p(origin), solution_eps,
                                         convergence_eps, max_iterations, _p(tmat), _p(sq), ctypes.byref(used),
                                         ctypes.byref(mi), ctypes.byref(me))
        xv = self.vol_radius()
        r2 = np.asarray(self.rad) ** 2 / xv ** 2
        qt = (sq * r2[None, :]).sum(axis=1)
        qtot = np.array([qt[0], qt[1], qt[0] + qt[2] - qt[1]])
        return dict(tmat=tmat, order=used.value, tmo=tmo, sphere_qeff=sq, qtot=qtot, status=st, maxiter=mi.value,
                    maxerr=me.value, origin=origin, trans_order=to)

    def scattering(self, amnp, trans_eps=1.0e-5, maxt=100, nangles=181):
        """fosmexpansion + fosmcalc: returns dict(ntot, s00.., g, smat (nangles,4,4))."""
        nt, origin, to = self.t_matrix_order(trans_eps, maxt)
        a0 = self.merge_to_common_origin(amnp, nt, origin, to)
        return gsf_scattering(nt, a0, nangles) | dict(t_matrix_order=nt, amnp0=a0)


def gsf_scattering(nt, a0, nangles=181):
    L = lib()
    W = 2 * nt + 1
    s = [np.zeros(16 * W) for _ in range(4)]
    a0 = np.asfortranarray(a0, np.complex128)
    L.orc_fosmexpansion(nt, _p(a0), _p(s[0]), _p(s[1]), _p(s[2]), _p(s[3]))
    smat = np.zeros((nangles, 4, 4))
    pi_ref = float(np.float32(np.pi))
    for i in range(nangles):
        ct = np.cos(pi_ref / 180.0 * (0.0 + 180.0 * (i / (nangles - 1))))
        if ct == 1.0:
            ct = 0.9999999
        if ct == -1.0:
            ct = -0.9999999
        sm = np.zeros(16)
        L.orc_fosmcalc(nt, _p(s[0]), _p(s[1]), _p(s[2]), _p(s[3]), ct, _p(sm))
        smat[i] = sm.reshape(4, 4, order="F")
    s00 = s[0].reshape(W, 4, 4).transpose(0, 2, 1)   # [w][i][j]
    g = s00[1, 0, 0] / (3.0 * s00[0, 0, 0])
    return dict(s00=s[0], s02=s[1], sp22=s[2], sm22=s[3], g=g, smat=smat)


def rotcoef(cbe, kmax, nmax):
    L = lib()
    dc = np.zeros((nmax * (nmax + 2) + 1, 2 * kmax + 1), np.float64)
    L.orc_x_rotcoef(cbe, kmax, nmax, _p(dc))
    return dc  # dc[nk, m+kmax]


def vcfunc(m, n, k, l):
    L = lib()
    v = np.zeros(n + l + 1)
    L.orc_x_vcfunc(m, n, k, l, _p(v))
    return v


def atcdim(n, l):
    return lib().orc_x_atcdim(n, l)


def moffset(m, n, l):
    return lib().orc_x_moffset(m, n, l)


def axial(itype, r, ri, nmax, lmax):
    L = lib()
    ac = np.zeros(atcdim(nmax, lmax), np.complex128)
    L.orc_x_axial(itype, r, complex(ri).real, complex(ri).imag, nmax, lmax, _p(ac))
    return ac


def mieoa(x, ri, qeps):
    L = lib()
    nodr = c_int(0)
    if qeps < 0:
        n = int(np.ceil(-qeps))
    else:
        n = 200
    anp = np.zeros(4 * max(n, 1) + 4 * 64, np.complex128)
    ainv = np.zeros_like(anp)
    qe, qs, qa = c_double(), c_double(), c_double()
    L.orc_x_mieoa(x, complex(ri).real, complex(ri).imag, qeps, ctypes.byref(nodr), ctypes.byref(qe),
                  ctypes.byref(qs), ctypes.byref(qa), _p(anp), _p(ainv))
    nd = nodr.value
    return dict(order=nd, qext=qe.value, qsca=qs.value, qabs=qa.value, anp=anp[:4 * nd].reshape(nd, 2, 2),
                anp_inv=ainv[:4 * nd].reshape(nd, 2, 2))


def translate_rot(ns, nt, rvec, a, vtype=3, sop=False, top=False):
    L = lib()
    rv = np.ascontiguousarray(rvec, np.float64)
    a = np.ascontiguousarray(a, np.complex128)
    g = np.zeros(2 * nt * (nt + 2), np.complex128)
    L.orc_x_translate_rot(ns, nt, _p(rv), vtype, _p(a), _p(g), int(sop), int(top))
    return g


def gentranmatrix(ns, nt, rvec, vtype=3):
    L = lib()
    rv = np.ascontiguousarray(rvec, np.float64)
    nbs, nbt = ns * (ns + 2), nt * (nt + 2)
    ac = np.zeros(nbt * nbs * 2, np.complex128)
    L.orc_x_gentranmatrix(ns, nt, _p(rv), vtype, _p(ac))
    return ac.reshape(2, nbs, nbt).transpose(2, 1, 0)  # [row kla, col mna, mode]


def tmatrix_symmetrize(tmo, tmat):
    """The complex(4) T matrix as the random-orientation reader fills it."""
    nblkt = 2 * tmo * (tmo + 2)
    tmat = np.asfortranarray(tmat, np.complex128)
    tc = np.zeros((nblkt, nblkt), np.complex64, order="F")
    lib().orc_tmatrix_symmetrize(tmo, _p(tmat), _p(tc))
    return tc


def tmatrix_qext_qsca(tmo, tmat, xv):
    tmat = np.asfortranarray(tmat, np.complex128)
    qe, qs = c_double(0.0), c_double(0.0)
    lib().orc_tmatrix_qext_qsca(tmo, _p(tmat), xv, ctypes.byref(qe), ctypes.byref(qs))
    return qe.value, qs.value


def ranorientscatmatrix(tmo, tmat, rimed_re=1.0, nangles=181):
    """Orientation-averaged scattering matrix from the T matrix: dict(sm, smcf
    (2tmo+1, 4, 4) expansion coefficients [w][i][j], smat (nangles, 4, 4) at
    theta_i = i*pi/(nangles-1) with the reference's pi, coherent = smcf[0,0,0])."""
    L_ = lib()
    W = 2 * tmo + 1
    sm = np.zeros(16 * W)
    smcf = np.zeros(16 * W)
    tmat = np.asfortranarray(tmat, np.complex128)
    L_.orc_ranorientscatmatrix(tmo, _p(tmat), rimed_re, _p(sm), _p(smcf))
    pi_ref = float(np.float32(np.pi))
    smat = np.zeros((nangles, 4, 4))
    for i in range(nangles):
        ct = np.cos(float(i) * pi_ref / float(nangles - 1))
        o = np.zeros(16)
        L_.orc_ranorienscatmatrixcalc(ct, _p(sm), 2 * tmo, _p(o))
        smat[i] = o.reshape(4, 4, order="F")
    sm3 = sm.reshape(W, 4, 4).transpose(0, 2, 1)
    cf3 = smcf.reshape(W, 4, 4).transpose(0, 2, 1)
    return dict(sm=sm3, smcf=cf3, smat=smat, coherent=cf3[0, 0, 0], sm_raw=sm, smcf_raw=smcf)


def scatteringmatrix(nodrt, amn0, ct, phi, rotate=False, rimed_re=1.0):
    """scatteringmatrix (normalize_s11 false) at one direction: (sa[4], sm (4,4))."""
    a0 = np.asfortranarray(amn0, np.complex128)
    sa = np.zeros(4, np.complex128)
    sm = np.zeros(16)
    lib().orc_scatteringmatrix(nodrt, _p(a0), ct, phi, int(rotate), rimed_re, _p(sa), _p(sm))
    return sa, sm.reshape(4, 4, order="F")


def incident_plane_scattering(nodrt, amn0, increment=1.0, alpha=0.0, rotate=False, rimed_re=1.0):
    """The non-azimuth-averaged scattering matrix of a single-origin expansion
    over theta = -180..180 degrees (udim = floor(180.00001/increment)):
    returns (theta (2udim+1,), smat (2udim+1, 4, 4))."""
    udim = int(np.floor(180.00001 / increment))
    ldim, amax = -udim, 180.0
    amin = amax * (-1 if udim > 0 else 0)
    a0 = np.asfortranarray(amn0, np.complex128)
    n = udim - ldim + 1
    sm = np.zeros(16 * n)
    lib().orc_incident_plane_scattering(nodrt, _p(a0), ldim, udim, amin, amax, alpha, int(rotate), rimed_re, _p(sm))
    theta = np.array([amin + (i - ldim) / (udim - ldim) * (amax - amin) for i in range(ldim, udim + 1)])
    return theta, sm.reshape(n, 4, 4).transpose(0, 2, 1)
