"""Host-side mirror of MSTM's solver call surface, backed by the CUDA library.

Names and argument meanings follow the Fortran routines they replace
(dmckwski/MSTM, december2023 tree):

=====================  ==========================================================
``SphereCluster``      spheredata + mie module state, miecoefcalc
                       (mstm-modules-33.f90:5088-5131, 5301-5407)
``sphereinteraction``  sphereinteraction (mstm-scatprops-26.f90:25-180)
``cbicg``              cbicg (mstm-solver-8.f90:654-949)
``sphereplanewavecoef``sphereplanewavecoef (mstm-scatprops-26.f90:217-284)
``fixedorsoln``        fixedorsoln (mstm-solver-8.f90:350-569)
``qtotcalc``           qtotcalc (mstm-scatprops-26.f90:872-912)
=====================  ==========================================================

Vectors are complex128 numpy arrays in MSTM's layout (each sphere block is
a(0:L+1,1:L,1:2) column-major).  All arithmetic runs on the GPU; the status
conventions match the reference (istat 0 converged, 1 not converged) and
errors raise ``MstmgError``.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import c_double, c_int, check

PRECISIONS = {"fp64": 0, "mixed": 1}


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class _Context:
    """What a cluster context and an ensemble context share: lifetime, the
    Mie coefficients, positions, the interaction matvec and solve statistics."""

    def close(self):
        if self.ctx:
            self._L.mstmg_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def vol_radius(self):
        return self._L.mstmg_vol_radius(self.ctx)

    def set_positions(self, positions):
        pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
        check(self._L.mstmg_ctx_set_positions(self.ctx, _ptr(pos)), "set_positions")
        self.positions = pos

    def host_spheres(self):
        """findhostspheres: (the sphere holding each sphere, -1 for none;
        the number of spheres with a host)."""
        h = np.zeros(self.number_spheres, np.int32)
        nh = self._L.mstmg_host_spheres(self.ctx, _ptr(h))
        if nh < 0:
            check(nh, "host_spheres")
        return h, nh

    def host_mie_coefficients(self):
        """The D, U, V Mie coefficients of the host spheres (an_mie layout,
        zero for spheres holding no others)."""
        nt = int(4 * self.sphere_order.sum())
        d, u, v = (np.zeros(nt, np.complex128) for _ in range(3))
        check(self._L.mstmg_host_mie_coefficients(self.ctx, _ptr(d), _ptr(u), _ptr(v)), "host_mie")
        return d, u, v

    def miecoefcalc(self):
        nt = int(4 * self.sphere_order.sum())
        an = np.zeros(nt, np.complex128)
        qe = np.zeros(self.number_spheres)
        qa = np.zeros(self.number_spheres)
        check(self._L.mstmg_mie_coefficients(self.ctx, _ptr(an), _ptr(qe), _ptr(qa)), "mie")
        return an, qe, qa

    def sphereinteraction(self, ain, con_tran=None, mie_mult=None, initial_run=False):
        ain = np.asfortranarray(np.asarray(ain, np.complex128).reshape(self.number_eqns, -1, order="F"))
        nrhs = ain.shape[1]
        out = np.zeros((self.number_eqns, nrhs), np.complex128, order="F")
        ct = np.array(con_tran if con_tran is not None else [0] * nrhs, np.int32)
        mm = np.array(mie_mult if mie_mult is not None else [1] * nrhs, np.int32)
        check(self._L.mstmg_interaction(self.ctx, nrhs, _ptr(ain), _ptr(out), _ptr(ct), _ptr(mm), int(initial_run)),
              "sphereinteraction")
        return out


    def last_stats(self):
        it = np.zeros(2, np.int32)
        outer, p64, p32 = c_int(0), c_int(0), c_int(0)
        check(self._L.mstmg_last_stats(self.ctx, _ptr(it), ctypes.byref(outer), ctypes.byref(p64), ctypes.byref(p32)),
              "stats")
        return dict(iterations=it.tolist(), outer=outer.value, passes64=p64.value, passes32=p32.value,
                    host_syncs=self._L.mstmg_last_host_syncs(self.ctx))

class SphereCluster(_Context):
    """One cluster of external spheres in a medium (free space by default).

    positions: (N,3); radii: (N,) size parameters; ref_index: (N,) complex or scalar.
    mie_epsilon: MSTM's mie_epsilon (negative -L forces order L).
    precision: "fp64" (drop-in) or "mixed" (FP32 Krylov passes from FP64 true
    residuals; mixed_solver 2 = restarted GMRES, the default).
    """

    def __init__(self, positions, radii, ref_index, mie_epsilon=1.0e-6, precision="fp64", device=0,
                 medium_index=1.0, inner_eps=1.0e-8, max_outer=30, generic_kernel=False, tile_ctas_per_sm=0, fp32_chunk=0,
                 mixed_solver=2, gmres_restart=0, tensor_core=0, tile_pairs=0):
        self._L = _lib.lib()
        pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
        rad = np.ascontiguousarray(np.asarray(radii, np.float64).reshape(-1))
        n = len(rad)
        ri = np.asarray(ref_index, np.complex128)
        if ri.ndim == 0:
            ri = np.full(n, ri)
        ri2 = np.ascontiguousarray(np.stack([ri.real, ri.imag], axis=1))
        opts = _lib.MstmgOpts()
        self._L.mstmg_default_opts(ctypes.byref(opts))
        opts.precision = PRECISIONS[precision]
        opts.device = device
        opts.medium_re = float(np.real(medium_index))
        opts.medium_im = float(np.imag(medium_index))
        opts.inner_eps = inner_eps
        opts.max_outer = max_outer
        opts.generic_kernel = int(generic_kernel)
        opts.tile_ctas_per_sm = int(tile_ctas_per_sm)
        opts.fp32_chunk = int(fp32_chunk)
        opts.mixed_solver = int(mixed_solver)
        opts.gmres_restart = int(gmres_restart)
        opts.tensor_core = int(tensor_core)
        opts.tile_pairs = int(tile_pairs)
        self.ctx = ctypes.c_void_p()
        check(self._L.mstmg_ctx_create(ctypes.byref(self.ctx), n, _ptr(pos), _ptr(rad), _ptr(ri2), float(mie_epsilon),
                                       ctypes.byref(opts)), "mstmg_ctx_create")
        self.number_spheres = n
        self.positions, self.radii = pos, rad
        self.number_eqns = self._L.mstmg_neqns(self.ctx)
        self.sphere_order = np.zeros(n, np.int32)
        self.sphere_offset = np.zeros(n + 1, np.int32)
        check(self._L.mstmg_sphere_orders(self.ctx, _ptr(self.sphere_order), _ptr(self.sphere_offset)), "orders")
        self.precision = precision

    def sphereinteraction_ex(self, ain, con_tran=None, mie_mult=None, initial_run=False, rhs_list=None, fft_option=-1,
                             store_matrix_option=True, skip_external_translation=False):
        """sphereinteraction with rhs_list, fft_option (-1: as set up),
        store_matrix_option and skip_external_translation."""
        ain = np.asfortranarray(np.asarray(ain, np.complex128).reshape(self.number_eqns, -1, order="F"))
        nrhs = ain.shape[1]
        out = np.zeros((self.number_eqns, nrhs), np.complex128, order="F")
        ct = np.array(con_tran if con_tran is not None else [0] * nrhs, np.int32)
        mm = np.array(mie_mult if mie_mult is not None else [1] * nrhs, np.int32)
        rl = None if rhs_list is None else np.array(rhs_list, np.int32)
        check(self._L.mstmg_interaction_ex(self.ctx, nrhs, _ptr(ain), _ptr(out), _ptr(ct), _ptr(mm), int(initial_run),
                                           None if rl is None else _ptr(rl), int(fft_option), int(bool(store_matrix_option)),
                                           int(bool(skip_external_translation))), "sphereinteraction_ex")
        return out

    def cbicg(self, pnp, anp, niter=10000, eps=1.0e-6, initialize=True):
        pnp = np.ascontiguousarray(pnp, np.complex128)
        x = np.array(anp, np.complex128, copy=True)
        it = c_int(0)
        err = c_double(0.0)
        rc = check(self._L.mstmg_bicg(self.ctx, niter, eps, _ptr(pnp), _ptr(x), int(initialize), ctypes.byref(it),
                                      ctypes.byref(err)), "cbicg")
        return x, it.value, err.value

    def sphereplanewavecoef(self, alpha=0.0, sinc=0.0, direction=1):
        out = np.zeros((self.number_eqns, 2), np.complex128, order="F")
        check(self._L.mstmg_planewave(self.ctx, alpha, sinc, direction, _ptr(out)), "sphereplanewavecoef")
        return out

    def fixedorsoln(self, eps=1.0e-6, niter=10000, alpha=0.0, sinc=0.0, direction=1):
        """Returns dict(amnp, qeff (3,3,N), qtot (3,3), maxerr, maxiter, istat, iterations)."""
        amnp = np.zeros((self.number_eqns, 2), np.complex128, order="F")
        qeff = np.zeros((3, 3, self.number_spheres), np.float64, order="F")
        qtot = np.zeros((3, 3), np.float64, order="F")
        me = c_double(0.0)
        mi = c_int(0)
        st = check(self._L.mstmg_fixed_orientation(self.ctx, alpha, sinc, direction, eps, niter, _ptr(amnp), _ptr(qeff),
                                                   _ptr(qtot), ctypes.byref(me), ctypes.byref(mi)), "fixedorsoln")
        stats = self.last_stats()
        return dict(amnp=amnp, qeff=qeff, qtot=qtot, maxerr=me.value, maxiter=mi.value, istat=st, **stats)

    def set_pair_shard(self, shard, nshards):
        """Translate only the tiles t with t % nshards == shard (the pairs of one
        rank of a group; see mstm_b200.shard).  nshards = 1 restores all pairs."""
        check(self._L.mstmg_set_pair_shard(self.ctx, int(shard), int(nshards)), "set_pair_shard")

    def fixed_orientation_rhs(self, alpha=0.0, sinc=0.0, direction=1):
        """Right-hand sides Mie x plane wave of both polarisations (neqns x 2)."""
        out = np.zeros((self.number_eqns, 2), np.complex128, order="F")
        check(self._L.mstmg_fixed_orientation_rhs(self.ctx, alpha, sinc, direction, _ptr(out)), "fixed_orientation_rhs")
        return out

    def efficiencies(self, amnp, alpha=0.0, sinc=0.0, direction=1):
        """Efficiencies of a solution amnp (neqns x 2): dict(qeff (3,3,N), qtot (3,3))."""
        a = np.asfortranarray(amnp, np.complex128)
        qeff = np.zeros((3, 3, self.number_spheres), np.float64, order="F")
        qtot = np.zeros((3, 3), np.float64, order="F")
        check(self._L.mstmg_efficiencies(self.ctx, alpha, sinc, direction, _ptr(a), _ptr(qeff), _ptr(qtot)), "efficiencies")
        return dict(qeff=qeff, qtot=qtot)

    def scattering(self, amnp, trans_eps=1.0e-5, max_t_order=100, nangles=181):
        """Azimuth-averaged scattering matrix (nangles, 4, 4), asymmetry parameter
        g, t_matrix_order and the common-origin expansion amnp0 (2T(T+2), 2;
        TE/TM) of a fixed-orientation solution amnp (neqns, 2)."""
        amnp = np.asfortranarray(amnp, np.complex128)
        smat = np.zeros(16 * nangles)
        g, tmo = c_double(0.0), c_int(0)
        tcap = max(max_t_order, int(self.sphere_order.max()))
        cap = 2 * tcap * (tcap + 2)
        a0 = np.zeros((cap, 2), np.complex128, order="F")
        check(self._L.mstmg_scattering(self.ctx, _ptr(amnp), trans_eps, max_t_order, nangles, _ptr(smat), ctypes.byref(g),
                                       ctypes.byref(tmo), _ptr(a0), cap), "scattering")
        T = tmo.value
        nb0 = 2 * T * (T + 2)
        amnp0 = np.asfortranarray(a0.reshape(-1, order="F")[:2 * nb0].reshape(nb0, 2, order="F"))
        return dict(smat=smat.reshape(nangles, 4, 4).transpose(0, 2, 1).copy(), g=g.value, t_matrix_order=T, amnp0=amnp0)

    def translation_pass(self, x, con_tran=None, precision="fp64"):
        """y = H x, the pair translation pass alone (external_to_external_expansion,
        mstm-modules-33.f90:6390-6525) with the FP64 ("fp64") or FP32 ("fp32")
        operators, or ("tc") the tensor-core pass (dense TF32 hi/lo operators,
        plain columns only)."""
        x = np.asfortranarray(np.asarray(x, np.complex128).reshape(self.number_eqns, -1))
        ncols = x.shape[1]
        y = np.zeros_like(x, order="F")
        ct = None if con_tran is None else np.ascontiguousarray(np.asarray(con_tran, np.int32))
        prec = {"fp64": 0, "fp32": 1, "mixed": 1, "tc": 2}[precision]
        check(self._L.mstmg_translation_pass(self.ctx, prec, ncols, None if ct is None else _ptr(ct),
                                             _ptr(x), _ptr(y)), "translation_pass")
        return y

    def gsf_coefficients(self, amnp0, t_matrix_order):
        """fosmexpansion of a common-origin expansion: dict(s00, s02, sp22, sm22),
        each (2T+1, 4, 4) [w][i][j]."""
        T = int(t_matrix_order)
        W = 2 * T + 1
        a0 = np.asfortranarray(amnp0, np.complex128)
        coef = np.zeros(4 * 16 * W)
        check(self._L.mstmg_gsf_coefficients(self.ctx, T, _ptr(a0), _ptr(coef)), "gsf_coefficients")
        c = coef.reshape(4, W, 4, 4).transpose(0, 1, 3, 2)
        return dict(s00=c[0].copy(), s02=c[1].copy(), sp22=c[2].copy(), sm22=c[3].copy())

    def scattering_plane(self, amnp0, t_matrix_order, increment=1.0, alpha=0.0, rotate_plane=False):
        """Scattering matrix without azimuthal averaging (scatteringmatrix,
        mstm-scatprops-26.f90:1498-1573, normalize_s11 false) at the directions
        scattering_matrix_calculation uses when azimuthal_average is false:
        theta = -180..180 degrees in steps of 180/udim, udim =
        floor(180.00001/increment), in the plane of azimuth alpha (theta < 0
        on the far side).  Returns (theta (2udim+1,), smat (2udim+1, 4, 4))."""
        T = int(t_matrix_order)
        udim = int(np.floor(180.00001 / increment))
        ldim, amax = -udim, 180.0
        amin = -amax
        a0 = np.asfortranarray(amnp0, np.complex128)
        if a0.shape != (2 * T * (T + 2), 2):
            raise ValueError(f"amnp0 must be ({2 * T * (T + 2)}, 2), got {a0.shape}")
        n = udim - ldim + 1
        sm = np.zeros(16 * n)
        check(self._L.mstmg_scattering_plane(self.ctx, T, _ptr(a0), ldim, udim, amin, amax, alpha, int(bool(rotate_plane)),
                                             _ptr(sm)), "scattering_plane")
        theta = np.array([amin + (i - ldim) / (udim - ldim) * (amax - amin) for i in range(ldim, udim + 1)])
        return theta, sm.reshape(n, 4, 4).transpose(0, 2, 1).copy()

    def fft_setup(self, cell_volume_fraction=0.2, d_cell=0.0, node_order=-1, neighbor_node_model=2):
        """Use MSTM's FFT translation (fft_translation_option): near pairs direct,
        the rest through cell nodes and an FFT convolution.  Returns the grid
        chosen: dict(cell_dim, d_cell, node_order, near_pairs)."""
        cd = np.zeros(3, np.int32)
        dc, no, npair = c_double(0.0), c_int(0), c_int(0)
        check(self._L.mstmg_fft_setup(self.ctx, cell_volume_fraction, d_cell, node_order, neighbor_node_model, _ptr(cd),
                                      ctypes.byref(dc), ctypes.byref(no), ctypes.byref(npair)), "fft_setup")
        return dict(cell_dim=cd.tolist(), d_cell=dc.value, node_order=no.value, near_pairs=npair.value)

    def t_matrix_order(self, trans_eps=1.0e-5, max_t_order=100):
        """Order of the cluster T matrix about the cluster origin (tranordertest for
        every sphere, mstm-modules-33.f90:1896-1942); also fixes the per-sphere
        translation orders that tmatrix_solution uses."""
        t = c_int(0)
        check(self._L.mstmg_t_matrix_order(self.ctx, trans_eps, max_t_order, ctypes.byref(t)), "t_matrix_order")
        return t.value

    def tmatrix_solution(self, t_matrix_order=None, solution_eps=1.0e-6, convergence_eps=1.0e-6, max_iterations=10000,
                         trans_eps=1.0e-5, max_t_order=100):
        """tmatrix_solution (mstm-solver-8.f90:22-332): the cluster T matrix,
        (nblkt, nblkt) complex with nblkt = 2 T (T+2), column 2(l(l+1)+k-1)+q-1 for
        the unit TE (q=1) / TM (q=2) field of degree k and order l, rows
        2(n(n+1)+m-1)+p-1 (rows of order n > l are left zero, as the reference
        writes them); plus the per-sphere efficiencies summed over the columns
        (3, N), the orientation-averaged (Qext, Qabs, Qsca), the order kept
        (the loop stops once Qext changes by less than convergence_eps), and
        the largest iteration count and residual of the column solves."""
        if t_matrix_order is None:
            t_matrix_order = self.t_matrix_order(trans_eps, max_t_order)
        T = int(t_matrix_order)
        nb = 2 * T * (T + 2)
        tm = np.zeros((nb, nb), np.complex128, order="F")
        sq = np.zeros((3, self.number_spheres), np.float64, order="F")
        qt = np.zeros(3)
        used, mi, me = c_int(0), c_int(0), c_double(0.0)
        st = self._L.mstmg_tmatrix(self.ctx, T, solution_eps, convergence_eps, max_iterations, _ptr(tm), _ptr(sq), _ptr(qt),
                                   ctypes.byref(used), ctypes.byref(mi), ctypes.byref(me))
        if st < 0:
            check(st, "tmatrix")
        return dict(tmat=tm, t_matrix_order=T, order=used.value, sphere_qeff=sq, qtot=qt, istat=st, maxiter=mi.value,
                    maxerr=me.value, outer=self.last_stats()["outer"])

    def tmatrix_qext_qsca(self, tmat, t_matrix_order):
        """Orientation-averaged Qext, Qsca from the T matrix as the random-orientation
        reader forms them (mstm-scatprops-26.f90:2103-2122)."""
        tmat = np.asfortranarray(tmat, np.complex128)
        qe, qs = c_double(0.0), c_double(0.0)
        check(self._L.mstmg_tmatrix_qext_qsca(self.ctx, int(t_matrix_order), _ptr(tmat), ctypes.byref(qe), ctypes.byref(qs)),
              "tmatrix_qext_qsca")
        return qe.value, qs.value

    def ranorientscatmatrix(self, tmat, t_matrix_order, nangles=181):
        """Orientation-averaged scattering matrix from the T matrix: GSF expansion
        coefficients sm, smcf (2T+1, 4, 4) [w][i][j] (total and coherent part),
        the elements smat (nangles, 4, 4) at theta_i = i*pi/(nangles-1), and the
        coherent scattering ratio smcf[0,0,0]."""
        T = int(t_matrix_order)
        W = 2 * T + 1
        tmat = np.asfortranarray(tmat, np.complex128)
        sm = np.zeros(16 * W)
        cf = np.zeros(16 * W)
        smat = np.zeros(16 * max(nangles, 1))
        check(self._L.mstmg_ranorient_scattering(self.ctx, T, _ptr(tmat), nangles, _ptr(sm), _ptr(cf), _ptr(smat)),
              "ranorientscatmatrix")
        sm3 = sm.reshape(W, 4, 4).transpose(0, 2, 1).copy()
        cf3 = cf.reshape(W, 4, 4).transpose(0, 2, 1).copy()
        out = dict(sm=sm3, smcf=cf3, coherent=cf3[0, 0, 0])
        if nangles > 0:
            out["smat"] = smat.reshape(nangles, 4, 4).transpose(0, 2, 1).copy()
        return out

    def operator_bytes(self, precision="fp64"):
        s, c = c_double(0.0), c_double(0.0)
        check(self._L.mstmg_operator_bytes(self.ctx, PRECISIONS[precision], ctypes.byref(s), ctypes.byref(c)), "bytes")
        return s.value, c.value

    def time_translation(self, precision="fp64", nrhs=2, reps=10):
        """Milliseconds per translation pass: "fp64", "mixed" (FP32 rotation
        kernels) or "tc" (plain columns on the tensor cores)."""
        ms = c_double(0.0)
        prec = {"fp64": 0, "mixed": 1, "fp32": 1, "tc": 2}[precision]
        check(self._L.mstmg_time_translation(self.ctx, prec, nrhs, reps, ctypes.byref(ms)), "time")
        return ms.value


class SphereEnsemble(_Context):
    """Independent configurations solved together (mstmg_ensemble_create; no
    counterpart in MSTM, which solves one configuration per run).

    configs: list of (positions (N_c, 3), radii (N_c,), ref_index (N_c,) or
    scalar).  The context holds no pairs between configurations, and
    fixedorsoln() runs every configuration's two polarisations through the
    mixed GMRES together, one translation pass a step for the whole ensemble,
    each system to the reference's criterion on its own configuration.
    """

    def __init__(self, configs, mie_epsilon=1.0e-6, device=0, medium_index=1.0, gmres_restart=0, max_outer=30, inner_eps=1.0e-8,
                 tile_ctas_per_sm=0):
        self._L = _lib.lib()
        pos, rad, ri, start = [], [], [], [0]
        for p_, r_, m_ in configs:
            p_ = np.asarray(p_, np.float64).reshape(-1, 3)
            r_ = np.asarray(r_, np.float64).reshape(-1)
            m_ = np.asarray(m_, np.complex128)
            pos.append(p_)
            rad.append(r_)
            ri.append(np.full(len(r_), m_) if m_.ndim == 0 else m_.reshape(-1))
            start.append(start[-1] + len(r_))
        pos = np.ascontiguousarray(np.concatenate(pos))
        rad = np.ascontiguousarray(np.concatenate(rad))
        ri = np.concatenate(ri)
        ri2 = np.ascontiguousarray(np.stack([ri.real, ri.imag], axis=1))
        self.config_start = np.ascontiguousarray(start, np.int32)
        self.number_configs = len(configs)
        opts = _lib.MstmgOpts()
        self._L.mstmg_default_opts(ctypes.byref(opts))
        opts.precision = PRECISIONS["mixed"]
        opts.device = device
        opts.medium_re = float(np.real(medium_index))
        opts.medium_im = float(np.imag(medium_index))
        opts.gmres_restart = int(gmres_restart)
        opts.max_outer = max_outer
        opts.inner_eps = inner_eps
        opts.tile_ctas_per_sm = int(tile_ctas_per_sm)
        self.ctx = ctypes.c_void_p()
        check(self._L.mstmg_ensemble_create(ctypes.byref(self.ctx), self.number_configs, _ptr(self.config_start), len(rad), _ptr(pos),
                                            _ptr(rad), _ptr(ri2), float(mie_epsilon), ctypes.byref(opts)), "mstmg_ensemble_create")
        self.number_spheres = len(rad)
        self.number_eqns = self._L.mstmg_neqns(self.ctx)
        self.sphere_order = np.zeros(len(rad), np.int32)
        self.sphere_offset = np.zeros(len(rad) + 1, np.int32)
        check(self._L.mstmg_sphere_orders(self.ctx, _ptr(self.sphere_order), _ptr(self.sphere_offset)), "orders")

    def fixedorsoln(self, eps=1.0e-6, niter=10000, alpha=0.0, sinc=0.0, direction=1):
        """Returns dict(amnp (neqns, 2), qeff (3, 3, N), qtot (nconfig, 3, 3),
        iterations (nconfig, 2) in Arnoldi-step pairs, errors (nconfig, 2),
        istat, and amnp_of(c): configuration c's rows of amnp)."""
        nc = self.number_configs
        amnp = np.zeros((self.number_eqns, 2), np.complex128, order="F")
        qeff = np.zeros((3, 3, self.number_spheres), np.float64, order="F")
        qtot = np.zeros((3, 3, nc), np.float64, order="F")
        its = np.zeros(2 * nc, np.int32)
        errs = np.zeros(2 * nc, np.float64)
        st = check(self._L.mstmg_ensemble_fixed_orientation(self.ctx, alpha, sinc, direction, eps, niter, _ptr(amnp), _ptr(qeff), _ptr(qtot),
                                                            _ptr(its), _ptr(errs)), "ensemble fixedorsoln")
        off = self.sphere_offset
        start = self.config_start
        return dict(amnp=amnp, qeff=qeff, qtot=np.moveaxis(qtot, 2, 0).copy(), iterations=its.reshape(nc, 2), errors=errs.reshape(nc, 2),
                    istat=st, amnp_of=lambda c: amnp[off[start[c]]:off[start[c + 1]]])


def qtotcalc(qeff, radii, vol_radius):
    """qtotcalc (mstm-scatprops-26.f90:872-912) for external spheres: area-weighted
    totals with Qsca = Qext + Qinc - Qabs.  qeff: (3,3,N)."""
    q = np.einsum("kpi,i->kp", qeff, np.asarray(radii) ** 2) / vol_radius ** 2
    q = q.copy()
    q[2, :] = q[0, :] + q[2, :] - q[1, :]
    return q
