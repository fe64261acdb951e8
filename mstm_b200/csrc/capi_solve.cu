// capi_solve.cu -- the solvers behind the C ABI: cbicg (batched BiCG, FP64),
// fixedorsoln and its mixed-precision forms, ensembles, and the many-system
// solvers the T matrix uses (BiCG, FP32 residual replacement, FP32 BiCG in
// FP64 refinement, restarted GMRES with FP64 true residuals).
#include "ctx.cuh"

// The incident plane wave at every sphere the wave reaches (sphereplanewavecoef,
// scatprops:262-281): all spheres, or those outside every other sphere
static void planewave_ctx(mstmg_ctx* c, double alpha, double sinc, int dir)
{
    launch_planewave(alpha, sinc, dir, c->lmax, c->neqns, c->slot_full.p, c->d_order.p, c->d_offset.p, c->pos.p, c->pw0.p, c->drot.p,
                     c->pmnp.p, c->st, c->n, c->hs.on() ? c->hs.d_outside.p : nullptr);
}

// qefficiencyfactors + qtotcalc of the solution amnp (device, 2 columns) for
// the incident field in c->pmnp (scatprops:782-912).  With host spheres the
// exciting fields are the interaction without the Mie multiply plus the
// incident field, in Y64's first two columns.
static int qeff_ctx(mstmg_ctx* c, const zd* amnp)
{
    const int ne = c->neqns;
    const zd* g = nullptr;
    if (c->hs.on()) {
        int rc = ensure_ops(c, 0, false);
        if (rc) return rc;
        rc = translate<double>(c, amnp, c->Y64.p, 2, 0u);
        if (rc) return rc;
        launch_add_correction_d(2 * ne, c->Y64.p, c->pmnp.p, c->st);
        g = c->Y64.p;
    }
    launch_qeff(c->n, c->d_order.p, c->d_offset.p, c->d_mie_offset.p, c->rad.p, mk(c->opts.medium_re, c->opts.medium_im), c->an_inv.p,
                amnp, c->pmnp.p, ne, c->qeff.p, c->xg, c->qtot.p, c->st, c->hs.on() ? c->hs.d_rext.p : nullptr, g,
                c->hs.on() ? c->hs.d_host.p : nullptr, c->hs.on() ? c->hs.qv.p : nullptr, c->hs.d_hstart.p, c->hs.d_held.p);
    CK(cudaGetLastError());
    return MSTMG_OK;
}

// ---------------------------------------------------------------------------
// Batched BiCG: S independent systems advance in lockstep, sharing one
// translation pass per iteration ([p_1, w_1, p_2, w_2, ...], the w columns as
// conjugate-transpose products).  With S = 1 this is cbicg's single-rank
// iteration (mstm-solver-8.f90:828-947) step for step.
//   have_x0: the initial residual is b - A x0 (one extra pass); otherwise x0 = 0.
// ---------------------------------------------------------------------------
template <typename T>
int bicg_batched(mstmg_ctx* c, int S, const cpx<T>* const* b, BicgVecs<T>* v, bool have_x0, int niter, const double* eps,
                        int* iters, double* errs, int* status)
{
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    const cpx<T>* an = nullptr;
    if (sizeof(T) == 8) an = (const cpx<T>*)c->an.p;
    else an = (const cpx<T>*)c->an32.p;
    cpx<T>* X = (sizeof(T) == 8) ? (cpx<T>*)c->X64.p : (cpx<T>*)c->X32.p;
    cpx<T>* Y = (sizeof(T) == 8) ? (cpx<T>*)c->Y64.p : (cpx<T>*)c->Y32.p;
    double* part = c->part.p;
    const int partstride = 3 * c->nsm * 4 / 1;
    (void)partstride;
    bool active[4];
    int rc;
    // initial residuals
    if (have_x0) {
        for (int s = 0; s < S; s++) CK(cudaMemcpyAsync(X + (size_t)s * ne, v[s].x, sizeof(cpx<T>) * ne, cudaMemcpyDeviceToDevice, c->st));
        rc = translate<T>(c, X, Y, S, 0u);
        if (rc) return rc;
    }
    // host spheres: the Mie multiply runs apart (mie_all), the fused kernels take y as M y
    const bool hosts = sizeof(T) == 8 && c->hs.on();
    const cpx<T>* anf = hosts ? nullptr : an;
    for (int s = 0; s < S; s++) {
        if (!have_x0) CK(cudaMemsetAsync(v[s].x, 0, sizeof(cpx<T>) * ne, c->st));
        if (hosts && have_x0) mie_all(c, 1, 0, (const zd*)(Y + (size_t)s * ne), (zd*)(Y + (size_t)s * ne));
        launch_init<T>(sm, anf, b[s], v[s].x, Y + (size_t)s * ne, have_x0 ? 1 : 0, v[s].r, v[s].p, v[s].w, v[s].q, part, c->sc.p + s, 1,
                       c->nsm, c->st);
    }
    CK(cudaMemcpyAsync(c->h_sc, c->sc.p, sizeof(BicgScalars) * S, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int s = 0; s < S; s++) {
        iters[s] = 0;
        errs[s] = 0.0;
        status[s] = 0;
        active[s] = !c->h_sc[s].stop;
    }
    int nact = 0;
    for (int s = 0; s < S; s++) nact += active[s];
    for (int it = 1; it <= niter && nact > 0; it++) {
        int slots[4], a = 0;
        for (int s = 0; s < S; s++)
            if (active[s]) slots[a++] = s;
        unsigned mask = 0;
        for (int k = 0; k < a; k++) {
            int s = slots[k];
            CK(cudaMemcpyAsync(X + (size_t)(2 * k) * ne, v[s].p, sizeof(cpx<T>) * ne, cudaMemcpyDeviceToDevice, c->st));
            if (hosts) mie_all(c, -1, 1, (const zd*)v[s].w, (zd*)(X + (size_t)(2 * k + 1) * ne));
            else launch_mie<T>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, an, -1, 1, v[s].w, X + (size_t)(2 * k + 1) * ne, c->st);
            mask |= 2u << (2 * k);
        }
        rc = translate<T>(c, X, Y, 2 * a, mask);
        if (rc) return rc;
        for (int k = 0; k < a; k++) {
            int s = slots[k];
            if (hosts) mie_all(c, 1, 0, (const zd*)(Y + (size_t)(2 * k) * ne), (zd*)(Y + (size_t)(2 * k) * ne));
            launch_post<T>(sm, anf, v[s].p, v[s].w, Y + (size_t)(2 * k) * ne, Y + (size_t)(2 * k + 1) * ne, v[s].cap, v[s].caw, part,
                           c->sc.p + s, c->nsm, c->st);
            launch_upd<T>(ne, v[s].x, v[s].r, v[s].q, v[s].p, v[s].w, v[s].cap, v[s].caw, part, c->sc.p + s, eps[s], c->nsm, c->st);
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(c->h_sc, c->sc.p, sizeof(BicgScalars) * S, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        for (int k = 0; k < a; k++) {
            int s = slots[k];
            iters[s] = it;
            errs[s] = c->h_sc[s].eerr;
            if (c->h_sc[s].breakdown) {
                active[s] = false;
                status[s] = 2;
            } else if (c->h_sc[s].stop) {
                active[s] = false;
            }
        }
        nact = 0;
        for (int s = 0; s < S; s++) nact += active[s];
    }
    for (int s = 0; s < S; s++)
        if (active[s]) iters[s] = niter + 1;   // Fortran DO-loop exit value when the cap is reached
    return check_kernel_err(c);
}

template <typename T> static BicgVecs<T> vecs_at(cpx<T>* base, int ne, int s)
{
    cpx<T>* b = base + (size_t)s * 7 * ne;
    BicgVecs<T> v;
    v.x = b;
    v.r = b + ne;
    v.p = b + 2 * ne;
    v.w = b + 3 * ne;
    v.q = b + 4 * ne;
    v.cap = b + 5 * ne;
    v.caw = b + 6 * ne;
    return v;
}

// cbicg with niter < 0: the order-of-scattering iteration (mstm-solver-8.f90:787-822),
// x += M H p, p = M H p, until ||M H p||^2 / ||b||^2 < eps or -niter steps.
// *err keeps the reference's value: the error at the exit, 0 when the count ran out.
int oos_solve(mstmg_ctx* c, const zd* b, zd* x, int niter, double eps, int* iter, double* err)
{
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    zd* cp = c->X64.p + 2 * (size_t)ne;
    zd* cr = c->Y64.p + 2 * (size_t)ne;
    launch_rr_dot_norm(ne, b, c->part.p, c->small.p, c->nsm, c->st);
    CK(cudaMemcpyAsync(c->h_small, c->small.p, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const double enorm = c->h_small[0];
    CK(cudaMemcpyAsync(cp, x, sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
    int it;
    double emax = 0.0;
    for (it = 1; it <= -niter; it++) {
        int rc = translate<double>(c, cp, c->Y64.p, 1, 0u);
        if (rc) return rc;
        mie_all(c, 1, 0, c->Y64.p, cr);
        launch_add_correction_d(ne, x, cr, c->st);
        CK(cudaMemcpyAsync(cp, cr, sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
        launch_rr_dot_norm(ne, cr, c->part.p, c->small.p, c->nsm, c->st);
        CK(cudaMemcpyAsync(c->h_small, c->small.p, sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        double eerr = enorm > 0.0 ? c->h_small[0] / enorm : 0.0;
        if (eerr < eps) {
            emax = eerr;
            break;
        }
    }
    *iter = it;
    *err = emax;
    return check_kernel_err(c);
}

extern "C" int mstmg_bicg(mstmg_ctx* c, int niter, double eps, const double* pnp, double* anp, int initialize, int* iter, double* err)
{
    NvtxRange nvtx_("mstmg_bicg");
    if (!c || !pnp || !anp) return MSTMG_ERR_ARG;
    if (int rc0 = reject_ensemble(c, "mstmg_bicg")) return rc0;
    if (int rc1 = reject_sharded(c, "mstmg_bicg")) return rc1;
    int rc = ensure_ops(c, 0, initialize != 0);
    if (rc) return rc;
    const int ne = c->neqns;
    BicgVecs<double> v = vecs_at<double>(c->vec64.p, ne, 0);
    CK(copy_in(c->bvec64.p, pnp, sizeof(zd) * ne, c->st));
    CK(copy_in(v.x, anp, sizeof(zd) * ne, c->st));
    const zd* bb[1] = {c->bvec64.p};
    int it = 0, st = 0;
    double e = 0.0;
    if (niter == 0) {
        set_err("mstmg_bicg: niter = 0 (the reference's Mie-multiply-only mode) is not on this path");
        return MSTMG_ERR_UNSUPPORTED;
    }
    // a zero right-hand side returns at once, anp untouched (cbicg, solver:694)
    launch_rr_dot_norm(ne, c->bvec64.p, c->part.p, c->small.p, c->nsm, c->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_small, c->small.p, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (c->h_small[0] == 0.0) {
        if (iter) *iter = 0;
        if (err) *err = 0.0;
        return MSTMG_OK;
    }
    if (niter < 0) rc = oos_solve(c, c->bvec64.p, v.x, niter, eps, &it, &e);
    else rc = bicg_batched<double>(c, 1, bb, &v, true, niter, &eps, &it, &e, &st);
    if (rc) return rc;
    CK(copy_out(anp, v.x, sizeof(zd) * ne, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (iter) *iter = it;
    if (err) *err = e;
    return st == 2 ? MSTMG_ERR_BREAKDOWN : MSTMG_OK;
}

extern "C" int mstmg_planewave(mstmg_ctx* c, double alpha, double sinc, int dir, double* pmnp)
{
    if (!c || !pmnp) return MSTMG_ERR_ARG;
    planewave_ctx(c, alpha, sinc, dir);
    CK(cudaGetLastError());
    CK(copy_out(pmnp, c->pmnp.p, sizeof(zd) * 2 * (size_t)c->neqns, c->st));
    CK(cudaStreamSynchronize(c->st));
    return MSTMG_OK;
}

// Mixed precision: FP64 outer refinement around FP32 inner BiCG, both
// polarisations at once.  x (FP64, 2 systems) starts at the Mie solution.
int solve_mixed(mstmg_ctx* c, zd* const* b, zd* const* x, double eps, int niter, int* iters, double* errs, int* status)
{
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    int rc = ensure_ops(c, 0, false);
    if (rc) return rc;
    rc = ensure_ops(c, 1, false);
    if (rc) return rc;
    int S = 2;
    double err[2] = {1.0, 1.0};
    bool act[2] = {true, true};
    int total_it[2] = {0, 0};
    c->outer = 0;
    for (int s = 0; s < S; s++) status[s] = 0;
    for (int outer = 0; outer < c->opts.max_outer; outer++) {
        // FP64 true residual r = b - x + M H x for the active systems
        int slots[2], a = 0;
        for (int s = 0; s < S; s++)
            if (act[s]) slots[a++] = s;
        if (a == 0) break;
        for (int k = 0; k < a; k++)
            CK(cudaMemcpyAsync(c->X64.p + (size_t)k * ne, x[slots[k]], sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
        rc = translate<double>(c, c->X64.p, c->Y64.p, a, 0u);
        if (rc) return rc;
        for (int k = 0; k < a; k++) {
            int s = slots[k];
            launch_resid<double, float>(sm, c->an.p, b[s], x[s], c->Y64.p + (size_t)k * ne, c->rvec32.p + (size_t)s * ne, c->part.p,
                                        c->small.p + 2 * s, c->nsm, c->st);
        }
        CK(cudaMemcpyAsync(c->h_small, c->small.p, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        c->outer = outer + 1;
        int na = 0;
        double inner_eps[2];
        for (int k = 0; k < a; k++) {
            int s = slots[k];
            double rr = c->h_small[2 * s], bb = c->h_small[2 * s + 1];
            err[s] = (bb > 0.0) ? rr / bb : 0.0;
            if (err[s] < eps || total_it[s] >= niter) act[s] = false;
            else {
                na++;
                double target = eps / err[s] * 0.01;
                inner_eps[s] = std::max(target, c->opts.inner_eps);
            }
        }
        if (na == 0) break;
        // inner FP32 solves for the active systems, batched
        int S2 = 0, map[2];
        const zf* bb32[2];
        BicgVecs<float> vv[2];
        double ie[2];
        for (int s = 0; s < S; s++)
            if (act[s]) {
                map[S2] = s;
                bb32[S2] = c->rvec32.p + (size_t)s * ne;
                vv[S2] = vecs_at<float>(c->vec32.p, ne, S2);
                ie[S2] = inner_eps[s];
                S2++;
            }
        int it2[2] = {0, 0}, st2[2] = {0, 0};
        double e2[2];
        int cap = niter;
        for (int k = 0; k < S2; k++) cap = std::min(cap, niter - total_it[map[k]]);
        if (cap < 1) cap = 1;
        rc = bicg_batched<float>(c, S2, bb32, vv, false, cap, ie, it2, e2, st2);
        if (rc) return rc;
        for (int k = 0; k < S2; k++) {
            int s = map[k];
            total_it[s] += std::min(it2[k], cap);
            launch_add_correction_f(ne, x[s], vv[k].x, c->st);
            if (st2[k] == 2) status[s] = 2;
        }
        CK(cudaGetLastError());
    }
    for (int s = 0; s < S; s++) {
        iters[s] = total_it[s];
        errs[s] = err[s];
    }
    return MSTMG_OK;
}

// systems of an ensemble: segment offsets and lengths per system (device),
// vectors of ldv elements in the GMRES work


static int fixed_orientation_impl(mstmg_ctx* c, double alpha, double sinc, int dir, double eps, int niter, const double* x0, double fallback,
                                  int* used_guess, double* guess_res, double* amnp, double* qeff, double* qtot, double* maxerr, int* maxiter);

extern "C" int mstmg_fixed_orientation(mstmg_ctx* c, double alpha, double sinc, int dir, double eps, int niter, double* amnp,
                                       double* qeff, double* qtot, double* maxerr, int* maxiter)
{
    NvtxRange nvtx_("mstmg_fixed_orientation");
    return fixed_orientation_impl(c, alpha, sinc, dir, eps, niter, nullptr, 0.0, nullptr, nullptr, amnp, qeff, qtot, maxerr, maxiter);
}

extern "C" int mstmg_fixed_orientation_guess(mstmg_ctx* c, double alpha, double sinc, int dir, double eps, int niter, const double* x0,
                                             double fallback_residual, int* used_guess, double* guess_residual, double* amnp, double* qeff,
                                             double* qtot, double* maxerr, int* maxiter)
{
    if (!x0) {
        set_err("mstmg_fixed_orientation_guess: x0 required");
        return MSTMG_ERR_ARG;
    }
    return fixed_orientation_impl(c, alpha, sinc, dir, eps, niter, x0, fallback_residual, used_guess, guess_residual, amnp, qeff, qtot,
                                  maxerr, maxiter);
}

static int fixed_orientation_impl(mstmg_ctx* c, double alpha, double sinc, int dir, double eps, int niter, const double* x0, double fallback,
                                  int* used_guess, double* guess_res, double* amnp, double* qeff, double* qtot, double* maxerr, int* maxiter)
{
    if (!c || !amnp) return MSTMG_ERR_ARG;
    if (int rc0 = reject_ensemble(c, "mstmg_fixed_orientation")) return rc0;
    if (int rc1 = reject_sharded(c, "mstmg_fixed_orientation")) return rc1;
    if (c->hs.on() && (x0 || (niter > 0 && c->opts.precision == MSTMG_PRECISION_MIXED && c->opts.mixed_solver != 2))) {
        set_err("mstmg_fixed_orientation: with spheres inside other spheres the solve is the FP64 BiCG or the mixed GMRES "
                "(mixed_solver 2), without an initial guess");
        return MSTMG_ERR_UNSUPPORTED;
    }
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    c->passes64 = c->passes32 = 0;
    c->outer = 0;
    // operators are (re)generated for this configuration: the reference's initial_run
    int rc = ensure_ops_both(c, true, c->opts.precision == MSTMG_PRECISION_MIXED, true);
    if (rc) return rc;
    planewave_ctx(c, alpha, sinc, dir);
    zd* bvec = c->bvec64.p;   // pmnpan for both polarisations: 2 x ne
    for (int p = 0; p < 2; p++)
        mie_all(c, 1, 0, c->pmnp.p + (size_t)p * ne, bvec + (size_t)p * ne);
    CK(cudaGetLastError());
    int istat = 0;
    int it[2] = {0, 0}, st[2] = {0, 0};
    double er[2] = {0.0, 0.0};
    // initial guesses: MSTM's Mie solution (solver:482-483), or the caller's
    // guess where its FP64 relative residual is at most `fallback`
    zd* xinit = bvec;
    if (x0) {
        zd* g = c->X64.p + 2 * (size_t)ne;   // columns 2, 3 of the work block
        CK(copy_in(g, x0, sizeof(zd) * 2 * (size_t)ne, c->st));
        CK(cudaMemcpyAsync(c->X64.p, g, sizeof(zd) * 2 * (size_t)ne, cudaMemcpyDeviceToDevice, c->st));
        rc = translate<double>(c, c->X64.p, c->Y64.p, 2, 0u);
        if (rc) return rc;
        for (int p = 0; p < 2; p++)
            launch_resid<double, double>(sm, c->an.p, bvec + (size_t)p * ne, g + (size_t)p * ne, c->Y64.p + (size_t)p * ne,
                                         c->Y64.p + (size_t)(2 + p) * ne, c->part.p, c->small.p + 2 * p, c->nsm, c->st);
        CK(cudaMemcpyAsync(c->h_small, c->small.p, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        for (int p = 0; p < 2; p++) {
            double rr = c->h_small[2 * p], bb = c->h_small[2 * p + 1];
            double res = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
            bool use = res <= fallback;
            if (guess_res) guess_res[p] = res;
            if (used_guess) used_guess[p] = use ? 1 : 0;
            if (!use) CK(cudaMemcpyAsync(g + (size_t)p * ne, bvec + (size_t)p * ne, sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
        }
        // the BiCG work below reuses X64/Y64; keep the guesses in the amnp buffer
        CK(cudaMemcpyAsync(c->amnp.p, g, sizeof(zd) * 2 * (size_t)ne, cudaMemcpyDeviceToDevice, c->st));
        xinit = c->amnp.p;
    }
    if (niter < 0) {
        for (int p = 0; p < 2; p++) {
            if (xinit != c->amnp.p)
                CK(cudaMemcpyAsync(c->amnp.p + (size_t)p * ne, xinit + (size_t)p * ne, sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
            rc = oos_solve(c, bvec + (size_t)p * ne, c->amnp.p + (size_t)p * ne, niter, eps, &it[p], &er[p]);
            if (rc) return rc;
        }
    } else if (niter == 0) {
        if (xinit != c->amnp.p)
            for (int p = 0; p < 2; p++)
                CK(cudaMemcpyAsync(c->amnp.p + (size_t)p * ne, bvec + (size_t)p * ne, sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
        if (c->hs.on()) {
            // the couplings through the host spheres alone, applied twice
            // (solver:509-518): x += (M H_host) x + (M H_host)^2 x
            CK(cudaMemcpyAsync(c->X64.p, c->amnp.p, sizeof(zd) * 2 * (size_t)ne, cudaMemcpyDeviceToDevice, c->st));
            for (int k = 0; k < 2; k++) {
                CK(cudaMemsetAsync(c->Y64.p, 0, sizeof(zd) * 2 * (size_t)ne, c->st));
                rc = translate_hosts(c, c->X64.p, c->Y64.p, 2, 0u);
                if (rc) return rc;
                mie_all(c, 1, 0, c->Y64.p, c->X64.p);
                mie_all(c, 1, 0, c->Y64.p + ne, c->X64.p + ne);
            }
            launch_add_correction_d(2 * ne, c->amnp.p, c->X64.p, c->st);
        }
    } else if (c->opts.precision == MSTMG_PRECISION_MIXED) {
        zd* xs[2] = {c->amnp.p, c->amnp.p + ne};
        zd* bs[2] = {bvec, bvec + ne};
        if (xinit != c->amnp.p)
            for (int p = 0; p < 2; p++) CK(cudaMemcpyAsync(xs[p], bs[p], sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
        if (c->opts.mixed_solver == 1) {
            rc = solve_mixed(c, bs, xs, eps, niter, it, er, st);
        } else if (c->opts.mixed_solver == 2) {
            // both polarisations as two systems of the restarted GMRES
            if (!c->fo_gm_ready) {
                if ((rc = c->fo64.init(2, ne, c->nsm, false)) || (rc = c->fo_gm.setup(2, ne, c->opts.gmres_restart, "mstmg_fixed_orientation")))
                    return rc;
                c->fo_gm_ready = true;
            }
            std::vector<int> its, sts;
            std::vector<double> ers;
            int oc = 0;
            rc = solve_multi_gmres(c, c->fo64, c->fo_gm, 2, bvec, c->amnp.p, eps, niter, its, ers, sts, &oc);
            c->outer = oc;
            for (int p = 0; p < 2; p++) {
                it[p] = its[p];
                er[p] = ers[p];
                st[p] = sts[p];
            }
        } else {
            // both polarisations as two systems of the many-system residual-replacement solver
            if (!c->fo_ready) {
                if ((rc = c->fo64.init(2, ne, c->nsm, false)) || (rc = c->fo32.init(2, ne, c->nsm, true))) return rc;
                CK(c->fo_rr.alloc(4));
                CK(c->fo_idx.alloc(4));
                c->fo_ready = true;
            }
            std::vector<int> its, sts;
            std::vector<double> ers;
            int oc = 0;
            rc = solve_multi_rr(c, c->fo64, c->fo32, c->fo_rr, c->fo_idx, 2, bvec, c->amnp.p, eps, niter, its, ers, sts, &oc);
            c->outer = oc;
            for (int p = 0; p < 2; p++) {
                it[p] = its[p];
                er[p] = ers[p];
                st[p] = sts[p];
            }
        }
        if (rc) return rc;
    } else {
        // the reference's order: polarisation 1 then 2, each from x0 = Mie*f
        for (int p = 0; p < 2; p++) {
            BicgVecs<double> v = vecs_at<double>(c->vec64.p, ne, 0);
            CK(cudaMemcpyAsync(v.x, xinit + (size_t)p * ne, sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
            const zd* bb[1] = {bvec + (size_t)p * ne};
            rc = bicg_batched<double>(c, 1, bb, &v, true, niter, &eps, &it[p], &er[p], &st[p]);
            if (rc) return rc;
            CK(cudaMemcpyAsync(c->amnp.p + (size_t)p * ne, v.x, sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
        }
    }
    // fixedorsoln resets maxiter/maxerr per polarisation, so the second one is reported
    int mi = it[1];
    double me = er[1];
    if (mi > niter || me > eps) istat = 1;
    if (st[0] == 2 || st[1] == 2) istat = 1;
    c->iters[0] = it[0];
    c->iters[1] = it[1];
    rc = qeff_ctx(c, c->amnp.p);
    if (rc) return rc;
    CK(copy_out(amnp, c->amnp.p, sizeof(zd) * 2 * (size_t)ne, c->st));
    if (qeff) CK(copy_out(qeff, c->qeff.p, sizeof(double) * 9 * (size_t)c->n, c->st));
    if (qtot) CK(copy_out(qtot, c->qtot.p, sizeof(double) * 9, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (maxerr) *maxerr = me;
    if (maxiter) *maxiter = mi;
    rc = check_kernel_err(c);
    if (rc) return rc;
    return istat;
}

// Fixed-orientation solves of every configuration of an ensemble at once:
// per configuration and polarisation the mixed GMRES of fixedorsoln's system
// (solver:350-569; x0 = Mie f, the reference's criterion per system), all
// systems advancing together so that one translation pass a step serves the
// whole ensemble.
extern "C" int mstmg_ensemble_fixed_orientation(mstmg_ctx* c, double alpha, double sinc, int dir, double eps, int niter, double* amnp,
                                                double* qeff, double* qtot, int* iterations, double* errors)
{
    NvtxRange nvtx_("mstmg_ensemble_fixed_orientation");
    if (!c || c->cfg_start.empty()) {
        set_err("mstmg_ensemble_fixed_orientation: not an ensemble context (mstmg_ensemble_create)");
        return MSTMG_ERR_ARG;
    }
    if (!amnp || niter < 1 || !(eps > 0.0)) {
        set_err("mstmg_ensemble_fixed_orientation: bad arguments (amnp required, niter >= 1, eps > 0)");
        return MSTMG_ERR_ARG;
    }
    if (c->opts.precision != MSTMG_PRECISION_MIXED || c->opts.mixed_solver != 2) {
        set_err("mstmg_ensemble_fixed_orientation: ensembles are solved by the mixed GMRES (precision mixed, mixed_solver 2)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    const int ne = c->neqns, nc = (int)c->cfg_start.size() - 1, S = 2 * nc;
    SlotMaps sm = c->sm();
    c->passes64 = c->passes32 = 0;
    c->outer = 0;
    int rc = ensure_ops_both(c, true, true, true);
    if (rc) return rc;
    planewave_ctx(c, alpha, sinc, dir);
    zd* bvec = c->bvec64.p;
    for (int p = 0; p < 2; p++)
        mie_all(c, 1, 0, c->pmnp.p + (size_t)p * ne, bvec + (size_t)p * ne);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->amnp.p, bvec, sizeof(zd) * 2 * (size_t)ne, cudaMemcpyDeviceToDevice, c->st));
    if (!c->ens_gm.hh && (rc = c->ens_gm.setup(S, c->ens_ldv, c->opts.gmres_restart, "mstmg_ensemble_fixed_orientation"))) return rc;
    const EnsSeg seg{c->ens_off.p, c->ens_len.p, c->ens_ldv};
    std::vector<int> its, sts;
    std::vector<double> ers;
    int oc = 0;
    rc = solve_multi_gmres(c, c->fo64, c->ens_gm, S, bvec, c->amnp.p, eps, niter, its, ers, sts, &oc, &seg);
    if (rc) return rc;
    c->outer = oc;
    launch_qeff(c->n, c->d_order.p, c->d_offset.p, c->d_mie_offset.p, c->rad.p, mk(c->opts.medium_re, c->opts.medium_im), c->an_inv.p,
                c->amnp.p, c->pmnp.p, ne, c->qeff.p, c->xg, c->qtot.p, c->st);
    launch_qtot_configs(nc, c->d_cfg_start.p, c->rad.p, c->qeff.p, c->d_cfg_xg.p, c->cfg_qtot.p, c->st);
    CK(cudaGetLastError());
    CK(copy_out(amnp, c->amnp.p, sizeof(zd) * 2 * (size_t)ne, c->st));
    if (qeff) CK(copy_out(qeff, c->qeff.p, sizeof(double) * 9 * (size_t)c->n, c->st));
    if (qtot) CK(copy_out(qtot, c->cfg_qtot.p, sizeof(double) * 9 * (size_t)nc, c->st));
    CK(cudaStreamSynchronize(c->st));
    int istat = 0;
    for (int s = 0; s < S; s++) {
        if (iterations) iterations[s] = its[s];
        if (errors) errors[s] = ers[s];
        if (its[s] > niter || ers[s] > eps || sts[s] == 2) istat = 1;
    }
    c->iters[0] = its[0];
    c->iters[1] = its[1];
    rc = check_kernel_err(c);
    if (rc) return rc;
    return istat;
}

// The fixed-orientation system's right-hand sides, Mie x plane wave of both
// polarisations (fixedorsoln's pmnpan, mstm-solver-8.f90:465-483), for a
// caller that drives the iteration itself.
extern "C" int mstmg_fixed_orientation_rhs(mstmg_ctx* c, double alpha, double sinc, int dir, double* pmnpan)
{
    if (!c || !pmnpan) return MSTMG_ERR_ARG;
    if (int rc0 = reject_ensemble(c, "mstmg_fixed_orientation_rhs")) return rc0;
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    planewave_ctx(c, alpha, sinc, dir);
    for (int p = 0; p < 2; p++)
        mie_all(c, 1, 0, c->pmnp.p + (size_t)p * ne, c->bvec64.p + (size_t)p * ne);
    CK(cudaGetLastError());
    CK(copy_out(pmnpan, c->bvec64.p, sizeof(zd) * 2 * (size_t)ne, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_kernel_err(c);
}

// Efficiencies of a given fixed-orientation solution (qefficiencyfactors and
// qtotcalc, as mstmg_fixed_orientation reports them).
extern "C" int mstmg_efficiencies(mstmg_ctx* c, double alpha, double sinc, int dir, const double* amnp, double* qeff, double* qtot)
{
    if (!c || !amnp) return MSTMG_ERR_ARG;
    if (int rc0 = reject_ensemble(c, "mstmg_efficiencies")) return rc0;
    const int ne = c->neqns;
    planewave_ctx(c, alpha, sinc, dir);
    CK(copy_in(c->amnp.p, amnp, sizeof(zd) * 2 * (size_t)ne, c->st));
    if (int rq = qeff_ctx(c, c->amnp.p)) return rq;
    if (qeff) CK(copy_out(qeff, c->qeff.p, sizeof(double) * 9 * (size_t)c->n, c->st));
    if (qtot) CK(copy_out(qtot, c->qtot.p, sizeof(double) * 9, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_kernel_err(c);
}

extern "C" int mstmg_last_host_syncs(const mstmg_ctx* c) { return c ? c->host_syncs : -1; }

extern "C" int mstmg_last_stats(const mstmg_ctx* c, int* iters2, int* outer, int* passes64, int* passes32)
{
    if (!c) return MSTMG_ERR_ARG;
    if (iters2) { iters2[0] = c->iters[0]; iters2[1] = c->iters[1]; }
    if (outer) *outer = c->outer;
    if (passes64) *passes64 = c->passes64;
    if (passes32) *passes32 = c->passes32;
    return MSTMG_OK;
}

static int atcdim_h(int ntot, int ltot)
{
    int nmin = std::min(ntot, ltot), nmax = std::max(ntot, ltot);
    return 2 * (nmin * (1 - nmin * nmin + 3 * nmax * (2 + nmin))) / 3;
}

extern "C" int mstmg_operator_bytes(const mstmg_ctx* c, int prec, double* stored, double* canonical)
{
    if (!c) return MSTMG_ERR_ARG;
    double es = prec == 0 ? 8.0 : 4.0;
    // with host spheres the stored records include the regular translations
    // between hosts and the spheres they hold (FP64 only)
    const double hb = c->hs.on() ? (double)c->hs.hunits * 8.0 : 0.0;
    if (stored) *stored = ((prec != 0 && c->row32) ? (double)c->npairs * c->row32 * es : (double)c->op_units * es) + hb;
    if (canonical) {
        auto canon = [&](int a, int b) {
            int nmn = std::min(a, b), nmx = std::max(a, b);
            return (2.0 * nmn + 1) * (nmx * (nmx + 2) + 1) * es + atcdim_h(a, b) * 2 * es + (2.0 * nmx + 1) * 2 * es;
        };
        double s = 0.0;
        for (int i = 0; i < c->n - 1; i++)
            for (int j = i + 1; j < c->n; j++)
                if (!c->hs.on() || c->hs.host[i] == c->hs.host[j]) s += canon(c->order[i], c->order[j]);
        if (c->hs.on())
            for (int j = 0; j < c->n; j++)
                if (c->hs.host[j] >= 0) s += canon(c->order[c->hs.host[j]], c->order[j]);
        *canonical = s;
    }
    return MSTMG_OK;
}

// ---- many systems at once ----


// cbicg for the systems listed in sys (columns of B and of the work vectors),
// all advanced together; system s stops where cbicg would stop it.  X (w.v().X)
// holds the initial guesses when have_x0.  iters/errs/status are indexed by
// system; status 2 = breakdown.
template <typename T>
int bicg_multi(mstmg_ctx* c, MultiWork<T>& w, const cpx<T>* B, const std::vector<int>& sys, bool have_x0, int niter,
                      const std::vector<double>& eps, std::vector<int>& iters, std::vector<double>& errs, std::vector<int>& status)
{
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    const cpx<T>* an = (sizeof(T) == 8) ? (const cpx<T>*)c->an.p : (const cpx<T>*)c->an32.p;
    MultiVecs<T> v = w.v(ne);
    const int per_chunk = (sizeof(T) == 4) ? 2 : 1;   // systems per translation chunk ([p, w] column pairs)
    const int NR = 2 * per_chunk;
    iters.assign(w.S, 0);
    errs.assign(w.S, 0.0);
    status.assign(w.S, 0);
    int a = (int)sys.size();
    if (a == 0) return MSTMG_OK;
    for (int k = 0; k < a; k++) w.hact[k] = sys[k];
    CK(cudaMemcpyAsync(w.act.p, w.hact.data(), sizeof(int) * a, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(w.epsv.p, eps.data(), sizeof(double) * w.S, cudaMemcpyHostToDevice, c->st));
    int rc;
    if (have_x0) {
        int apad = ((a + NR - 1) / NR) * NR;
        launch_m_gather<T>(ne, a, apad, w.act.p, v.X, w.XP.p, c->nsm, c->st);
        if ((rc = translate_many<T>(c, w.XP.p, w.YP.p, apad, 0u))) return rc;
    } else {
        for (int k = 0; k < a; k++) CK(cudaMemsetAsync(v.X + (size_t)sys[k] * ne, 0, sizeof(cpx<T>) * ne, c->st));
    }
    // host spheres (FP64): the Mie multiply runs apart, the fused kernels take an = null
    const bool hosts = sizeof(T) == 8 && c->hs.on();
    if (hosts && have_x0)
        for (int k = 0; k < a; k++) mie_all(c, 1, 0, (const zd*)(w.YP.p + (size_t)k * ne), (zd*)(w.YP.p + (size_t)k * ne));
    launch_m_init<T>(sm, hosts ? nullptr : an, ne, a, w.act.p, B, v, w.YP.p, have_x0 ? 1 : 0, w.part.p, w.sc.p, c->nsm, c->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(w.hsc.data(), w.sc.p, sizeof(BicgScalars) * w.S, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    auto compact = [&]() -> int {
        int na = 0;
        for (int k = 0; k < a; k++) {
            int s = w.hact[k];
            const BicgScalars& q = w.hsc[s];
            if (q.breakdown) status[s] = 2;
            else if (!q.stop) w.hact[na++] = s;
        }
        bool changed = (na != a);
        a = na;
        if (changed && a > 0) CK(cudaMemcpyAsync(w.act.p, w.hact.data(), sizeof(int) * a, cudaMemcpyHostToDevice, c->st));
        return MSTMG_OK;
    };
    if ((rc = compact())) return rc;
    for (int it = 1; it <= niter && a > 0; it++) {
        int apad = ((a + per_chunk - 1) / per_chunk) * per_chunk;
        launch_m_pack<T>(sm, hosts ? nullptr : an, ne, a, apad, w.act.p, v.P, v.W, w.XP.p, c->nsm, c->st);
        if (hosts)
            for (int k = 0; k < a; k++)
                mie_all(c, -1, 0, (const zd*)(w.XP.p + (size_t)(2 * k + 1) * ne), (zd*)(w.XP.p + (size_t)(2 * k + 1) * ne));
        if ((rc = translate_many<T>(c, w.XP.p, w.YP.p, 2 * apad, 2u))) return rc;
        if (hosts)
            for (int k = 0; k < a; k++) mie_all(c, 1, 0, (const zd*)(w.YP.p + (size_t)(2 * k) * ne), (zd*)(w.YP.p + (size_t)(2 * k) * ne));
        launch_m_post<T>(sm, hosts ? nullptr : an, ne, a, w.act.p, v, w.YP.p, w.part.p, w.sc.p, c->nsm, c->st, w.cnt.p);
        launch_m_upd<T>(ne, a, w.act.p, v, w.part.p, w.sc.p, w.epsv.p, c->nsm, c->st, w.cnt.p);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(w.hsc.data(), w.sc.p, sizeof(BicgScalars) * w.S, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        for (int k = 0; k < a; k++) {
            int s = w.hact[k];
            iters[s] = it;
            errs[s] = w.hsc[s].eerr;
        }
        if ((rc = compact())) return rc;
    }
    for (int k = 0; k < a; k++) iters[w.hact[k]] = niter + 1;   // Fortran DO-loop exit value when the cap is reached
    return check_kernel_err(c);
}

// Mixed precision for S systems: FP64 outer refinement (true residual with the
// FP64 operators), FP32 inner BiCG on the residual systems, all systems in
// lockstep.  X (FP64, ne x S) holds the initial guesses on entry.
int solve_multi_mixed(mstmg_ctx* c, MultiWork<double>& w64, MultiWork<float>& w32, DevBuf<zf>& B32, DevBuf<double>& rr,
                             DevBuf<int>& idx, int S, const zd* B, zd* X, double eps, int niter, std::vector<int>& iters,
                             std::vector<double>& errs, std::vector<int>& status, int* outer_count)
{
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    std::vector<int> act(S), total(S, 0);
    for (int s = 0; s < S; s++) act[s] = s;
    iters.assign(S, 0);
    errs.assign(S, 1.0);
    status.assign(S, 0);
    std::vector<double> hrr(2 * (size_t)S), ieps(w32.S, 1.0);
    std::vector<int> it2, st2, map(2 * (size_t)S);
    std::vector<double> e2;
    int rc;
    *outer_count = 0;
    for (int outer = 0; outer < c->opts.max_outer && !act.empty(); outer++) {
        int a = (int)act.size();
        int apad = ((a + 1) / 2) * 2;
        CK(cudaMemcpyAsync(w64.act.p, act.data(), sizeof(int) * a, cudaMemcpyHostToDevice, c->st));
        launch_m_gather<double>(ne, a, apad, w64.act.p, X, w64.XP.p, c->nsm, c->st);
        if ((rc = translate_many<double>(c, w64.XP.p, w64.YP.p, apad, 0u))) return rc;
        launch_m_resid<float>(sm, c->an.p, ne, a, w64.act.p, B, X, w64.YP.p, B32.p, w64.part.p, rr.p, c->nsm, c->st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hrr.data(), rr.p, sizeof(double) * 2 * S, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        *outer_count = outer + 1;
        std::vector<int> inner, keep;   // inner: residual columns k to refine; keep: their systems
        int cap = niter;
        for (int k = 0; k < a; k++) {
            int s = act[k];
            double bb = hrr[2 * s + 1];
            errs[s] = bb > 0.0 ? hrr[2 * s] / bb : 0.0;
            if (errs[s] < eps || total[s] >= niter) continue;
            inner.push_back(k);
            keep.push_back(s);
            ieps[k] = std::max(eps / errs[s] * 0.01, c->opts.inner_eps);
            cap = std::min(cap, niter - total[s]);
        }
        if (inner.empty()) break;
        if (cap < 1) cap = 1;
        if ((rc = bicg_multi<float>(c, w32, B32.p, inner, false, cap, ieps, it2, e2, st2))) return rc;
        const int ni = (int)inner.size();
        for (int j = 0; j < ni; j++) {
            int k = inner[j], s = keep[j];
            total[s] += std::min(it2[k], cap);
            if (st2[k] == 2) status[s] = 2;
            map[j] = s;
            map[S + j] = k;
        }
        CK(cudaMemcpyAsync(idx.p, map.data(), sizeof(int) * 2 * S, cudaMemcpyHostToDevice, c->st));
        launch_m_addcorr<float>(ne, ni, idx.p, idx.p + S, X, w32.v(ne).X, c->st);
        CK(cudaGetLastError());
        act = keep;
    }
    for (int s = 0; s < S; s++) iters[s] = total[s];
    return check_kernel_err(c);
}

// Mixed precision for S systems by residual replacement ("reliable updates"):
// one FP32 BiCG per system, never restarted, all systems advanced together
// (one translation launch per step).  Whenever a system's recursive residual
// has fallen by `drop` since its last replacement, or claims convergence, its
// FP32 iterate is folded into the FP64 solution X, the FP64 true residual
// b - (I - M H) x replaces r, and csk/beta are recomputed from it.  The same
// FP64 pass also replaces every other system whose residual has fallen by
// `drop_soft`, so the systems share their FP64 passes.  A system stops when
// its true residual ratio is below eps.  X holds the initial guesses on entry.
// Used for the T-matrix columns and for the two polarisations of a
// fixed-orientation solve.
int solve_multi_rr(mstmg_ctx* c, MultiWork<double>& w64, MultiWork<float>& w32, DevBuf<double>& rr, DevBuf<int>& idx, int S,
                          const zd* B, zd* X, double eps, int niter, std::vector<int>& iters, std::vector<double>& errs,
                          std::vector<int>& status, int* outer_count)
{
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    const zf* an32 = (const zf*)c->an32.p;
    MultiVecs<float> v = w32.v(ne);
    const double drop = 1.0e-5, drop_soft = 1.0e-3;
    std::vector<int> act(S), tot(S, 0);
    std::vector<double> base(S, 1.0), ratio(S, 0.0), hrr(2 * (size_t)S);
    for (int s = 0; s < S; s++) act[s] = s;
    iters.assign(S, 0);
    errs.assign(S, 1.0);
    status.assign(S, 0);
    *outer_count = 0;
    int rc;
    // FP64 true residual of the systems in L, rounded into their FP32 r
    auto true_residual = [&](const std::vector<int>& Ls) -> int {
        const int a = (int)Ls.size();
        if (a == 0) return MSTMG_OK;
        const int apad = a == 1 ? 1 : ((a + 1) / 2) * 2;   // whole FP64 chunks of 2; a lone column alone
        CK(cudaMemcpyAsync(w64.act.p, Ls.data(), sizeof(int) * a, cudaMemcpyHostToDevice, c->st));
        launch_m_gather<double>(ne, a, apad, w64.act.p, X, w64.XP.p, c->nsm, c->st);
        int r2 = translate_many<double>(c, w64.XP.p, w64.YP.p, apad, 0u);
        if (r2) return r2;
        launch_m_resid<float>(sm, c->an.p, ne, a, w64.act.p, B, X, w64.YP.p, v.R, w64.part.p, rr.p, c->nsm, c->st, 1);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hrr.data(), rr.p, sizeof(double) * 2 * S, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        (*outer_count)++;
        for (int s : Ls) ratio[s] = hrr[2 * s + 1] > 0.0 ? hrr[2 * s] / hrr[2 * s + 1] : 0.0;
        return MSTMG_OK;
    };
    auto upload_act = [&]() -> int {
        if (!act.empty()) CK(cudaMemcpyAsync(w32.act.p, act.data(), sizeof(int) * act.size(), cudaMemcpyHostToDevice, c->st));
        return MSTMG_OK;
    };
    if ((rc = true_residual(act))) return rc;
    {
        std::vector<int> keep;
        for (int s : act) {
            base[s] = errs[s] = ratio[s];
            if (ratio[s] >= eps && niter > 0) keep.push_back(s);
        }
        act = keep;
    }
    if (act.empty()) return check_kernel_err(c);
    // FP32 BiCG from the true residual: x32 = 0, p = r, q = w = conj(r)
    if ((rc = upload_act())) return rc;
    for (int s : act) CK(cudaMemsetAsync(v.X + (size_t)s * ne, 0, sizeof(zf) * ne, c->st));
    launch_m_init<float>(sm, an32, ne, (int)act.size(), w32.act.p, v.R, v, nullptr, 0, w32.part.p, w32.sc.p, c->nsm, c->st);
    CK(cudaGetLastError());
    const int per_chunk = 2;   // systems per FP32 translation chunk ([p, w] column pairs)
    for (int it = 1; it <= niter && !act.empty(); it++) {
        const int a = (int)act.size();
        const int apad = a == 1 ? 1 : ((a + per_chunk - 1) / per_chunk) * per_chunk;   // a lone system: its 2 columns alone
        launch_m_pack<float>(sm, an32, ne, a, apad, w32.act.p, v.P, v.W, w32.XP.p, c->nsm, c->st);
        if ((rc = translate_many<float>(c, w32.XP.p, w32.YP.p, 2 * apad, 2u))) return rc;
        launch_m_post<float>(sm, an32, ne, a, w32.act.p, v, w32.YP.p, w32.part.p, w32.sc.p, c->nsm, c->st, w32.cnt.p);
        launch_m_upd1<float>(ne, a, w32.act.p, v, w32.part.p, w32.sc.p, c->nsm, c->st, w32.cnt.p);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(w32.hsc.data(), w32.sc.p, sizeof(BicgScalars) * S, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        std::vector<int> repl, keep;
        bool trigger = false;
        for (int s : act) {
            tot[s] = it;
            const BicgScalars& q = w32.hsc[s];
            if (q.breakdown) {
                // breakdown: fold the iterate in and report it
                status[s] = 2;
                continue;
            }
            if (q.stop || q.eerr * base[s] < eps || q.eerr < drop) trigger = true;
            keep.push_back(s);
        }
        // one FP64 pass serves every system close to its next replacement
        if (trigger)
            for (int s : keep) {
                const BicgScalars& q = w32.hsc[s];
                if (q.stop || q.eerr * base[s] < eps || q.eerr < drop_soft) repl.push_back(s);
            }
        for (int s : act)
            if (status[s] == 2) {
                std::vector<int> one{s};
                CK(cudaMemcpyAsync(idx.p, one.data(), sizeof(int), cudaMemcpyHostToDevice, c->st));
                launch_m_addcorr<float>(ne, 1, idx.p, idx.p, X, v.X, c->st);
            }
        if (!repl.empty()) {
            const int nr = (int)repl.size();
            CK(cudaMemcpyAsync(idx.p, repl.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, c->st));
            launch_m_addcorr<float>(ne, nr, idx.p, idx.p, X, v.X, c->st);
            for (int s : repl) CK(cudaMemsetAsync(v.X + (size_t)s * ne, 0, sizeof(zf) * ne, c->st));
            if ((rc = true_residual(repl))) return rc;
            std::vector<int> fix, keep2;
            for (int s : keep) {
                bool replaced = std::find(repl.begin(), repl.end(), s) != repl.end();
                if (replaced) {
                    errs[s] = base[s] = ratio[s];
                    if (ratio[s] < eps) continue;   // converged
                    fix.push_back(s);
                }
                keep2.push_back(s);
            }
            if (!fix.empty()) {
                CK(cudaMemcpyAsync(idx.p, fix.data(), sizeof(int) * fix.size(), cudaMemcpyHostToDevice, c->st));
                launch_m_rrfix<float>(ne, (int)fix.size(), idx.p, v, w32.part.p, w32.sc.p, c->nsm, c->st);
            }
            keep = keep2;
        }
        if (keep.size() != act.size()) {
            act = keep;
            if ((rc = upload_act())) return rc;
        }
        if (!act.empty()) launch_m_upd2<float>(ne, (int)act.size(), w32.act.p, v, w32.sc.p, c->nsm, c->st);
        CK(cudaGetLastError());
    }
    if (!act.empty()) {
        // iteration cap: fold the last FP32 steps in
        CK(cudaMemcpyAsync(idx.p, act.data(), sizeof(int) * act.size(), cudaMemcpyHostToDevice, c->st));
        launch_m_addcorr<float>(ne, (int)act.size(), idx.p, idx.p, X, v.X, c->st);
        for (int s : act) tot[s] = niter + 1;
    }
    for (int s = 0; s < S; s++) iters[s] = tot[s];
    return check_kernel_err(c);
}

// Mixed precision for S systems by restarted GMRES.  A cycle starts from the
// FP64 true residuals of its systems (one shared pass) and runs FP32 Arnoldi
// steps: one translation pass over the basis vectors of the systems still
// active, classical Gram-Schmidt applied twice with FP64 sums, and the
// Givens-rotated least-squares residual of each system tracked on the host.
// A system leaves the cycle when that estimate falls below its target
// (eps |b|^2 / 4, but no deeper than inner_eps times the cycle's starting
// residual; squared norms) or its Krylov space is invariant; the cycle ends
// when no system is left or after m steps.  Each system's correction is then
// summed into the FP64 solution X, and the next cycle's true residuals tell
// which systems are done: squared residual ratio below eps, the cbicg test
// of the reference.  iters counts Arnoldi steps in pairs (a BiCG iteration
// is two matvecs), so the cap niter allows 2 niter steps.  X holds the
// initial guesses on entry.
// With seg (an ensemble), system s = 2 c + p is the segment of configuration c
// in column p of the ne x 2 blocks B and X: every pass translates the two
// columns with the active systems' basis vectors in their segments (the
// operator has no pairs between configurations), and each system keeps its
// own basis, Hessenberg matrix and stopping test.
// x_zero: X holds zeros on entry, so the first cycle's true residual is B
// itself and needs no FP64 pass.
// W = XP - M Y for na columns; with host spheres the Mie multiply runs
// apart (on Y in place) and the kernel takes Y as M H v
static void gm_apply_ctx(mstmg_ctx* c, const SlotMaps& sm, const zf* an32, int ne, int na, const zf* XP, zf* Y, zf* W)
{
    if (c->hs.on()) {
        for (int k = 0; k < na; k++) mie_all<float>(c, 1, 0, Y + (size_t)k * ne, Y + (size_t)k * ne);
        launch_gm_apply(sm, nullptr, ne, na, XP, Y, W, c->nsm, c->st);
    } else {
        launch_gm_apply(sm, an32, ne, na, XP, Y, W, c->nsm, c->st);
    }
}

int solve_multi_gmres(mstmg_ctx* c, MultiWork<double>& w64, GmresWork& gw, int S, const zd* B, zd* X, double eps, int niter,
                             std::vector<int>& iters, std::vector<double>& errs, std::vector<int>& status, int* outer_count,
                             const EnsSeg* seg, bool x_zero)
{
    using C = std::complex<double>;
    NvtxRange nvtx_("mixed GMRES");
    c->host_syncs = 0;
    const int ne = c->neqns, m = gw.m, m1 = gw.m + 1;
    const int ldv = seg ? seg->ldv : ne;             // elements a basis vector is stored in
    const int* slen = seg ? seg->len : nullptr;      // elements a system's vectors hold
    // Arnoldi steps as CUDA graphs for the two-column solves (a fixed
    // orientation, an ensemble), whose steps are launch-bound on small
    // clusters: not with kernel timing (events) or the FFT path (cuFFT plans)
    bool graphs = gw.graphs_ok && (seg || S <= 2) && !c->timing && !(c->fft && c->fft->on);
    if (graphs && gw.graph_gen != c->layout_gen) {
        gw.drop_graphs();
        gw.graph_gen = c->layout_gen;
    }
    SlotMaps sm = c->sm();
    const zf* an32 = (const zf*)c->an32.p;
    const size_t O1 = gw.off1(), HP = gw.hpass();
    double* h1 = gw.h.p + O1;
    double* h2 = h1 + HP;
    const long long cap = 2LL * std::max(niter, 0);
    std::vector<int> act(S), cur;
    std::vector<long long> steps(S, 0);
    std::vector<double> hrr(2 * (size_t)S);
    for (int s = 0; s < S; s++) act[s] = s;
    iters.assign(S, 0);
    errs.assign(S, 1.0);
    status.assign(S, 0);
    *outer_count = 0;
    int rc;
    auto rot = [&](int s) { return (size_t)s * m; };
    auto colR = [&](int s, int j) { return &gw.Rm[((size_t)s * m + j) * m1]; };
    // a device-driven cycle leaves its step counts in gw.hkk (pinned), read
    // after the next synchronisation
    std::vector<int> dev_act;
    long long dev_per_step = 0;
    int dev_passes_per_step = 0;
    auto fold_device_cycle = [&]() {
        if (dev_act.empty()) return;
        for (int s : dev_act) {
            steps[s] += gw.hkk[s];
            if (gw.hkk[S + s] == 2) status[s] = 2;
        }
        const int nstep = gw.hkk[2 * S];
        launch_counter() += (long long)nstep * dev_per_step;
        c->passes32 += nstep * dev_passes_per_step;
        dev_act.clear();
    };
    for (int cyc = 0; cyc <= c->opts.max_outer && !act.empty(); cyc++) {
        // FP64 true residuals of the cycle's systems into R (FP32, by system,
        // or the two columns of an ensemble)
        int a = (int)act.size();
        if (seg) {
            CK(cudaMemcpyAsync(gw.act.p, act.data(), sizeof(int) * a, cudaMemcpyHostToDevice, c->st));
            if ((rc = translate_many<double>(c, X, c->Y64.p, 2, 0u))) return rc;
            CK(cudaMemsetAsync(gw.rr.p, 0, sizeof(double) * 2 * S, c->st));
            launch_eg_resid(sm, c->an.p, ne, ldv, a, gw.act.p, seg->off, seg->len, B, X, c->Y64.p, gw.R.p, gw.rr.p, c->nsm, c->st);
        } else {
            const int apad = a == 1 ? 1 : ((a + 1) / 2) * 2;
            CK(cudaMemcpyAsync(w64.act.p, act.data(), sizeof(int) * a, cudaMemcpyHostToDevice, c->st));
            if (x_zero && cyc == 0) {
                // H 0 = 0: the residual is B
                CK(cudaMemsetAsync(w64.YP.p, 0, sizeof(zd) * (size_t)ne * apad, c->st));
            } else {
                launch_m_gather<double>(ne, a, apad, w64.act.p, X, w64.XP.p, c->nsm, c->st);
                if ((rc = translate_many<double>(c, w64.XP.p, w64.YP.p, apad, 0u))) return rc;
            }
            if (c->hs.on()) {
                // host spheres: the Mie multiply apart, the residual kernel takes M H x
                for (int k = 0; k < a; k++) mie_all<double>(c, 1, 0, w64.YP.p + (size_t)k * ne, w64.YP.p + (size_t)k * ne);
                launch_m_resid<float>(sm, nullptr, ne, a, w64.act.p, B, X, w64.YP.p, gw.R.p, w64.part.p, gw.rr.p, c->nsm, c->st, 1);
            } else {
                launch_m_resid<float>(sm, c->an.p, ne, a, w64.act.p, B, X, w64.YP.p, gw.R.p, w64.part.p, gw.rr.p, c->nsm, c->st, 1);
            }
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hrr.data(), gw.rr.p, sizeof(double) * 2 * S, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        c->host_syncs++;
        (*outer_count)++;
        fold_device_cycle();
        std::vector<int> keep;
        for (int s : act) {
            const double bb = hrr[2 * s + 1];
            errs[s] = bb > 0.0 ? hrr[2 * s] / bb : 0.0;
            if (errs[s] >= eps && steps[s] < cap && status[s] != 2) keep.push_back(s);
        }
        act = keep;
        a = (int)act.size();
        if (a == 0 || cyc == c->opts.max_outer) break;
        CK(cudaMemcpyAsync(gw.act.p, act.data(), sizeof(int) * a, cudaMemcpyHostToDevice, c->st));
        // v_0 = r / |r|
        if (seg) launch_eg_start(ne, ldv, m1, a, gw.act.p, seg->off, seg->len, gw.R.p, gw.rr.p, 1.0e-35, gw.V.p, c->nsm, c->st);
        else launch_gm_scale(ne, m1, 0, a, gw.act.p, 1, gw.R.p, gw.rr.p, 2, 1.0e-35, gw.V.p, c->nsm, c->st);
        long long room = cap;
        for (int s : act) {
            const double beta2 = hrr[2 * s];
            gw.target[s] = std::max(0.25 * eps * hrr[2 * s + 1], c->opts.inner_eps * beta2);
            std::fill(gw.g.begin() + (size_t)s * m1, gw.g.begin() + (size_t)(s + 1) * m1, C(0.0));
            gw.g[(size_t)s * m1] = C(std::sqrt(beta2));
            gw.kk[s] = 0;
            gw.frozen[s] = 0;
            room = std::min(room, cap - steps[s]);
        }
        cur = act;
        const int jmax = (int)std::min<long long>(m, room);
        if (graphs && jmax > 0) {
            // the whole cycle on the device: one graph launch, its Arnoldi
            // step repeated under a conditional WHILE node until every system
            // has left or jmax steps are done; then the least-squares
            // solutions and the corrections, with no synchronisation
            const int na = a;
            std::vector<int> alive(S, 0);
            std::vector<double2> g0((size_t)S * m1, make_double2(0.0, 0.0));
            for (int s : act) {
                alive[s] = 1;
                g0[(size_t)s * m1] = make_double2(std::sqrt(hrr[2 * s]), 0.0);
            }
            const int zero = 0;
            CK(cudaMemcpyAsync(gw.dalive.p, alive.data(), sizeof(int) * S, cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(gw.dg.p, g0.data(), sizeof(double2) * g0.size(), cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(gw.dtarget.p, gw.target.data(), sizeof(double) * S, cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(gw.dj.p, &zero, sizeof(int), cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(gw.djmax.p, &jmax, sizeof(int), cudaMemcpyHostToDevice, c->st));
            CK(cudaMemsetAsync(gw.dkk.p, 0, sizeof(int) * S, c->st));
            CK(cudaMemsetAsync(gw.dstatus.p, 0, sizeof(int) * S, c->st));
            auto it = gw.cycles.find(na);
            if (it == gw.cycles.end()) {
                cudaGraph_t gr = nullptr, body = nullptr;
                cudaGraphExec_t ex = nullptr;
                cudaGraphConditionalHandle hc;
                bool ok = cudaGraphCreate(&gr, 0) == cudaSuccess && cudaGraphConditionalHandleCreate(&hc, gr, 1, cudaGraphCondAssignDefault) == cudaSuccess;
                cudaGraphNodeParams np = {};
                cudaGraphNode_t node;
                if (ok) {
                    np.type = cudaGraphNodeTypeConditional;
                    np.conditional.handle = hc;
                    np.conditional.type = cudaGraphCondTypeWhile;
                    np.conditional.size = 1;
                    ok = cudaGraphAddNode(&node, gr, nullptr, 0, &np) == cudaSuccess;
                }
                if (ok) body = np.conditional.phGraph_out[0];
                const long long l0 = launch_counter().load();
                const int p0 = c->passes32;
                int src = MSTMG_ERR_CUDA;
                if (ok) ok = cudaStreamBeginCaptureToGraph(c->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                if (ok) {
                    src = [&]() -> int {
                        GmDevState d = gw.dev();
                        if (seg) {
                            CK(cudaMemsetAsync(gw.XP.p, 0, sizeof(zf) * 2 * (size_t)ne, c->st));
                            launch_eg_gather_dev(ne, ldv, m1, na, gw.act.p, seg->off, seg->len, d.j, d.alive, gw.V.p, gw.XP.p, c->nsm, c->st);
                            int r2 = translate_many<float>(c, gw.XP.p, gw.Y.p, 2, 0u);
                            if (r2) return r2;
                            launch_eg_apply(sm, an32, ne, ldv, na, gw.act.p, seg->off, seg->len, gw.XP.p, gw.Y.p, gw.W.p, c->nsm, c->st);
                        } else {
                            launch_gm_gather_dev(ne, m1, na, na, gw.act.p, d.j, d.alive, gw.V.p, gw.XP.p, c->nsm, c->st);
                            int r2 = translate_many<float>(c, gw.XP.p, gw.Y.p, na, 0u);
                            if (r2) return r2;
                            gm_apply_ctx(c, sm, an32, ne, na, gw.XP.p, gw.Y.p, gw.W.p);
                        }
                        CK(cudaMemsetAsync(gw.h.p, 0, sizeof(double) * (O1 + 2 * HP), c->st));
                        launch_gm_dots_dev(ldv, S, m1, na, gw.act.p, d.j, gw.V.p, gw.W.p, h1, nullptr, c->nsm, c->st, slen);
                        launch_gm_update_dev(ldv, S, m1, na, gw.act.p, d.j, gw.V.p, h1, gw.W.p, nullptr, c->nsm, c->st, slen);
                        launch_gm_dots_dev(ldv, S, m1, na, gw.act.p, d.j, gw.V.p, gw.W.p, h2, h1, c->nsm, c->st, slen);
                        launch_gm_update_dev(ldv, S, m1, na, gw.act.p, d.j, gw.V.p, h2, gw.W.p, gw.h.p, c->nsm, c->st, slen);
                        launch_gm_scale_dev(ldv, m1, na, gw.act.p, d.j, gw.W.p, gw.h.p, 1.0e-35, gw.V.p, c->nsm, c->st, slen);
                        launch_gm_givens(S, m, na, gw.act.p, gw.h.p, h1, d, hc, c->st);
                        CK(cudaGetLastError());
                        return MSTMG_OK;
                    }();
                    cudaGraph_t cap = nullptr;
                    ok = cudaStreamEndCapture(c->st, &cap) == cudaSuccess && src == MSTMG_OK;
                }
                if (ok) ok = cudaGraphInstantiate(&ex, gr, 0) == cudaSuccess;
                if (gr) cudaGraphDestroy(gr);
                const long long dl = launch_counter().load() - l0;
                launch_counter() -= dl;   // counted per step when the graph runs
                const int dp = c->passes32 - p0;
                c->passes32 = p0;
                if (!ok) {
                    if (ex) cudaGraphExecDestroy(ex);
                    (void)cudaGetLastError();   // the failed capture's error
                    gw.graphs_ok = false;
                    graphs = false;
                } else {
                    it = gw.cycles.emplace(na, GmresWork::CycleGraph{ex, dl, dp}).first;
                }
            }
            if (graphs) {
                CK(cudaGraphLaunch(it->second.exec, c->st));
                dev_per_step = it->second.launches_per_step;
                dev_passes_per_step = it->second.passes32_per_step;
                // least-squares solutions on the device, summed into X
                GmDevState d = gw.dev();
                CK(cudaMemsetAsync(h2, 0, sizeof(double) * HP, c->st));
                CK(cudaMemsetAsync(gw.dkmax.p, 0, sizeof(int), c->st));
                launch_gm_backsolve(S, m, na, gw.act.p, d, h2, gw.dkmax.p, c->st);
                if (seg) launch_eg_combine_dev(ne, ldv, S, m1, na, gw.act.p, seg->off, seg->len, gw.V.p, h2, gw.dkmax.p, X, c->nsm, c->st);
                else launch_gm_combine_dev(ne, S, m1, na, gw.act.p, gw.V.p, h2, gw.dkmax.p, X, c->nsm, c->st);
                CK(cudaGetLastError());
                CK(cudaMemcpyAsync(gw.hkk, gw.dkk.p, sizeof(int) * S, cudaMemcpyDeviceToHost, c->st));
                CK(cudaMemcpyAsync(gw.hkk + S, gw.dstatus.p, sizeof(int) * S, cudaMemcpyDeviceToHost, c->st));
                CK(cudaMemcpyAsync(gw.hkk + 2 * S, gw.dj.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
                dev_act = act;
                continue;
            }
            // capture failed: the host-driven steps below
            CK(cudaMemcpyAsync(gw.act.p, act.data(), sizeof(int) * a, cudaMemcpyHostToDevice, c->st));
        }
        for (int j = 0; j < jmax && !cur.empty(); j++) {
            const int na = (int)cur.size();
            const size_t hn = (size_t)(j + 1) * S * 2;
            // one Arnoldi step on the device: the pass, the Mie multiply, two
            // Gram-Schmidt passes, the new basis vector, the Hessenberg column home
            auto step = [&]() -> int {
                int r2;
                if (seg) {
                    CK(cudaMemsetAsync(gw.XP.p, 0, sizeof(zf) * 2 * (size_t)ne, c->st));
                    launch_eg_gather(ne, ldv, m1, j, na, gw.act.p, seg->off, seg->len, gw.V.p, gw.XP.p, c->nsm, c->st);
                    if ((r2 = translate_many<float>(c, gw.XP.p, gw.Y.p, 2, 0u))) return r2;
                    launch_eg_apply(sm, an32, ne, ldv, na, gw.act.p, seg->off, seg->len, gw.XP.p, gw.Y.p, gw.W.p, c->nsm, c->st);
                } else {
                    const int npad = na <= 2 ? na : ((na + 3) / 4) * 4;   // whole FP32 chunks
                    launch_gm_gather(ne, m1, j, na, npad, gw.act.p, gw.V.p, gw.XP.p, c->nsm, c->st);
                    if ((r2 = translate_many<float>(c, gw.XP.p, gw.Y.p, npad, 0u))) return r2;
                    gm_apply_ctx(c, sm, an32, ne, na, gw.XP.p, gw.Y.p, gw.W.p);
                }
                CK(cudaMemsetAsync(gw.h.p, 0, sizeof(double) * (O1 + hn), c->st));
                CK(cudaMemsetAsync(h2, 0, sizeof(double) * hn, c->st));
                launch_gm_dots(ldv, S, m1, j + 1, na, gw.act.p, gw.V.p, gw.W.p, h1, nullptr, c->nsm, c->st, slen);
                launch_gm_update(ldv, S, m1, j + 1, na, gw.act.p, gw.V.p, h1, gw.W.p, nullptr, c->nsm, c->st, slen);
                launch_gm_dots(ldv, S, m1, j + 1, na, gw.act.p, gw.V.p, gw.W.p, h2, h1, c->nsm, c->st, slen);
                launch_gm_update(ldv, S, m1, j + 1, na, gw.act.p, gw.V.p, h2, gw.W.p, gw.h.p, c->nsm, c->st, slen);
                launch_gm_scale(ldv, m1, j + 1, na, gw.act.p, 0, gw.W.p, gw.h.p, 1, 1.0e-35, gw.V.p, c->nsm, c->st, slen);
                CK(cudaGetLastError());
                CK(cudaMemcpyAsync(gw.hh, gw.h.p, sizeof(double) * (O1 + hn), cudaMemcpyDeviceToHost, c->st));
                return MSTMG_OK;
            };
            if (graphs) {
                // replayed as a CUDA graph, captured the first time this (step,
                // active systems) shape comes up; plain launches if capture fails
                const long long key = ((long long)j << 32) | (long long)(unsigned)na;
                auto it = gw.graphs.find(key);
                if (it == gw.graphs.end()) {
                    const long long l0 = launch_counter().load();
                    const int p0 = c->passes32;
                    cudaGraph_t gr = nullptr;
                    cudaGraphExec_t ex = nullptr;
                    bool ok = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                    const int src = ok ? step() : MSTMG_ERR_CUDA;
                    if (ok) ok = cudaStreamEndCapture(c->st, &gr) == cudaSuccess && src == MSTMG_OK && gr != nullptr;
                    if (ok) ok = cudaGraphInstantiate(&ex, gr, 0) == cudaSuccess;
                    if (gr) cudaGraphDestroy(gr);
                    const long long dl = launch_counter().load() - l0;
                    launch_counter() -= dl;   // counted when the graph runs
                    const int dp = c->passes32 - p0;
                    c->passes32 = p0;
                    if (!ok) {
                        if (ex) cudaGraphExecDestroy(ex);
                        (void)cudaGetLastError();   // the failed capture's error
                        gw.graphs_ok = false;
                        graphs = false;
                        if ((rc = step())) return rc;
                    } else {
                        it = gw.graphs.emplace(key, GmresWork::StepGraph{ex, dl, dp}).first;
                    }
                }
                if (graphs) {
                    CK(cudaGraphLaunch(it->second.exec, c->st));
                    launch_counter() += it->second.launches;
                    c->passes32 += it->second.passes32;
                }
            } else if ((rc = step())) {
                return rc;
            }
            CK(cudaStreamSynchronize(c->st));
        c->host_syncs++;
            const double* H1 = gw.hh + O1;
            std::vector<int> next;
            for (int s : cur) {
                C* col = colR(s, j);
                double cn = 0.0;
                for (int i = 0; i <= j; i++) {
                    const size_t o = 2 * ((size_t)i * S + s);
                    col[i] = C(H1[o], H1[o + 1]);
                    cn += std::norm(col[i]);
                }
                const double hsub = std::sqrt(std::max(gw.hh[s], 0.0));
                for (int i = 0; i < j; i++) {   // the earlier rotations
                    const double ci = gw.cs[rot(s) + i];
                    const C si = gw.sn[rot(s) + i];
                    const C t = ci * col[i] + si * col[i + 1];
                    col[i + 1] = -std::conj(si) * col[i] + ci * col[i + 1];
                    col[i] = t;
                }
                const double aa = std::abs(col[j]), rho = std::sqrt(aa * aa + hsub * hsub);
                if (rho == 0.0) {   // A v_j = 0: the operator is singular
                    status[s] = 2;
                    continue;
                }
                const C ph = aa > 0.0 ? col[j] / aa : C(1.0);
                gw.cs[rot(s) + j] = aa / rho;
                gw.sn[rot(s) + j] = ph * hsub / rho;
                col[j] = ph * rho;
                C* gs = &gw.g[(size_t)s * m1];
                gs[j + 1] = -std::conj(gw.sn[rot(s) + j]) * gs[j];
                gs[j] = gw.cs[rot(s) + j] * gs[j];
                gw.kk[s] = j + 1;
                // leave: estimate below target, or the Krylov space is invariant
                if (std::norm(gs[j + 1]) >= gw.target[s] && hsub > 1.0e-13 * std::sqrt(cn + hsub * hsub)) next.push_back(s);
            }
            if (next.size() != cur.size()) {
                cur = next;
                if (!cur.empty()) CK(cudaMemcpyAsync(gw.act.p, cur.data(), sizeof(int) * cur.size(), cudaMemcpyHostToDevice, c->st));
            }
        }
        // least-squares solutions (zero-padded to the longest), summed into X
        int kmax = 0;
        for (int s : act) kmax = std::max(kmax, gw.kk[s]);
        if (kmax > 0) {
            std::fill(gw.ybuf.begin(), gw.ybuf.begin() + (size_t)kmax * S * 2, 0.0);
            std::vector<C> y(kmax);
            for (int s : act) {
                const int ks = gw.kk[s];
                const C* gs = &gw.g[(size_t)s * m1];
                for (int i = ks - 1; i >= 0; i--) {
                    C t = gs[i];
                    for (int l = i + 1; l < ks; l++) t -= colR(s, l)[i] * y[l];
                    y[i] = t / colR(s, i)[i];
                    gw.ybuf[2 * ((size_t)i * S + s)] = y[i].real();
                    gw.ybuf[2 * ((size_t)i * S + s) + 1] = y[i].imag();
                }
                steps[s] += ks;
            }
            CK(cudaMemcpyAsync(gw.act.p, act.data(), sizeof(int) * a, cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(h2, gw.ybuf.data(), sizeof(double) * 2 * (size_t)kmax * S, cudaMemcpyHostToDevice, c->st));
            if (seg) launch_eg_combine(ne, ldv, S, m1, kmax, a, gw.act.p, seg->off, seg->len, gw.V.p, h2, X, c->nsm, c->st);
            else launch_gm_combine(ne, S, m1, kmax, a, gw.act.p, gw.V.p, h2, X, c->nsm, c->st);
            CK(cudaGetLastError());
        }
    }
    if (!dev_act.empty()) {
        CK(cudaStreamSynchronize(c->st));
        c->host_syncs++;
        fold_device_cycle();
    }
    for (int s = 0; s < S; s++) {
        iters[s] = (int)((steps[s] + 1) / 2);
        if (errs[s] >= eps && steps[s] >= cap) iters[s] = niter + 1;   // the cap was reached
    }
    return check_kernel_err(c);
}


template int bicg_batched<double>(mstmg_ctx*, int, const zd* const*, BicgVecs<double>*, bool, int, const double*, int*, double*, int*);
template int bicg_multi<double>(mstmg_ctx*, MultiWork<double>&, const zd*, const std::vector<int>&, bool, int, const std::vector<double>&,
                                std::vector<int>&, std::vector<double>&, std::vector<int>&);
template int bicg_multi<float>(mstmg_ctx*, MultiWork<float>&, const zf*, const std::vector<int>&, bool, int, const std::vector<double>&,
                               std::vector<int>&, std::vector<double>&, std::vector<int>&);
