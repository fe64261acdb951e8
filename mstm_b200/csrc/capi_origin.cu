// capi_origin.cu -- cluster-origin post-processing behind the C ABI: the
// translation orders to the cluster origin (tranordertest), the merge to
// the common origin, the GSF expansion and scattering matrix of a
// fixed-orientation solution, and the cluster T matrix (tmatrix_solution)
// with its random-orientation averages.
#include "ctx.cuh"

// ---------------------------------------------------------------------------
// Scattering post-processing of a solution (main_calling_program,
// mstm-input-37.f90:1159-1197 and 1497-1532): translation orders and
// t_matrix_order, merge to the common origin, GSF expansion, azimuth-averaged
// scattering matrix on nangles polar angles 0..180 deg, and g.
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Cluster-origin post-processing and the T matrix
// ---------------------------------------------------------------------------

mstmg::Tables& big_tables()
{
    static thread_local mstmg::Tables* big = nullptr;
    if (!big) big = new mstmg::Tables(420);
    return *big;
}

// Device copies of the bcof / sqrt tables of big_tables().
struct BigTablesDev {
    DevBuf<double> bc, fnr;
    int nbc = 420;
};
static int upload_big(mstmg_ctx* c, BigTablesDev& d)
{
    mstmg::Tables& big = big_tables();
    CK(d.bc.alloc(big.bcof.size()));
    CK(d.fnr.alloc(big.fnr.size()));
    CK(cudaMemcpyAsync(d.bc.p, big.bcof.data(), sizeof(double) * big.bcof.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(d.fnr.p, big.fnr.data(), sizeof(double) * big.fnr.size(), cudaMemcpyHostToDevice, c->st));
    return MSTMG_OK;
}

// Cluster origin (mean position of the spheres) and the order each sphere
// needs to reach it (tranordertest, modules:1896-1942, capped at max_t_order);
// T = max(min(L, max_t_order), those orders)  (input:1179-1197).
static int origin_orders(mstmg_ctx* c, const BigTablesDev& bt, double trans_eps, int max_t_order, double* r0, DevBuf<int>& dtord,
                         std::vector<int>& tord, int* T)
{
    const int n = c->n;
    // with host spheres: over the spheres outside every other (input:1166-1197)
    auto outside = [&](int i) { return !c->hs.on() || c->hs.host[i] < 0; };
    r0[0] = r0[1] = r0[2] = 0.0;
    int nout = 0;
    for (int i = 0; i < n; i++)
        if (outside(i)) {
            nout++;
            for (int k = 0; k < 3; k++) r0[k] = r0[k] + c->hpos[3 * (size_t)i + k];
        }
    for (int k = 0; k < 3; k++) r0[k] = r0[k] / (double)nout;
    DevBuf<zd> tscr;
    const int sstride = 3 * (200 + MSTMG_LMAX + 4);
    CK(dtord.alloc(n));
    CK(tscr.alloc(tranorder_scratch(n, sstride)));
    launch_tranorder(n, c->pos.p, c->d_order.p, r0, c->opts.medium_re, trans_eps, max_t_order, bt.bc.p, bt.fnr.p, bt.nbc, tscr.p, sstride,
                     dtord.p, c->st);
    tord.resize(n);
    CK(cudaMemcpyAsync(tord.data(), dtord.p, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int t = std::min(c->lmax, max_t_order);
    for (int i = 0; i < n; i++)
        if (outside(i)) t = std::max(t, tord[i]);
    if (t > 200) {
        set_err("t_matrix_order above 200 is not supported");
        return MSTMG_ERR_UNSUPPORTED;
    }
    *T = t;
    return MSTMG_OK;
}

// Constant tables of a regular translation from source orders <= Ls to target
// orders <= Tt (the vcc_const combination of axialtrancoefinit, modules:1680-1722,
// the recurrence factors of axialtrancoefrecurrence up to max(Tt, Ls), and bcof(n,n)).
struct RegTables {
    DevBuf<double> vcc, f1, f2, f3, bcd;
    int vcT = 0, vcML = 0, FN = 0;
};
static int build_reg_tables(mstmg_ctx* c, int Tt, int Ls, RegTables& r)
{
    mstmg::Tables& big = big_tables();
    std::vector<double> vcc((size_t)Tt * Ls * (Ls + 2) * (Tt + Ls + 1), 0.0), vc1(2 * (Tt + Ls) + 4), vc2(2 * (Tt + Ls) + 4);
    for (int nn = 1; nn <= Tt; nn++)
        for (int l = 1; l <= Ls; l++) {
            double c1 = big.fnr[nn + nn + 1] * big.fnr[l + l + 1];
            big.vcfunc(-1, nn, 1, l, vc2.data());
            int wmin = std::abs(nn - l), wmax = nn + l, nlmin = std::min(l, nn);
            for (int m = -nlmin; m <= nlmin; m++) {
                int ml = l * (l + 1) + m;
                double c2 = -c1 * ((m & 1) ? -1.0 : 1.0);
                big.vcfunc(-m, nn, m, l, vc1.data());
                for (int w = wmin; w <= wmax; w++) {
                    int e = ((nn - l + w) % 4 + 4) % 4;
                    double ri = (e == 0 || e == 1) ? 1.0 : -1.0;
                    vcc[(size_t)(nn - 1) + (size_t)Tt * ((size_t)(ml - 1) + (size_t)Ls * (Ls + 2) * w)] = c2 * vc1[w] * vc2[w] * ri;
                }
            }
        }
    const int FN = std::max(Tt, Ls);
    size_t nf = (size_t)(2 * FN + 1) * FN;
    std::vector<double> f1(nf, 0.0), f2(nf, 0.0), f3(nf, 0.0);
    const std::vector<double>& fr = big.fnr;
    for (int m = -FN; m <= FN; m++)
        for (int l = std::max(1, std::abs(m)); l <= FN; l++) {
            size_t ix = (size_t)(m + FN) + (2 * FN + 1) * (size_t)(l - 1);
            int lp1 = l + 1, lm1 = l - 1;
            f1[ix] = fr[lm1] * fr[lp1] * fr[l - m] * fr[l + m] / fr[lm1 + l] / fr[l + lp1] / (double)l;
            f2[ix] = (double)m / (double)l / (double)lp1;
            f3[ix] = fr[l] * fr[l + 2] * fr[lp1 - m] * fr[lp1 + m] / fr[l + lp1] / fr[l + l + 3] / (double)lp1;
        }
    std::vector<double> bd(Tt + Ls + 4);
    for (int k = 0; k < (int)bd.size(); k++) bd[k] = big.bc(k, k);
    auto up = [&](DevBuf<double>& d, const std::vector<double>& h) -> int {
        CK(d.alloc(h.size()));
        CK(cudaMemcpyAsync(d.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->st));
        return MSTMG_OK;
    };
    int rc;
    if ((rc = up(r.vcc, vcc)) || (rc = up(r.f1, f1)) || (rc = up(r.f2, f2)) || (rc = up(r.f3, f3)) || (rc = up(r.bcd, bd))) return rc;
    // the host vectors are freed on return: wait for the copies
    CK(cudaStreamSynchronize(c->st));
    r.vcT = Tt;
    r.vcML = Ls * (Ls + 2);
    r.FN = FN;
    return MSTMG_OK;
}

static MergeArgs merge_args(mstmg_ctx* c, const RegTables& rt, const BigTablesDev& bt, const double* r0, const int* dtord)
{
    MergeArgs ma;
    ma.mode = 0;
    ma.out = nullptr;
    ma.ldo = 0;
    ma.nsph = c->n;
    ma.pos = c->pos.p;
    ma.order = c->d_order.p;
    ma.offset = c->d_offset.p;
    ma.tord = dtord;
    ma.r0[0] = r0[0];
    ma.r0[1] = r0[1];
    ma.r0[2] = r0[2];
    ma.rimed_re = c->opts.medium_re;
    ma.rimed_im = c->opts.medium_im;
    ma.vcc = rt.vcc.p;
    ma.vcT = rt.vcT;
    ma.vcML = rt.vcML;
    ma.fnm1 = rt.f1.p;
    ma.fnc = rt.f2.p;
    ma.fnp1 = rt.f3.p;
    ma.fcN = rt.FN;
    ma.fnr = bt.fnr.p;
    ma.bcofd = rt.bcd.p;
    ma.active = c->hs.on() ? c->hs.d_outside.p : nullptr;
    return ma;
}

extern "C" int mstmg_scattering(mstmg_ctx* c, const double* amnp, double trans_eps, int max_t_order, int nangles, double* smat,
                                double* g, int* t_matrix_order, double* amnp0, int amnp0_cap)
{
    if (int rc0 = reject_ensemble(c, "mstmg_scattering")) return rc0;
    NvtxRange nvtx_("mstmg_scattering");
    if (!c || !amnp || nangles < 2 || max_t_order < 1) {
        set_err("mstmg_scattering: bad arguments");
        return MSTMG_ERR_ARG;
    }
    const int n = c->n, L = c->lmax;
    BigTablesDev bt;
    int rc = upload_big(c, bt);
    if (rc) return rc;
    double r0[3];
    DevBuf<int> dtord;
    std::vector<int> tord;
    int T = 0;
    if ((rc = origin_orders(c, bt, trans_eps, max_t_order, r0, dtord, tord, &T))) return rc;
    RegTables rt;
    if ((rc = build_reg_tables(c, T, L, rt))) return rc;
    // merge to the common origin
    const int ne = c->neqns, nb0 = 2 * T * (T + 2);
    DevBuf<zd> dsrc, da0, mscr;
    CK(dsrc.alloc(2 * (size_t)ne));
    CK(copy_in(dsrc.p, amnp, sizeof(zd) * 2 * (size_t)ne, c->st));
    CK(da0.alloc(2 * (size_t)nb0));
    CK(cudaMemsetAsync(da0.p, 0, sizeof(zd) * 2 * (size_t)nb0, c->st));
    int grid = std::min(n, c->nsm * 2);
    size_t stride = merge_scratch_per_cta(T, L);
    CK(mscr.alloc((size_t)grid * stride));
    MergeArgs ma = merge_args(c, rt, bt, r0, dtord.p);
    ma.T = T;
    ma.amnp = dsrc.p;
    ma.ld = ne;
    ma.npol = 2;
    ma.amnp0 = da0.p;
    ma.ld0 = nb0;
    ma.scratch = mscr.p;
    ma.scratch_stride = stride;
    launch_merge(ma, grid, c->st);
    CK(cudaGetLastError());
    // GSF expansion and scattering matrix
    const int W = 2 * T + 1;
    DevBuf<double> ds, fscr, cscr, dsm;
    CK(ds.alloc(4 * 16 * (size_t)W));
    CK(cudaMemsetAsync(ds.p, 0, sizeof(double) * 4 * 16 * (size_t)W, c->st));
    CK(fscr.alloc(fosm_scratch_doubles(T)));
    launch_fosm(T, da0.p, bt.bc.p, bt.fnr.p, bt.nbc, ds.p, ds.p + 16 * W, ds.p + 32 * W, ds.p + 48 * W, fscr.p, c->st);
    CK(cscr.alloc(fosmcalc_scratch_doubles(T, nangles)));
    CK(dsm.alloc(16 * (size_t)nangles));
    launch_fosmcalc(T, nangles, ds.p, ds.p + 16 * W, ds.p + 32 * W, ds.p + 48 * W, bt.fnr.p, rt.bcd.p, cscr.p, dsm.p, c->st);
    CK(cudaGetLastError());
    double s0[2];
    CK(cudaMemcpyAsync(&s0[0], ds.p + 0, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&s0[1], ds.p + 16, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    if (smat) CK(copy_out(smat, dsm.p, sizeof(double) * 16 * (size_t)nangles, c->st));
    if (amnp0 && amnp0_cap >= nb0) CK(copy_out(amnp0, da0.p, sizeof(zd) * 2 * (size_t)nb0, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (g) *g = s0[1] / (3.0 * s0[0]);
    if (t_matrix_order) *t_matrix_order = T;
    return check_kernel_err(c);
}

extern "C" int mstmg_gsf_coefficients(mstmg_ctx* c, int t_matrix_order, const double* amnp0, double* coef)
{
    const int T = t_matrix_order;
    if (!c || !amnp0 || !coef || T < 1 || T > 200) {
        set_err("mstmg_gsf_coefficients: bad arguments");
        return MSTMG_ERR_ARG;
    }
    BigTablesDev bt;
    int rc = upload_big(c, bt);
    if (rc) return rc;
    const size_t nb0 = 2 * (size_t)T * (T + 2);
    const int W = 2 * T + 1;
    DevBuf<zd> da0;
    DevBuf<double> ds, fscr;
    CK(da0.alloc(2 * nb0));
    CK(copy_in(da0.p, amnp0, sizeof(zd) * 2 * nb0, c->st));
    CK(ds.alloc(4 * 16 * (size_t)W));
    CK(cudaMemsetAsync(ds.p, 0, sizeof(double) * 4 * 16 * (size_t)W, c->st));
    CK(fscr.alloc(fosm_scratch_doubles(T)));
    launch_fosm(T, da0.p, bt.bc.p, bt.fnr.p, bt.nbc, ds.p, ds.p + 16 * W, ds.p + 32 * W, ds.p + 48 * W, fscr.p, c->st);
    CK(cudaGetLastError());
    CK(copy_out(coef, ds.p, sizeof(double) * 4 * 16 * (size_t)W, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_kernel_err(c);
}

extern "C" int mstmg_scattering_plane(mstmg_ctx* c, int t_matrix_order, const double* amnp0, int ldim, int udim, double amin, double amax,
                                      double alpha, int rotate_plane, double* sm)
{
    const int T = t_matrix_order;
    if (!c || !amnp0 || !sm || T < 1 || udim <= ldim) {
        set_err("mstmg_scattering_plane: bad arguments");
        return MSTMG_ERR_ARG;
    }
    if (T > PS_TMAX) {
        set_err("mstmg_scattering_plane: t_matrix_order above 200 is not supported");
        return MSTMG_ERR_UNSUPPORTED;
    }
    mstmg::Tables& big = big_tables();
    std::vector<double> bd(T + 1);
    for (int k = 0; k <= T; k++) bd[k] = big.bc(k, k);
    const size_t nb0 = 2 * (size_t)T * (T + 2);
    const int nang = udim - ldim + 1;
    DevBuf<double> dfnr, dbd, dsm;
    DevBuf<zd> da0;
    CK(dfnr.alloc(2 * T + 2));
    CK(dbd.alloc(T + 1));
    CK(da0.alloc(2 * nb0));
    CK(dsm.alloc(16 * (size_t)nang));
    CK(cudaMemcpyAsync(dfnr.p, big.fnr.data(), sizeof(double) * (2 * T + 2), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(dbd.p, bd.data(), sizeof(double) * (T + 1), cudaMemcpyHostToDevice, c->st));
    CK(copy_in(da0.p, amnp0, sizeof(zd) * 2 * nb0, c->st));
    PlaneSmArgs a;
    a.T = T;
    a.a0 = da0.p;
    a.ldim = ldim;
    a.udim = udim;
    a.amin = amin;
    a.amax = amax;
    a.alpha = alpha;
    a.rotate = rotate_plane ? 1 : 0;
    a.rimed_re = c->opts.medium_re;
    a.fnr = dfnr.p;
    a.bcofd = dbd.p;
    a.smat = dsm.p;
    launch_planesm(a, c->st);
    CK(cudaGetLastError());
    CK(copy_out(sm, dsm.p, sizeof(double) * 16 * (size_t)nang, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_kernel_err(c);
}

extern "C" int mstmg_t_matrix_order(mstmg_ctx* c, double trans_eps, int max_t_order, int* t_matrix_order)
{
    if (int rc0 = reject_ensemble(c, "mstmg_t_matrix_order")) return rc0;
    if (!c || max_t_order < 1 || !t_matrix_order) {
        set_err("mstmg_t_matrix_order: bad arguments");
        return MSTMG_ERR_ARG;
    }
    BigTablesDev bt;
    int rc = upload_big(c, bt);
    if (rc) return rc;
    double r0[3];
    DevBuf<int> dtord;
    int T = 0;
    if ((rc = origin_orders(c, bt, trans_eps, max_t_order, r0, dtord, c->tord, &T))) {
        c->tord.clear();
        return rc;
    }
    *t_matrix_order = T;
    return MSTMG_OK;
}

extern "C" int mstmg_tmatrix(mstmg_ctx* c, int t_matrix_order, double solution_eps, double convergence_eps, int max_iterations,
                             double* tmat, double* sphere_qeff, double* qtot, int* order_used, int* maxiter, double* maxerr)
{
    if (int rc0 = reject_ensemble(c, "mstmg_tmatrix")) return rc0;
    if (c && c->hs.on() && c->opts.precision == MSTMG_PRECISION_MIXED && c->opts.mixed_solver != 2) {
        set_err("mstmg_tmatrix: with spheres inside other spheres the columns are solved by the FP64 BiCG or the mixed GMRES "
                "(mixed_solver 2)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    if (int rc1 = reject_sharded(c, "mstmg_tmatrix")) return rc1;
    NvtxRange nvtx_("mstmg_tmatrix");
    if (!c || t_matrix_order < 1 || t_matrix_order > 200 || !tmat || max_iterations < 1) {
        set_err("mstmg_tmatrix: bad arguments (1 <= t_matrix_order <= 200, max_iterations >= 1, tmat required)");
        return MSTMG_ERR_ARG;
    }
    if ((int)c->tord.size() != c->n) {
        set_err("mstmg_tmatrix: call mstmg_t_matrix_order first (it sets the translation orders)");
        return MSTMG_ERR_ARG;
    }
    const bool mixed = c->opts.precision == MSTMG_PRECISION_MIXED;
    int rc = ensure_ops_both(c, true, mixed, false);
    if (rc) return rc;
    const int n = c->n, L = c->lmax, ne = c->neqns, TM = t_matrix_order;
    // With the tensor-core pass serving the mixed GMRES, the columns of
    // several consecutive orders are solved together (up to TM_GROUP columns)
    // so that the pass's 128-column tiles fill; the orders of a group are then
    // post-processed one by one as the reference's loop over l does
    // (solver:141-318), and the order at which the extinction converges ends
    // the loop there (later orders of its group are dropped unused).
    const bool grouped = mixed && c->opts.mixed_solver == 2 && tc_eligible(c);
    const int TM_GROUP = 256;
    auto cols_of = [](int q) { return 2 * (2 * q + 1); };
    const int nblkt = 2 * TM * (TM + 2), Sord = cols_of(TM), Smax = grouped ? std::max(Sord, TM_GROUP) : Sord;
    BigTablesDev bt;
    if ((rc = upload_big(c, bt))) return rc;
    // the cluster origin: the mean of the spheres outside every other (input:1166-1177)
    double r0[3] = {0.0, 0.0, 0.0};
    int nout = 0;
    for (int i = 0; i < n; i++)
        if (!c->hs.on() || c->hs.host[i] < 0) {
            nout++;
            for (int k = 0; k < 3; k++) r0[k] = r0[k] + c->hpos[3 * (size_t)i + k];
        }
    for (int k = 0; k < 3; k++) r0[k] = r0[k] / (double)nout;
    DevBuf<int> dtord;
    CK(dtord.alloc(n));
    CK(cudaMemcpyAsync(dtord.p, c->tord.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
    RegTables rtm, rtd;   // merge: spheres -> origin; distribute: origin -> spheres
    if ((rc = build_reg_tables(c, TM, L, rtm)) || (rc = build_reg_tables(c, L, TM, rtd))) return rc;
    const int grid = std::min(n, c->nsm * 2);
    const size_t strm = merge_scratch_per_cta(TM, L), strd = merge_scratch_per_cta(L, TM);
    DevBuf<zd> mscr, P0, PK, B64, A0, dT, X64;
    DevBuf<double> qcol, dsq, qsum, rr;
    DevBuf<zf> B32;
    DevBuf<int> idx;
    CK(mscr.alloc((size_t)grid * merge_chunks(Sord) * std::max(strm, strd)));
    CK(P0.alloc((size_t)2 * TM * (TM + 2) * Sord));
    CK(A0.alloc((size_t)2 * TM * (TM + 2) * Sord));
    CK(PK.alloc((size_t)ne * Smax));
    CK(B64.alloc((size_t)ne * Smax));
    CK(dT.alloc((size_t)nblkt * nblkt));
    CK(cudaMemsetAsync(dT.p, 0, sizeof(zd) * (size_t)nblkt * nblkt, c->st));
    CK(qcol.alloc((size_t)3 * n * Sord));
    CK(dsq.alloc((size_t)3 * n));
    CK(cudaMemsetAsync(dsq.p, 0, sizeof(double) * 3 * n, c->st));
    CK(qsum.alloc(3));
    MultiWork<double> w64;
    MultiWork<float> w32;
    if ((rc = w64.init(Smax, ne, c->nsm, !mixed))) return rc;
    GmresWork& gw = c->tm_gm;
    if (mixed && c->opts.mixed_solver == 2 && !(gw.hh && gw.ne == ne && gw.S >= Smax) &&
        (rc = gw.setup(Smax, ne, c->opts.gmres_restart, "mstmg_tmatrix")))
        return rc;
    if (mixed) {
        CK(X64.alloc((size_t)ne * Smax));
        if (c->opts.mixed_solver != 2) {   // FP32 BiCG work
            if ((rc = w32.init(Smax, ne, c->nsm, true))) return rc;
            CK(B32.alloc((size_t)ne * Smax));
            CK(rr.alloc(2 * (size_t)Smax));
            CK(idx.alloc(2 * (size_t)Smax));
        }
    }
    zd* X = mixed ? X64.p : w64.v(ne).X;
    SlotMaps sm = c->sm();
    const zd rimed = mk(c->opts.medium_re, c->opts.medium_im);
    int istat = 0, mit = 0, used = TM, outer_total = 0;
    double merr = 0.0, qold = 0.0, hq[3] = {0.0, 0.0, 0.0};
    bool done = false;
    for (int la = 1; la <= TM && !done;) {
        int lb = la, Sg = cols_of(la);
        while (grouped && lb < TM && Sg + cols_of(lb + 1) <= TM_GROUP) Sg += cols_of(++lb);
        // right-hand sides: unit TE/TM fields of orders la..lb at the origin,
        // distributed to the spheres, one order after the other in the columns
        CK(cudaMemsetAsync(PK.p, 0, sizeof(zd) * (size_t)ne * Sg, c->st));
        for (int q = la, col0 = 0; q <= lb; col0 += cols_of(q), q++) {
            launch_tm_rhs(q, P0.p, c->st);
            MergeArgs md = merge_args(c, rtd, bt, r0, dtord.p);
            md.mode = 1;
            md.out = PK.p + (size_t)col0 * ne;
            md.ldo = ne;
            md.T = q;
            md.amnp = P0.p;
            md.ld = 2 * q * (q + 2);
            md.npol = cols_of(q);
            md.amnp0 = nullptr;
            md.ld0 = 0;
            md.scratch = mscr.p;
            md.scratch_stride = strd;
            launch_merge(md, grid, c->st);
        }
        // b = Mie f, initial guess b (solver:185-187); the grouped mixed
        // GMRES starts from zero instead, whose residual b needs no FP64 pass
        // (the Krylov space holds b after the first step)
        if (c->hs.on())
            for (int k = 0; k < Sg; k++) mie_all<double>(c, 1, 0, PK.p + (size_t)k * ne, B64.p + (size_t)k * ne);
        else
            launch_m_mie(sm, c->an.p, ne, Sg, PK.p, B64.p, c->st);
        if (grouped) CK(cudaMemsetAsync(X, 0, sizeof(zd) * (size_t)ne * Sg, c->st));
        else CK(cudaMemcpyAsync(X, B64.p, sizeof(zd) * (size_t)ne * Sg, cudaMemcpyDeviceToDevice, c->st));
        CK(cudaGetLastError());
        std::vector<int> its;
        std::vector<double> errs;
        std::vector<int> sts;
        if (mixed) {
            int oc = 0;
            if (c->opts.mixed_solver == 1)
                rc = solve_multi_mixed(c, w64, w32, B32, rr, idx, Sg, B64.p, X, solution_eps, max_iterations, its, errs, sts, &oc);
            else if (c->opts.mixed_solver == 2)
                rc = solve_multi_gmres(c, w64, gw, Sg, B64.p, X, solution_eps, max_iterations, its, errs, sts, &oc, nullptr, grouped);
            else
                rc = solve_multi_rr(c, w64, w32, rr, idx, Sg, B64.p, X, solution_eps, max_iterations, its, errs, sts, &oc);
            outer_total += oc;
        } else {
            std::vector<int> sys(Sg);
            for (int k = 0; k < Sg; k++) sys[k] = k;
            std::vector<double> ev(Smax, solution_eps);
            w64.S = Smax;
            rc = bicg_multi<double>(c, w64, B64.p, sys, true, max_iterations, ev, its, errs, sts);
        }
        if (rc) return rc;
        for (int q = la, col0 = 0; q <= lb; col0 += cols_of(q), q++) {
            const int S = cols_of(q), nb = 2 * q * (q + 2);
            for (int k = col0; k < col0 + S; k++) {
                mit = std::max(mit, its[k]);
                merr = std::max(merr, errs[k]);
                if (its[k] > max_iterations || errs[k] > solution_eps || sts[k] == 2) istat = 1;
            }
            zd* Xq = X + (size_t)col0 * ne;
            // per-sphere efficiencies of every column, summed; with host
            // spheres the exciting fields are the interaction without the Mie
            // multiply plus the incident field (qefficiencyfactors), in B64
            const zd* G = nullptr;
            if (c->hs.on()) {
                if ((rc = translate_many<double>(c, Xq, B64.p, S, 0u))) return rc;
                launch_add_correction_d(S * ne, B64.p, PK.p + (size_t)col0 * ne, c->st);
                G = B64.p;
            }
            launch_tm_qeff(n, S, c->d_order.p, c->d_offset.p, c->d_mie_offset.p, c->rad.p, rimed, c->an_inv.p, Xq, PK.p + (size_t)col0 * ne,
                           ne, qcol.p, c->st, G, c->hs.on() ? c->hs.d_rext.p : nullptr);
            launch_tm_qsum(n, S, qcol.p, c->rad.p, c->xg, dsq.p, qsum.p, c->st);
            // merge the solutions to the origin: T-matrix columns of order q
            CK(cudaMemsetAsync(A0.p, 0, sizeof(zd) * (size_t)nb * S, c->st));
            MergeArgs mm = merge_args(c, rtm, bt, r0, dtord.p);
            mm.T = q;
            mm.amnp = Xq;
            mm.ld = ne;
            mm.npol = S;
            mm.amnp0 = A0.p;
            mm.ld0 = nb;
            mm.scratch = mscr.p;
            mm.scratch_stride = strm;
            launch_merge(mm, grid, c->st);
            launch_tm_store(q, TM, A0.p, dT.p, c->st);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(hq, qsum.p, sizeof(double) * 3, cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
            double converr = hq[0] - qold;
            qold = hq[0];
            if (convergence_eps > 0.0 && converr < convergence_eps) {
                used = q;
                done = true;
                break;
            }
        }
        la = lb + 1;
    }
    c->outer = outer_total;
    CK(copy_out(tmat, dT.p, sizeof(zd) * (size_t)nblkt * nblkt, c->st));
    if (sphere_qeff) CK(copy_out(sphere_qeff, dsq.p, sizeof(double) * 3 * n, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (qtot) {
        qtot[0] = hq[0];
        qtot[1] = hq[1];
        qtot[2] = hq[0] + hq[2] - hq[1];   // qtotcalc: Qsca = Qext + Qinc - Qabs
    }
    if (order_used) *order_used = used;
    if (maxiter) *maxiter = mit;
    if (maxerr) *maxerr = merr;
    rc = check_kernel_err(c);
    if (rc) return rc;
    return istat ? MSTMG_NOT_CONVERGED : MSTMG_OK;
}

extern "C" int mstmg_tmatrix_qext_qsca(mstmg_ctx* c, int t_matrix_order, const double* tmat, double* qext, double* qsca)
{
    if (!c || t_matrix_order < 1 || t_matrix_order > 200 || !tmat) {
        set_err("mstmg_tmatrix_qext_qsca: bad arguments");
        return MSTMG_ERR_ARG;
    }
    const size_t nblkt = 2 * (size_t)t_matrix_order * (t_matrix_order + 2);
    DevBuf<zd> dT;
    DevBuf<float> tc;
    DevBuf<double> out;
    CK(dT.alloc(nblkt * nblkt));
    CK(tc.alloc(2 * nblkt * nblkt));
    CK(out.alloc(2));
    CK(copy_in(dT.p, tmat, sizeof(zd) * nblkt * nblkt, c->st));
    launch_tm_qext_qsca(t_matrix_order, dT.p, c->xg, tc.p, out.p, c->st);
    CK(cudaGetLastError());
    double h[2];
    CK(cudaMemcpyAsync(h, out.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (qext) *qext = h[0];
    if (qsca) *qsca = h[1];
    return MSTMG_OK;
}

extern "C" int mstmg_ranorient_scattering(mstmg_ctx* c, int t_matrix_order, const double* tmat, int nangles, double* sm, double* smcf,
                                          double* smat)
{
    NvtxRange nvtx_("mstmg_ranorient_scattering");
    const int T = t_matrix_order;
    if (!c || T < 1 || T > 60 || !tmat || (nangles > 0 && nangles < 2)) {
        set_err("mstmg_ranorient_scattering: bad arguments (1 <= t_matrix_order <= 60, nangles 0 or >= 2)");
        return MSTMG_ERR_ARG;
    }
    BigTablesDev bt;
    int rc = upload_big(c, bt);
    if (rc) return rc;
    const size_t nblkt = 2 * (size_t)T * (T + 2);
    const int W = 2 * T + 1;
    DevBuf<zd> dT, trace, dm, dmcf, fm;
    DevBuf<float2> tc;
    DevBuf<double> dsm, dsmat, vscr, dscr, dbcd;
    CK(dT.alloc(nblkt * nblkt));
    CK(copy_in(dT.p, tmat, sizeof(zd) * nblkt * nblkt, c->st));
    CK(tc.alloc(nblkt * nblkt));
    CK(trace.alloc(4 * (size_t)T));
    CK(dm.alloc(ro_dm_elems(T)));
    CK(dmcf.alloc(ro_dm_elems(T)));
    CK(cudaMemsetAsync(dm.p, 0, sizeof(zd) * ro_dm_elems(T), c->st));
    CK(cudaMemsetAsync(dmcf.p, 0, sizeof(zd) * ro_dm_elems(T), c->st));
    CK(fm.alloc((size_t)W * 2 * 3 * T * 2 * T * 2));
    CK(dsm.alloc(2 * 16 * (size_t)W));
    CK(vscr.alloc(ro_vscr_doubles(T, c->nsm)));
    const int nang = nangles > 0 ? nangles : 1;
    CK(dscr.alloc((size_t)nang * (16 * (2 * T) + 40)));
    CK(dsmat.alloc(16 * (size_t)nang));
    std::vector<double> bd(2 * T + 4);
    for (int k = 0; k < (int)bd.size(); k++) bd[k] = big_tables().bc(k, k);
    CK(dbcd.alloc(bd.size()));
    CK(cudaMemcpyAsync(dbcd.p, bd.data(), sizeof(double) * bd.size(), cudaMemcpyHostToDevice, c->st));
    RoArgs a;
    a.nodr = T;
    a.tc = tc.p;
    a.trace = trace.p;
    a.dm = dm.p;
    a.dmcf = dmcf.p;
    a.fm = fm.p;
    a.sm = dsm.p;
    a.smcf = dsm.p + 16 * W;
    a.bcof = bt.bc.p;
    a.fnr = bt.fnr.p;
    a.nbc = bt.nbc;
    a.vscr = vscr.p;
    a.rimed_re = c->opts.medium_re;
    if (launch_ranorient(a, dT.p, nangles, dbcd.p, dscr.p, dsmat.p, c->nsm, c->st) != 0) {
        set_err("mstmg_ranorient_scattering: t_matrix_order too large for the shared-memory layout");
        return MSTMG_ERR_UNSUPPORTED;
    }
    CK(cudaGetLastError());
    if (sm) CK(copy_out(sm, dsm.p, sizeof(double) * 16 * W, c->st));
    if (smcf) CK(copy_out(smcf, dsm.p + 16 * W, sizeof(double) * 16 * W, c->st));
    if (smat && nangles > 0) CK(copy_out(smat, dsmat.p, sizeof(double) * 16 * (size_t)nangles, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_kernel_err(c);
}

