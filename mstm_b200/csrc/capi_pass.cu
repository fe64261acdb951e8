// capi_pass.cu -- the pair operators and the translation passes behind the C
// ABI: operator generation, the rotation kernels (tiled / order-generic), the
// tensor-core pass of many columns, the FFT path (node_selection, the kernel
// spectra and fft_external_to_external_expansion), sphereinteraction and the
// translation-pass entry points.
#include "ctx.cuh"

// ---------------------------------------------------------------------------
// operators and the translation pass
// ---------------------------------------------------------------------------
// Generate the stored pair operators.  want64 / want32 select the FP64 and
// FP32 records; both come out of one pass of the generator when both are due.
DenseArgs dense_args(mstmg_ctx* c)
{
    DenseArgs d;
    d.npairs = c->ndense;
    d.pairs = c->dpairs.p;
    d.order = c->d_order.p;
    d.offset = c->d_offset.p;
    d.pos = c->pos.p;
    d.off = c->doff.p;
    d.rec64 = nullptr;
    d.rec32 = nullptr;
    d.rimed_re = c->opts.medium_re;
    d.rimed_im = c->opts.medium_im;
    d.pmed = c->hs.on() ? c->hs.dmed.p : nullptr;
    d.g.tc = c->gt_tc.p;
    d.g.nmax = c->gt_nmax;
    d.g.nd = c->gt_nmax * (c->gt_nmax + 2);
    d.g.fnr = c->gt_fnr.p;
    d.g.bcd = c->gt_bcd.p;
    return d;
}

int ensure_ops_both(mstmg_ctx* c, bool want64, bool want32, bool force)
{
    if (c->npairs == 0 && c->ndense == 0) return MSTMG_OK;
    bool need64 = want64 && (force || !c->ops64_ready);
    bool need32 = want32 && (force || !c->ops32_ready);
    if (!need64 && !need32) return MSTMG_OK;
    if (c->ndense > 0) {
        DenseArgs d = dense_args(c);
        const void* was[2] = {c->dop64.p, c->dop32.p};
        if (need64) {
            CK(c->dop64.alloc(c->dense_units));
            d.rec64 = c->dop64.p;
        }
        if (need32) {
            CK(c->dop32.alloc(c->dense_units));
            d.rec32 = c->dop32.p;
        }
        if (was[0] != c->dop64.p || was[1] != c->dop32.p) c->layout_gen++;
        launch_dense_gen(d, c->st);
        CK(cudaGetLastError());
    }
    if (c->npairs == 0) {
        if (need64) c->ops64_ready = true;
        if (need32) c->ops32_ready = true;
        return MSTMG_OK;
    }
    {
        const void* was[2] = {c->op64.p, c->op32.p};
        if (need64) CK(c->op64.alloc(c->op_units));
        if (need32) CK(c->op32.alloc(c->row32 ? (long long)c->npairs * c->row32 : c->op_units));
        if (was[0] != c->op64.p || was[1] != c->op32.p) c->layout_gen++;
        // row records: the padding of every row reads as zero
        if (need32 && c->row32) CK(cudaMemsetAsync(c->op32.p, 0, sizeof(float) * (size_t)c->npairs * c->row32, c->st));
    }
    NvtxRange nvtx_("pair operator generation");
    OpGenArgs a;
    a.npairs = c->npairs;
    a.pairs = c->pairs.p;
    a.pos = c->pos.p;
    a.order = c->d_order.p;
    a.opoff = c->opoff.p;
    a.op64 = need64 ? c->op64.p : nullptr;
    a.op32 = need32 ? c->op32.p : nullptr;
    a.row32 = c->row32;
    a.vcc = c->vcc.p;
    a.vnmax = c->vn;
    a.fnr = c->fnr.p;
    a.rfnr = c->rfnr.p;
    a.bcofd = c->bcofd.p;
    a.rimed_re = c->opts.medium_re;
    a.rimed_im = c->opts.medium_im;
    a.pmed = c->hs.on() ? c->hs.pmed.p : nullptr;
    a.err = c->err.p;
    CK(c->opgen_xi.alloc(opgen_xi_scratch(std::max(c->npairs, c->hs.nhp))));
    a.xi = c->opgen_xi.p;
    launch_opgen(a, c->nsm, c->st);
    CK(cudaGetLastError());
    if ((need64 || need32) && c->hs.nhp > 0) {
        // regular translations between hosts and the spheres they hold, in
        // the host's index (external_to_internal_expansion, modules:6579-6592)
        HostSpheres& h = c->hs;
        if (need64) CK(h.hop64.alloc(h.hunits));
        if (need32) CK(h.hop32.alloc(h.hunits));
        OpGenArgs b = a;
        b.npairs = h.nhp;
        b.pairs = h.hpairs.p;
        b.pos = h.xpos.p;
        b.opoff = h.hopoff.p;
        b.op64 = need64 ? h.hop64.p : nullptr;
        b.op32 = need32 ? h.hop32.p : nullptr;
        b.row32 = 0;
        b.pmed = h.hmed.p;
        b.regular = 1;
        launch_opgen(b, c->nsm, c->st);
        CK(cudaGetLastError());
        if (need64) h.hops_ready = true;
        if (need32) h.hops32_ready = true;
    }
    if (need64) c->ops64_ready = true;
    if (need32) c->ops32_ready = true;
    return MSTMG_OK;
}

// y[:, 0:nrhs] += the host-sphere couplings of x (external_to_internal_expansion)
template <typename T> int translate_hosts(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int nrhs, unsigned contran)
{
    HostSpheres& h = c->hs;
    if (!h.on()) return MSTMG_OK;
    if (h.nhp > 0) {
        if (sizeof(T) == 8 ? !h.hops_ready : !h.hops32_ready) {
            set_err("internal error: host-sphere operators not generated");
            return MSTMG_ERR_ARG;
        }
        TransArgs<T> a;
        a.npairs = h.nhp;
        a.pairs = h.hpairs.p;
        a.order = c->d_order.p;
        a.offset = c->d_offset.p;
        a.ops = sizeof(T) == 8 ? (const T*)h.hop64.p : (const T*)h.hop32.p;
        a.opoff = h.hopoff.p;
        a.x = x;
        a.y = y;
        a.ld = c->neqns;
        a.nrhs = nrhs;
        a.contran = contran;
        a.lmax = h.hlmax;
        a.maxrec = h.hmaxrec;
        a.err = c->err.p;
        launch_translate<T>(a, c->nsm, c->st);
    }
    launch_mtransfer<T>(h.nzp, h.zpairs.p, c->d_order.p, c->d_offset.p, x, y, c->neqns, nrhs, c->st);
    CK(cudaGetLastError());
    return MSTMG_OK;
}
template int translate_hosts<double>(mstmg_ctx*, const zd*, zd*, int, unsigned);
template int translate_hosts<float>(mstmg_ctx*, const zf*, zf*, int, unsigned);

template <typename T> void mie_all(mstmg_ctx* c, int idir, int conj_in, const cpx<T>* x, cpx<T>* y)
{
    SlotMaps sm = c->sm();
    const bool d = sizeof(T) == 8;
    const cpx<T>* an = d ? (const cpx<T>*)c->an.p : (const cpx<T>*)c->an32.p;
    if (c->hs.on()) {
        const HostSpheres& h = c->hs;
        launch_hmie<T>(sm.nslots, c->n, sm.slot, sm.order, sm.offset, sm.mie_offset, h.d_hoff.p, an,
                       d ? (const cpx<T>*)h.dn.p : (const cpx<T>*)h.dn32.p, d ? (const cpx<T>*)h.un.p : (const cpx<T>*)h.un32.p,
                       d ? (const cpx<T>*)h.vn.p : (const cpx<T>*)h.vn32.p, idir, conj_in, x, y, c->st);
    } else {
        launch_mie<T>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, an, idir, conj_in, x, y, c->st);
    }
}
template void mie_all<double>(mstmg_ctx*, int, int, const zd*, zd*);
template void mie_all<float>(mstmg_ctx*, int, int, const zf*, zf*);

int ensure_ops(mstmg_ctx* c, int prec, bool force) { return ensure_ops_both(c, prec == 0, prec == 1, force); }

template <typename T> static const T* ops_ptr(mstmg_ctx* c);
template <> const double* ops_ptr<double>(mstmg_ctx* c) { return c->op64.p; }
template <> const float* ops_ptr<float>(mstmg_ctx* c) { return c->op32.p; }

// FP32 passes on row records: the row kernel, in groups of 4, 2 or 1 columns
// when the pass has another column count (the records fit no other kernel)
template <typename T> static int rows_pass(mstmg_ctx*, const TiledArgs<T>&, int, int, unsigned) { return -1; }
template <> int rows_pass<float>(mstmg_ctx* c, const TiledArgs<float>& tf, int nrhs, int nchunk, unsigned contran)
{
    if (rows_supported(c->tile_L, nrhs)) return launch_translate_rows(tf, c->tile_L, c->nsm, c->st);
    if (nchunk != 1) return -1;
    int rc = 0;
    for (int c0 = 0; c0 < nrhs && rc == 0;) {
        const int w = nrhs - c0 >= 4 ? 4 : (nrhs - c0 >= 2 ? 2 : 1);
        TiledArgs<float> tw = tf;
        tw.x = tf.x + (size_t)c0 * c->neqns;
        tw.y = tf.y + (size_t)c0 * c->neqns;
        tw.nrhs = w;
        tw.contran = (contran >> c0) & ((1u << w) - 1u);
        rc = launch_translate_rows(tw, c->tile_L, c->nsm, c->st);
        c0 += w;
    }
    return rc;
}

// y[:, 0:nrhs*nchunk] = H x[:, 0:nrhs*nchunk]  (y zeroed here).  nchunk > 1
// only on the tiled path: contran then applies to column r of every chunk.
template <typename T> int translate(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int nrhs, unsigned contran, int nchunk)
{
    NvtxRange nvtx_(sizeof(T) == 8 ? "translation pass FP64" : "translation pass FP32");
    CK(cudaMemsetAsync(y, 0, sizeof(cpx<T>) * (size_t)c->neqns * nrhs * nchunk, c->st));
    if (c->hs.on()) {
        if (nchunk > 1) return MSTMG_ERR_UNSUPPORTED;
        int rh = translate_hosts<T>(c, x, y, nrhs, contran);
        if (rh) return rh;
    }
    if (c->ndense > 0) {
        if (nchunk > 1) return MSTMG_ERR_UNSUPPORTED;
        const T* drec = sizeof(T) == 8 ? (const T*)c->dop64.p : (const T*)c->dop32.p;
        launch_dense_apply<T>(dense_args(c), drec, x, y, c->neqns, nrhs, contran, c->st);
        CK(cudaGetLastError());
    }
    // a sharded context: shard 0 adds the FFT path's far field, every shard its near-pair tiles
    const bool far = c->fft && c->fft->on && c->shard == 0;
    if (c->npairs == 0) return far ? fft_far<T>(c, x, y, nrhs * nchunk, contran) : MSTMG_OK;
    TransArgs<T> a;
    a.npairs = c->npairs;
    a.pairs = c->pairs.p;
    a.order = c->d_order.p;
    a.offset = c->d_offset.p;
    a.ops = ops_ptr<T>(c);
    a.opoff = c->opoff.p;
    a.x = x;
    a.y = y;
    a.ld = c->neqns;
    a.nrhs = nrhs;
    a.contran = contran;
    a.lmax = c->pair_lmax;
    a.uniform = c->pair_uniform ? 1 : 0;
    a.maxrec = c->maxrec;
    a.err = c->err.p;
    TiledArgs<T> ta;
    // FP64 passes of orders 3 and 4 run the order-generic kernel on the tile
    // ordered pairs (faster there than the rotation-tiled kernel); FP32 passes
    // take the row kernel from order 3
    bool use_tiled = c->tiled && (sizeof(T) == 4 || c->tile_L >= 5) && (tiled_supported(c->tile_L, nrhs) || (sizeof(T) == 4 && c->row32));
    if (use_tiled) {
        ta.ntiles = c->ntiles;
        ta.tiles = c->tiles.p;
        ta.pairs = c->pairs.p;
        ta.ops = ops_ptr<T>(c);
        ta.x = x;
        ta.y = y;
        ta.ld = c->neqns;
        ta.nrhs = nrhs;
        ta.nchunk = nchunk;
        ta.nsph = c->n;
        ta.contran = contran;
        ta.err = c->err.p;
        ta.ctas_per_sm = c->opts.tile_ctas_per_sm;
        ta.tsph = c->tsph.p;
        ta.pslot = c->pslot.p;
        ta.pairs_per_step = c->opts.tile_pairs;
        ta.soff = c->hs.on() ? c->d_offset.p : nullptr;
    }
    if (nchunk > 1 && !use_tiled) return MSTMG_ERR_UNSUPPORTED;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->timing) {
        for (cudaEvent_t* ev : {&e0, &e1}) {
            if (!c->ev_pool.empty()) { *ev = c->ev_pool.back(); c->ev_pool.pop_back(); }
            else CK(cudaEventCreate(ev));
        }
        CK(cudaEventRecord(e0, c->st));
    }
    if (use_tiled && sizeof(T) == 4 && c->row32) {
        const int rc = rows_pass(c, ta, nrhs, nchunk, contran);
        if (rc != 0) {
            if (e0) c->ev_pool.push_back(e0);
            if (e1) c->ev_pool.push_back(e1);
            set_err("FP32 translation pass: no row-kernel configuration for this order and column count");
            return MSTMG_ERR_UNSUPPORTED;
        }
    } else if (!use_tiled || launch_translate_tiled<T>(ta, c->tile_L, c->nsm, c->st) != 0) {
        if (nchunk > 1) {
            if (e0) c->ev_pool.push_back(e0);
            if (e1) c->ev_pool.push_back(e1);
            return MSTMG_ERR_UNSUPPORTED;
        }
        launch_translate<T>(a, c->nsm, c->st);
    }
    CK(cudaGetLastError());
    if (c->timing) {
        CK(cudaEventRecord(e1, c->st));
        c->pending.push_back({e0, e1, sizeof(T) == 8 ? 0 : 1});
    }
    if (sizeof(T) == 8) c->passes64++;
    else c->passes32++;
    if (far) return fft_far<T>(c, x, y, nrhs * nchunk, contran);
    return MSTMG_OK;
}

// Columns per chunk of FP32 tiled passes: opts.fp32_chunk when set (2 or 4),
// otherwise chosen once per context by timing one pass over the caller's
// columns in chunks of 4 and of 2 (each run twice, the second timed), which
// depends on the order and the cluster size (4 wins at L = 9, 2 at L = 8 and
// for small column counts).  The timing passes write y, which the caller's
// own pass then overwrites.
int fp32_chunk(mstmg_ctx* c, const zf* x, zf* y, int ncols, unsigned pattern2)
{
    if (c->opts.fp32_chunk == 2 || c->opts.fp32_chunk == 4) return c->opts.fp32_chunk;
    if (c->chunk32 > 0) return c->chunk32;
    if (!c->tiled || ncols < 4 || ncols % 4 != 0 || !tiled_supported(c->tile_L, 2) || !tiled_supported(c->tile_L, 4)) return 4;
    auto expand = [&](int w) {
        unsigned m = 0;
        for (int r = 0; r < w; r++)
            if ((pattern2 >> (r & 1)) & 1u) m |= 1u << r;
        return m;
    };
    cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
    for (auto& ev : e)
        if (cudaEventCreate(&ev) != cudaSuccess) {
            for (auto& f : e)
                if (f) cudaEventDestroy(f);
            return 4;
        }
    float ms[2] = {0.f, 0.f};
    const int nr[2] = {4, 2};
    const bool timing = c->timing;
    c->timing = false;
    bool ok = true;
    for (int v = 0; v < 2 && ok; v++) {
        ok = translate<float>(c, x, y, nr[v], expand(nr[v]), ncols / nr[v]) == MSTMG_OK;
        cudaEventRecord(e[0], c->st);
        ok = ok && translate<float>(c, x, y, nr[v], expand(nr[v]), ncols / nr[v]) == MSTMG_OK;
        cudaEventRecord(e[1], c->st);
        ok = ok && cudaEventSynchronize(e[1]) == cudaSuccess && cudaEventElapsedTime(&ms[v], e[0], e[1]) == cudaSuccess;
    }
    c->timing = timing;
    for (auto& f : e) cudaEventDestroy(f);
    if (!ok) return 4;
    c->passes32 -= 4;   // the timing passes are not the caller's
    c->chunk32 = ms[1] < ms[0] ? 2 : 4;
    return c->chunk32;
}

// ---------------------------------------------------------------------------
// the tensor-core pass of many FP32 columns (tcpass.cu)
// ---------------------------------------------------------------------------
// Columns from which a plain (no conjugate-transpose column) FP32 pass goes to
// the tensor cores: one M tile costs the same for 1 or 128 columns, and at 12
// columns it already beats the rotation kernel.
#define TC_MIN_COLS 12

// One sphere order (5..10), pairs translated directly (no FFT, no dense
// pairs): the cases the dense TF32 images serve.
bool tc_eligible(const mstmg_ctx* c)
{
    if (c->opts.tensor_core < 0 || c->tc_state < 0 || c->nshards > 1 || c->hs.on()) return false;
    if (!c->tiled || c->ndense > 0 || (c->fft && c->fft->on) || c->npairs == 0) return false;
    return c->lmax >= 5 && tc_geom(c->lmax).NP <= 128;
}

// Build the dense operator images of every ordered pair (both directions of
// each pair of the context's list), unless they would take more than a third
// of the free device memory (the context then keeps the rotation kernels).
int ensure_tc(mstmg_ctx* c)
{
    if (c->tc_state == 1) return MSTMG_OK;
    if (!tc_eligible(c)) return MSTMG_ERR_UNSUPPORTED;
    NvtxRange nvtx_("tensor-core operator images");
    const TcGeom g = tc_geom(c->lmax);
    std::vector<int2> pr(c->npairs);
    CK(cudaMemcpyAsync(pr.data(), c->pairs.p, sizeof(int2) * c->npairs, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    std::vector<std::vector<int>> nbr(c->n);
    for (const int2& q : pr) {
        nbr[q.x].push_back(q.y);
        nbr[q.y].push_back(q.x);
    }
    std::vector<int> rstart(c->n + 1, 0), rsrc;
    std::vector<int2> ent;
    rsrc.reserve(2 * (size_t)c->npairs);
    ent.reserve(2 * (size_t)c->npairs);
    for (int i = 0; i < c->n; i++) {
        std::sort(nbr[i].begin(), nbr[i].end());
        rstart[i] = (int)rsrc.size();
        for (int j : nbr[i]) {
            rsrc.push_back(j);
            ent.push_back(make_int2(i, j));
        }
    }
    rstart[c->n] = (int)rsrc.size();
    const size_t need = ent.size() * tc_himg_floats(g) * sizeof(float);
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    if (need > fr / 3) {
        c->tc_state = -1;
        set_err("tensor-core operator images (" + std::to_string(need >> 20) + " MiB) exceed a third of the free device memory");
        return MSTMG_ERR_UNSUPPORTED;
    }
    if (int rg = ensure_gentran(c, c->lmax)) return rg;
    const void* was = c->tc_h.p;
    CK(c->tc_h.alloc(ent.size() * tc_himg_floats(g)));
    CK(c->tc_ent.alloc(ent.size()));
    CK(c->tc_rstart.alloc(rstart.size()));
    CK(c->tc_rsrc.alloc(rsrc.size()));
    if (was != c->tc_h.p) c->layout_gen++;
    CK(cudaMemcpyAsync(c->tc_ent.p, ent.data(), sizeof(int2) * ent.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->tc_rstart.p, rstart.data(), sizeof(int) * rstart.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->tc_rsrc.p, rsrc.data(), sizeof(int) * rsrc.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemsetAsync(c->tc_h.p, 0, need, c->st));   // the padded rows and sources stay zero
    TcGenArgs a;
    a.nent = (int)ent.size();
    a.ent = c->tc_ent.p;
    a.pos = c->pos.p;
    a.geo = g;
    a.rimed_re = c->opts.medium_re;
    a.rimed_im = c->opts.medium_im;
    a.g.tc = c->gt_tc.p;
    a.g.nmax = c->gt_nmax;
    a.g.nd = c->gt_nmax * (c->gt_nmax + 2);
    a.g.fnr = c->gt_fnr.p;
    a.g.bcd = c->gt_bcd.p;
    a.himg = c->tc_h.p;
    launch_tc_gen(a, c->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->st));   // the host vectors above are freed on return
    c->tc_nent = (int)ent.size();
    c->tc_state = 1;
    return MSTMG_OK;
}

// y[:, 0:ncols] = H x[:, 0:ncols] (no conjugate-transpose columns) on the
// tensor cores; y zeroed here
int tc_translate(mstmg_ctx* c, const zf* x, zf* y, int ncols)
{
    NvtxRange nvtx_("translation pass FP32 tensor cores");
    if (int rc = ensure_tc(c)) return rc;
    const TcGeom g = tc_geom(c->lmax);
    const int nmt = (ncols + TC_M - 1) / TC_M;
    const int mtn = tc_tiles_per_cta(g, nmt);
    const void* was = c->tc_a.p;
    CK(c->tc_a.alloc((size_t)((nmt + mtn - 1) / mtn * mtn) * c->n * tc_aimg_floats(g)));
    if (was != c->tc_a.p) c->layout_gen++;
    CK(cudaMemsetAsync(y, 0, sizeof(zf) * (size_t)c->neqns * ncols, c->st));
    TcPassArgs a;
    a.nsph = c->n;
    a.geo = g;
    a.ld = c->neqns;
    a.ncols = ncols;
    a.nmt = nmt;
    a.rstart = c->tc_rstart.p;
    a.rsrc = c->tc_rsrc.p;
    a.nent = c->tc_nent;
    a.himg = c->tc_h.p;
    a.aimg = c->tc_a.p;
    a.x = x;
    a.y = y;
    a.err = c->err.p;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->timing) {
        for (cudaEvent_t* ev : {&e0, &e1}) {
            if (!c->ev_pool.empty()) { *ev = c->ev_pool.back(); c->ev_pool.pop_back(); }
            else CK(cudaEventCreate(ev));
        }
        CK(cudaEventRecord(e0, c->st));
    }
    if (launch_tc_pass(a, c->nsm, c->st) != 0) {
        if (e0) c->ev_pool.push_back(e0);
        if (e1) c->ev_pool.push_back(e1);
        set_err("tensor-core pass: unsupported geometry");
        return MSTMG_ERR_UNSUPPORTED;
    }
    CK(cudaGetLastError());
    if (c->timing) {
        CK(cudaEventRecord(e1, c->st));
        c->pending.push_back({e0, e1, 2});
    }
    c->passes32++;
    c->tc_passes++;
    return MSTMG_OK;
}

// Many columns: y[:, 0:ncols] = H x[:, 0:ncols], where column k is a
// conjugate-transpose product when bit (k & 1) of pattern2 is set (BiCG packs
// [p_1, w_1, p_2, w_2, ...]: pattern2 = 2).  On the tiled path the columns go
// in chunks of 4 or 2 (FP32, fp32_chunk) or 2 (FP64) through one launch;
// otherwise in groups of up to 4 columns, one launch each.
template <typename T> int translate_many(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int ncols, unsigned pattern2)
{
    auto expand = [&](int w) {
        unsigned m = 0;
        for (int r = 0; r < w; r++)
            if ((pattern2 >> (r & 1)) & 1u) m |= 1u << r;
        return m;
    };
    int NR = 2;
    if constexpr (sizeof(T) == 4) {
        // many plain columns: the tensor-core pass when the context has (or can
        // build) its dense operator images
        if (pattern2 == 0 && ncols >= TC_MIN_COLS && tc_eligible(c)) {
            int rc = tc_translate(c, x, y, ncols);
            if (rc != MSTMG_ERR_UNSUPPORTED) return rc;
        }
        NR = fp32_chunk(c, x, y, ncols, pattern2);
    }
    if (c->tiled && (sizeof(T) == 4 || c->tile_L >= 5) && ncols > NR && ncols % NR == 0 && tiled_supported(c->tile_L, NR)) {
        int rc = translate<T>(c, x, y, NR, expand(NR), ncols / NR);
        if (rc != MSTMG_ERR_UNSUPPORTED) return rc;
    }
    if (ncols <= 4) return translate<T>(c, x, y, ncols, expand(ncols));
    const size_t ld = (size_t)c->neqns;
    for (int k = 0; k < ncols; k += 4) {
        int w = std::min(4, ncols - k);
        int rc = translate<T>(c, x + (size_t)k * ld, y + (size_t)k * ld, w, expand(w));
        if (rc) return rc;
    }
    return MSTMG_OK;
}

int interaction_impl(mstmg_ctx* c, int nrhs, const double* ain, double* aout, const int* con_tran, const int* mie_mult,
                            int initial_run, const int* rhs_list, int skip_external)
{
    if (!c || nrhs < 1 || nrhs > 4 || !ain || !aout) {
        set_err("mstmg_interaction: bad arguments (nrhs must be 1..4)");
        return MSTMG_ERR_ARG;
    }
    int rc = skip_external ? MSTMG_OK : ensure_ops(c, 0, initial_run != 0);
    if (rc) return rc;
    const int ne = c->neqns;
    unsigned mask = 0;
    CK(copy_in(c->X64.p, ain, sizeof(zd) * (size_t)ne * nrhs, c->st));
    // columns left out of rhs_list are not translated: their output is zero
    if (rhs_list)
        for (int r = 0; r < nrhs; r++)
            if (!rhs_list[r]) CK(cudaMemsetAsync(c->X64.p + (size_t)r * ne, 0, sizeof(zd) * ne, c->st));
    for (int r = 0; r < nrhs; r++) {
        int ct = con_tran ? con_tran[r] : 0;
        int mm = mie_mult ? mie_mult[r] : 1;
        zd* col = c->X64.p + (size_t)r * ne;
        if (ct) {
            mask |= 1u << r;
            if (mm) mie_all<double>(c, -1, 1, col, col);
            else launch_conj_copy<double>(ne, col, col, c->st);
        }
    }
    if (skip_external) {
        // no pair translation: only the host-sphere couplings (none without
        // host spheres; no plane boundaries on this path)
        CK(cudaMemsetAsync(c->Y64.p, 0, sizeof(zd) * (size_t)ne * nrhs, c->st));
        if (c->hs.on()) {
            rc = ensure_ops(c, 0, initial_run != 0);
            if (rc) return rc;
            rc = translate_hosts<double>(c, c->X64.p, c->Y64.p, nrhs, mask);
            if (rc) return rc;
        }
    } else {
        rc = translate<double>(c, c->X64.p, c->Y64.p, nrhs, mask);
        if (rc) return rc;
    }
    for (int r = 0; r < nrhs; r++) {
        int ct = con_tran ? con_tran[r] : 0;
        int mm = mie_mult ? mie_mult[r] : 1;
        zd* col = c->Y64.p + (size_t)r * ne;
        if (!ct) {
            if (mm) mie_all<double>(c, 1, 0, col, col);
        } else {
            launch_conj_copy<double>(ne, col, col, c->st);
        }
    }
    CK(cudaGetLastError());
    CK(copy_out(aout, c->Y64.p, sizeof(zd) * (size_t)ne * nrhs, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_kernel_err(c);
}

extern "C" int mstmg_interaction(mstmg_ctx* c, int nrhs, const double* ain, double* aout, const int* con_tran, const int* mie_mult,
                                 int initial_run)
{
    NvtxRange nvtx_("mstmg_interaction");
    return interaction_impl(c, nrhs, ain, aout, con_tran, mie_mult, initial_run, nullptr, 0);
}

extern "C" int mstmg_interaction_ex(mstmg_ctx* c, int nrhs, const double* ain, double* aout, const int* con_tran, const int* mie_mult,
                                    int initial_run, const int* rhs_list, int fft_option, int store_matrix_option,
                                    int skip_external_translation)
{
    NvtxRange nvtx_("mstmg_interaction_ex");
    if (!c) return MSTMG_ERR_ARG;
    const bool fft_on = c->fft && c->fft->on;
    if ((fft_option == 1 && !fft_on) || (fft_option == 0 && fft_on)) {
        set_err("mstmg_interaction_ex: fft_option differs from the context's set-up (mstmg_fft_setup decides it per context)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    (void)store_matrix_option;   // the pair operators are always stored
    return interaction_impl(c, nrhs, ain, aout, con_tran, mie_mult, initial_run, rhs_list, skip_external_translation);
}

// ---------------------------------------------------------------------------
// FFT translation (fft_translation-5.f90)
// ---------------------------------------------------------------------------

static int check235(int n) /* fft:1052-1066 */
{
    int nn = n, ifac = 2;
    for (int ll = 1; ll <= 3; ll++) {
        while (nn % ifac == 0) nn /= ifac;
        ifac += ll;
    }
    return nn == 1;
}
static int correct235(int n) /* fft:1068-1076 (n >= 1: a flat extent gives one cell) */
{
    int n1 = n < 1 ? 1 : n;
    while (!check235(n1)) n1++;
    return n1;
}

// Far part: y += S Jns conv(Jsn S x) for up to 4 columns per pass.
template <typename T> int fft_far(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int ncols, unsigned contran)
{
    FftState& F = *c->fft;
    const int pi = sizeof(T) == 8 ? 0 : 1;
    const size_t per = (size_t)2 * F.nbN * F.N8;
    DevBuf<cpx<T>>& A = *reinterpret_cast<DevBuf<cpx<T>>*>(sizeof(T) == 8 ? (void*)&F.A64 : (void*)&F.A32);
    DevBuf<cpx<T>>& G = *reinterpret_cast<DevBuf<cpx<T>>*>(sizeof(T) == 8 ? (void*)&F.G64 : (void*)&F.G32);
    const cpx<T>* Jsn = sizeof(T) == 8 ? (const cpx<T>*)F.Jsn64.p : (const cpx<T>*)F.Jsn32.p;
    const cpx<T>* Jns = sizeof(T) == 8 ? (const cpx<T>*)F.Jns64.p : (const cpx<T>*)F.Jns32.p;
    if (!Jsn || !Jns) {
        set_err("FFT translation: node translations missing for this precision");
        return MSTMG_ERR_CUDA;
    }
    CK(A.alloc(4 * per));
    CK(G.alloc(4 * per));
    FftMArgs m;
    m.nsph = c->n;
    m.No = F.No;
    m.nbmax = c->lmax * (c->lmax + 2);
    m.N8 = F.N8;
    m.order = c->d_order.p;
    m.offset = c->d_offset.p;
    m.joff = F.joff.p;
    m.slot = F.slot.p;
    const size_t ld = (size_t)c->neqns;
    for (int k0 = 0; k0 < ncols; k0 += 4) {
        const int w = std::min(4, ncols - k0);
        const unsigned mask = (contran >> k0) & 0xFu;
        if (!F.have[pi][w]) {
            int nn[3] = {2 * F.cd[2], 2 * F.cd[1], 2 * F.cd[0]};
            if (cufftPlanMany(&F.plan[pi][w], 3, nn, nullptr, 1, (int)F.N8, nullptr, 1, (int)F.N8, sizeof(T) == 8 ? CUFFT_Z2Z : CUFFT_C2C,
                              w * 2 * F.nbN) != CUFFT_SUCCESS) {
                set_err("FFT translation: cufftPlanMany failed");
                return MSTMG_ERR_CUDA;
            }
            F.have[pi][w] = true;
        }
        cufftSetStream(F.plan[pi][w], c->st);
        CK(cudaMemsetAsync(A.p, 0, sizeof(cpx<T>) * w * per, c->st));
        launch_fft_s2n<T>(m, Jsn, x + (size_t)k0 * ld, (int)ld, w, mask, A.p, c->st);
        cufftResult fr;
        if (sizeof(T) == 8) fr = cufftExecZ2Z(F.plan[pi][w], (cufftDoubleComplex*)A.p, (cufftDoubleComplex*)A.p, CUFFT_FORWARD);
        else fr = cufftExecC2C(F.plan[pi][w], (cufftComplex*)A.p, (cufftComplex*)A.p, CUFFT_FORWARD);
        if (fr != CUFFT_SUCCESS) {
            set_err("FFT translation: forward transform failed");
            return MSTMG_ERR_CUDA;
        }
        launch_fft_mul<T>(F.nbN, F.N8, w, F.H.p, A.p, G.p, c->nsm, c->st);
        if (sizeof(T) == 8) fr = cufftExecZ2Z(F.plan[pi][w], (cufftDoubleComplex*)G.p, (cufftDoubleComplex*)G.p, CUFFT_INVERSE);
        else fr = cufftExecC2C(F.plan[pi][w], (cufftComplex*)G.p, (cufftComplex*)G.p, CUFFT_INVERSE);
        if (fr != CUFFT_SUCCESS) {
            set_err("FFT translation: inverse transform failed");
            return MSTMG_ERR_CUDA;
        }
        launch_fft_n2s<T>(m, Jns, G.p, w, mask, y + (size_t)k0 * ld, (int)ld, c->st);
        CK(cudaGetLastError());
    }
    return MSTMG_OK;
}

// node_selection (fft:654-825) with target box = the sphere-centre extents,
// the near-pair list, the node translations and the kernel spectra.
// Grouped tiles (the tiled kernels' tiles over listed spheres): the spheres
// of `members`, taken list by list, form groups of TILE_B; a tile holds the pairs
// of pr between two groups (or inside one), its spheres listed by slot
// (c->tsph) and each pair's slots (c->pslot).  pr is reordered tile by tile,
// the pairs of a tile in slot-disjoint couples where it has them (the row
// kernel runs such a couple as one step); tl gets the tiles.
int group_tiles(mstmg_ctx* c, const std::vector<std::vector<int>>& members, std::vector<int2>& pr, std::vector<int4>& tl)
{
    const int B = TILE_B, n = c->n;
    c->tsph.release();
    c->pslot.release();
    tl.clear();
    std::vector<int> grp(n, -1), gs(n, 0);
    int k = 0;
    for (const auto& cm : members)
        for (int i : cm) {
            grp[i] = k / B;
            gs[i] = k % B;
            k++;
        }
    const long long ng = (k + B - 1) / B;
    std::vector<int> gmem((size_t)std::max(ng, 1LL) * B, -1);
    for (int i = 0; i < n; i++)
        if (grp[i] >= 0) gmem[(size_t)grp[i] * B + gs[i]] = i;
    std::vector<long long> key(pr.size());
    std::vector<int> idx(pr.size());
    for (size_t q = 0; q < pr.size(); q++) {
        if (grp[pr[q].x] < 0 || grp[pr[q].y] < 0) {
            set_err("internal error: a pair's sphere is in no tile group");
            return MSTMG_ERR_ARG;
        }
        const long long ga = std::min(grp[pr[q].x], grp[pr[q].y]), gb = std::max(grp[pr[q].x], grp[pr[q].y]);
        key[q] = ga * ng + gb;
        idx[q] = (int)q;
    }
    std::stable_sort(idx.begin(), idx.end(), [&](int u, int v) { return key[u] < key[v]; });
    std::vector<int2> pr2(pr.size());
    std::vector<int> ts;
    std::vector<short2> ps(pr.size());
    size_t q = 0;
    while (q < idx.size()) {
        const long long kk = key[idx[q]];
        const int ga = (int)(kk / ng), gb = (int)(kk % ng);
        const size_t start = q;
        for (int s = 0; s < B; s++) ts.push_back(gmem[(size_t)ga * B + s]);
        for (int s = 0; s < B; s++) ts.push_back(ga == gb ? -1 : gmem[(size_t)gb * B + s]);
        for (; q < idx.size() && key[idx[q]] == kk; q++) {
            const int2 p2 = pr[idx[q]];
            pr2[q] = p2;
            const short si = (short)(grp[p2.x] == ga ? gs[p2.x] : B + gs[p2.x]);
            const short sj = (short)(grp[p2.y] == ga ? gs[p2.y] : B + gs[p2.y]);
            ps[q] = make_short2(si, sj);
        }
        for (size_t u = start; u + 1 < q;) {
            const short2 a0 = ps[u];
            bool found = false;
            for (size_t v = u + 1; v < q && !found; v++) {
                const short2 b0 = ps[v];
                if (a0.x != b0.x && a0.x != b0.y && a0.y != b0.x && a0.y != b0.y) {
                    std::swap(ps[u + 1], ps[v]);
                    std::swap(pr2[u + 1], pr2[v]);
                    found = true;
                }
            }
            u += found ? 2 : 1;
        }
        // z: the tile's row of the sphere lists (tiles may be dealt to shards)
        tl.push_back(make_int4((int)start, (int)(q - start), (int)tl.size(), ga == gb ? 1 : 0));
    }
    pr.swap(pr2);
    if (!ts.empty()) {
        CK(c->tsph.alloc(ts.size()));
        CK(c->pslot.alloc(ps.size()));
        CK(cudaMemcpy(c->tsph.p, ts.data(), sizeof(int) * ts.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c->pslot.p, ps.data(), sizeof(short2) * ps.size(), cudaMemcpyHostToDevice));
    }
    return MSTMG_OK;
}

int fft_build(mstmg_ctx* c)
{
    FftState& F = *c->fft;
    const int n = c->n;
    double tmin[3] = {1e10, 1e10, 1e10}, tmax[3] = {-1e10, -1e10, -1e10};
    for (int i = 0; i < n; i++)
        for (int m = 0; m < 3; m++) {
            tmin[m] = std::min(tmin[m], c->hpos[3 * (size_t)i + m]);
            tmax[m] = std::max(tmax[m], c->hpos[3 * (size_t)i + m]);
        }
    double amean = 0.0, svol = 0.0;
    for (int i = 0; i < n; i++) {
        amean += c->radius[i];
        svol += c->radius[i] * c->radius[i] * c->radius[i];
    }
    svol = std::pow(svol, 1.0 / 3.0);
    amean = amean / (double)n;
    double tvol = 1.0;
    for (int m = 0; m < 3; m++) tvol *= std::max(tmax[m] - tmin[m], amean);
    double dc = F.d_in;
    if (!(F.d_in > 0.0)) {
        double fv = F.fv_in;
        if (fv <= 0.0) {
            fv = 4.0 * MSTMG_REF_PI / 3.0 * svol * svol * svol / tvol;
            fv = std::min(fv, 1.0);
            fv = std::max(fv, 0.02);
        }
        dc = std::pow(4.0 * MSTMG_REF_PI / 3.0 / fv / (double)n, 1.0 / 3.0) * svol;
    }
    for (int m = 0; m < 3; m++) F.cd[m] = correct235((int)std::ceil((tmax[m] - tmin[m]) / dc));
    dc = 0.0;
    for (int m = 0; m < 3; m++) dc = std::max(dc, (tmax[m] - tmin[m]) / (double)F.cd[m]);
    F.dcell = dc;
    for (int m = 0; m < 3; m++) F.cb[m] = tmin[m];
    F.No = F.no_in > 0 ? F.no_in : -F.no_in + (int)std::ceil(dc);
    F.nbN = F.No * (F.No + 2);
    if (F.No < 1 || F.nbN > FFT_NBN_MAX || 2 * F.No > GT_WMAX || F.No + c->lmax > GT_WMAX) {
        set_err("FFT translation: node order out of range (1..20)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    if (c->ndense > 0) {
        set_err("FFT translation: spheres below translation_switch_order are not supported on this path");
        return MSTMG_ERR_UNSUPPORTED;
    }
    F.N8 = (size_t)8 * F.cd[0] * F.cd[1] * F.cd[2];
    const double hr_bytes = 16.0 * 2.0 * F.nbN * F.nbN * (double)F.N8;
    if (hr_bytes > 16.0e9) {
        set_err("FFT translation: kernel table above 16 GB (grid or node order too large)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    // cells of the spheres, stencil, near pairs (j > i in neighbouring cells, the reference's order)
    std::vector<int> snode(3 * (size_t)n), slot(n);
    const int N0 = 2 * F.cd[0], N1 = 2 * F.cd[1];
    std::vector<std::vector<int>> members((size_t)F.cd[0] * F.cd[1] * F.cd[2]);
    for (int i = 0; i < n; i++) {
        int cc[3];
        for (int m = 0; m < 3; m++) {
            int nd = (int)std::floor((c->hpos[3 * (size_t)i + m] - tmin[m]) / dc) + 1;
            nd = std::min(nd, F.cd[m]);
            cc[m] = std::max(nd, 1);
            snode[3 * (size_t)i + m] = cc[m];
        }
        slot[i] = (cc[0] - 1) + N0 * ((cc[1] - 1) + N1 * (cc[2] - 1));
        members[(size_t)(cc[0] - 1) + (size_t)F.cd[0] * ((cc[1] - 1) + (size_t)F.cd[1] * (cc[2] - 1))].push_back(i);
    }
    F.nnb = 0;
    for (int iz = -1; iz <= 1; iz++)
        for (int iy = -1; iy <= 1; iy++)
            for (int ix = -1; ix <= 1; ix++) {
                int ir = ix * ix + iy * iy + iz * iz;
                if ((F.model_in == 0 && ir > 0) || (F.model_in == 1 && ir > 1) || (F.model_in == 2 && ir > 2)) continue;
                F.nbv[3 * F.nnb] = ix;
                F.nbv[3 * F.nnb + 1] = iy;
                F.nbv[3 * F.nnb + 2] = iz;
                F.nnb++;
            }
    std::vector<int2> pr;
    for (int i = 0; i < n; i++)
        for (int q = 0; q < F.nnb; q++) {
            int sx = snode[3 * (size_t)i] - F.nbv[3 * q], sy = snode[3 * (size_t)i + 1] - F.nbv[3 * q + 1], sz = snode[3 * (size_t)i + 2] - F.nbv[3 * q + 2];
            if (sx < 1 || sy < 1 || sz < 1 || sx > F.cd[0] || sy > F.cd[1] || sz > F.cd[2]) continue;
            for (int j : members[(size_t)(sx - 1) + (size_t)F.cd[0] * ((sy - 1) + (size_t)F.cd[1] * (sz - 1))])
                if (j > i) pr.push_back(make_int2(i, j));
        }
    // Grouped tiles for the tiled kernel (one sphere order it supports): the
    // spheres, taken cell by cell, form groups of TILE_B; a tile holds the
    // near pairs between two groups (or inside one), its spheres listed by
    // slot, so the near pairs of nearby spheres share the tiles' output
    // accumulation as the block tiles of a whole cluster do.
    std::vector<int4> tl;
    {
        const int lmin = *std::min_element(c->order.begin(), c->order.end());
        c->tiled = !c->opts.generic_kernel && lmin == c->lmax && lmin >= c->opts.translation_switch_order && tiled_supported(c->lmax, 1) &&
                   !pr.empty();
        c->tile_L = c->lmax;
        if (c->tiled) {
            if (int rg = group_tiles(c, members, pr, tl)) return rg;
        } else {
            c->tsph.release();
            c->pslot.release();
        }
    }
    int rc = upload_pairs(c, pr, (int)pr.size(), tl);   // synchronises: the host vectors above are done with
    if (rc) return rc;
    // node translations
    std::vector<long long> joff(n + 1);
    long long tot = 0;
    for (int i = 0; i < n; i++) {
        joff[i] = tot;
        tot += 2LL * F.nbN * c->order[i] * (c->order[i] + 2);
    }
    joff[n] = tot;
    CK(F.snode.alloc(3 * (size_t)n));
    CK(F.slot.alloc(n));
    CK(F.joff.alloc(n + 1));
    CK(cudaMemcpyAsync(F.snode.p, snode.data(), sizeof(int) * 3 * n, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(F.slot.p, slot.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(F.joff.p, joff.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, c->st));
    const int nmax = std::max(F.No, c->lmax);
    std::vector<double> tcv, bd(GT_WMAX + 2);
    gentran_constants(nmax, tcv);
    mstmg::Tables& big = big_tables();
    for (int k = 0; k < (int)bd.size(); k++) bd[k] = big.bc(k, k);
    DevBuf<double> dtc, dbd, dfnr;
    CK(dtc.alloc(tcv.size()));
    CK(dbd.alloc(bd.size()));
    CK(dfnr.alloc(big.fnr.size()));
    CK(cudaMemcpyAsync(dtc.p, tcv.data(), sizeof(double) * tcv.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(dbd.p, bd.data(), sizeof(double) * bd.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(dfnr.p, big.fnr.data(), sizeof(double) * big.fnr.size(), cudaMemcpyHostToDevice, c->st));
    GtConst g;
    g.tc = dtc.p;
    g.nmax = nmax;
    g.nd = nmax * (nmax + 2);
    g.fnr = dfnr.p;
    g.bcd = dbd.p;
    CK(F.Jsn64.alloc(tot));
    CK(F.Jns64.alloc(tot));
    FftJArgs ja;
    ja.nsph = n;
    ja.No = F.No;
    ja.order = c->d_order.p;
    ja.pos = c->pos.p;
    ja.snode = F.snode.p;
    ja.dcell = dc;
    for (int m = 0; m < 3; m++) ja.cb[m] = F.cb[m];
    ja.joff = F.joff.p;
    ja.Jsn = F.Jsn64.p;
    ja.Jns = F.Jns64.p;
    ja.rimed_re = c->opts.medium_re;
    ja.rimed_im = c->opts.medium_im;
    ja.g = g;
    launch_fft_j(ja, c->st);
    CK(cudaGetLastError());
    CK(F.Jsn32.alloc(tot));
    CK(F.Jns32.alloc(tot));
    launch_d2f((int)tot, F.Jsn64.p, F.Jsn32.p, c->st);
    launch_d2f((int)tot, F.Jns64.p, F.Jns32.p, c->st);
    // kernel spectra: real-space kernels (single-precision sums), double FFT, stored in single precision
    {
        DevBuf<zd> hr;
        const size_t nel = (size_t)2 * F.nbN * F.nbN;
        CK(hr.alloc(nel * F.N8));
        FftHArgs ha;
        for (int m = 0; m < 3; m++) ha.cd[m] = F.cd[m];
        ha.No = F.No;
        ha.nnb = F.nnb;
        for (int q = 0; q < 81; q++) ha.nbv[q] = F.nbv[q];
        ha.dcell = dc;
        ha.rimed_re = c->opts.medium_re;
        ha.rimed_im = c->opts.medium_im;
        ha.hr = hr.p;
        ha.g = g;
        launch_fft_hbuild(ha, c->nsm, c->st);
        CK(cudaGetLastError());
        cufftHandle hp;
        int nn[3] = {2 * F.cd[2], 2 * F.cd[1], 2 * F.cd[0]};
        // in batches of at most 1225 transforms (one mode of a node order 5 kernel)
        const int chunk = std::min<int>((int)nel, F.nbN * F.nbN);
        if (cufftPlanMany(&hp, 3, nn, nullptr, 1, (int)F.N8, nullptr, 1, (int)F.N8, CUFFT_Z2Z, chunk) != CUFFT_SUCCESS) {
            set_err("FFT translation: kernel plan failed");
            return MSTMG_ERR_CUDA;
        }
        cufftSetStream(hp, c->st);
        bool ok = true;
        for (size_t b = 0; b + (size_t)chunk <= nel && ok; b += chunk)
            ok = cufftExecZ2Z(hp, (cufftDoubleComplex*)(hr.p + b * F.N8), (cufftDoubleComplex*)(hr.p + b * F.N8), CUFFT_FORWARD) == CUFFT_SUCCESS;
        cufftDestroy(hp);
        if (!ok) {
            set_err("FFT translation: kernel transform failed");
            return MSTMG_ERR_CUDA;
        }
        CK(F.H.alloc(nel * F.N8));
        launch_fft_round(nel * F.N8, hr.p, F.H.p, c->st);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(c->st));
    }
    F.on = true;
    return check_kernel_err(c);
}

extern "C" int mstmg_fft_setup(mstmg_ctx* c, double cell_volume_fraction, double d_cell, int node_order, int neighbor_node_model,
                               int* cell_dim, double* d_cell_out, int* node_order_out, int* near_pairs)
{
    if (int rc0 = reject_ensemble(c, "mstmg_fft_setup")) return rc0;
    if (int rh = reject_hosts(c, "mstmg_fft_setup")) return rh;
    NvtxRange nvtx_("mstmg_fft_setup");
    if (!c || c->n < 2 || neighbor_node_model < 0 || neighbor_node_model > 2) {
        set_err("mstmg_fft_setup: bad arguments (two or more spheres, neighbor_node_model 0..2)");
        return MSTMG_ERR_ARG;
    }
    if (!c->fft) c->fft.reset(new FftState());
    FftState& F = *c->fft;
    F.drop_plans();
    F.on = false;
    F.fv_in = cell_volume_fraction;
    F.d_in = d_cell;
    F.no_in = node_order;
    F.model_in = neighbor_node_model;
    int rc = fft_build(c);
    if (rc) return rc;
    if (cell_dim)
        for (int m = 0; m < 3; m++) cell_dim[m] = F.cd[m];
    if (d_cell_out) *d_cell_out = F.dcell;
    if (node_order_out) *node_order_out = F.No;
    if (near_pairs) *near_pairs = c->npairs;
    return MSTMG_OK;
}

extern "C" int mstmg_translation_pass(mstmg_ctx* c, int prec, int ncols, const int* con_tran, const double* x, double* y)
{
    NvtxRange nvtx_("mstmg_translation_pass");
    if (!c || ncols < 1 || ncols > 256 || !x || !y || prec < 0 || prec > 2) {
        set_err("mstmg_translation_pass: bad arguments");
        return MSTMG_ERR_ARG;
    }
    if (prec == 2) {   // the tensor-core pass, required
        for (int k = 0; con_tran && k < ncols; k++)
            if (con_tran[k]) {
                set_err("mstmg_translation_pass: the tensor-core pass takes no conjugate-transpose columns");
                return MSTMG_ERR_UNSUPPORTED;
            }
        if (!tc_eligible(c)) {
            set_err("mstmg_translation_pass: no tensor-core pass for this context (one sphere order 5..10, direct pairs)");
            return MSTMG_ERR_UNSUPPORTED;
        }
    }
    int rc = prec == 2 ? MSTMG_OK : ensure_ops(c, prec, false);
    if (rc) return rc;
    const size_t ne = (size_t)c->neqns, cols = ne * ncols;
    // a period-2 con_tran pattern goes through the many-column path; anything
    // else in groups of up to 4 columns with their own masks
    bool per2 = true;
    for (int k = 2; k < ncols; k++) per2 = per2 && ((con_tran ? con_tran[k] != 0 : false) == (con_tran ? con_tran[k - 2] != 0 : false));
    unsigned pattern2 = 0;
    if (con_tran && con_tran[0]) pattern2 |= 1u;
    if (con_tran && ncols > 1 && con_tran[1]) pattern2 |= 2u;
    DevBuf<zd> x64, y64;
    CK(x64.alloc(cols));
    CK(y64.alloc(cols));
    CK(copy_in(x64.p, x, sizeof(zd) * cols, c->st));
    auto groups = [&](auto* xp, auto* yp) -> int {
        using TT = std::remove_pointer_t<decltype(xp)>;
        using T = decltype(TT::x);
        if (per2) return translate_many<T>(c, xp, yp, ncols, pattern2);
        for (int k = 0; k < ncols; k += 4) {
            int w = std::min(4, ncols - k);
            unsigned m = 0;
            for (int r = 0; r < w; r++)
                if (con_tran && con_tran[k + r]) m |= 1u << r;
            int rr = translate<T>(c, xp + k * ne, yp + k * ne, w, m);
            if (rr) return rr;
        }
        return MSTMG_OK;
    };
    if (prec == 0) {
        if ((rc = groups(x64.p, y64.p))) return rc;
    } else {
        DevBuf<zf> x32, y32;
        CK(x32.alloc(cols));
        CK(y32.alloc(cols));
        launch_d2f((int)cols, x64.p, x32.p, c->st);
        if (prec == 2) rc = tc_translate(c, x32.p, y32.p, ncols);
        else rc = groups(x32.p, y32.p);
        if (rc) return rc;
        CK(cudaMemsetAsync(y64.p, 0, sizeof(zd) * cols, c->st));
        launch_add_correction_f((int)cols, y64.p, y32.p, c->st);
        CK(cudaGetLastError());
        CK(copy_out(y, y64.p, sizeof(zd) * cols, c->st));
        CK(cudaStreamSynchronize(c->st));
        return check_kernel_err(c);
    }
    CK(copy_out(y, y64.p, sizeof(zd) * cols, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_kernel_err(c);
}

extern "C" int mstmg_time_translation(mstmg_ctx* c, int prec, int nrhs, int reps, double* ms)
{
    if (!c || nrhs < 1 || nrhs > 256 || reps < 1 || prec < 0 || prec > 2) return MSTMG_ERR_ARG;
    if (prec == 2 && !tc_eligible(c)) {
        set_err("mstmg_time_translation: no tensor-core pass for this context");
        return MSTMG_ERR_UNSUPPORTED;
    }
    int rc = prec == 2 ? ensure_tc(c) : ensure_ops(c, prec, false);
    if (rc) return rc;
    DevBuf<zd> x64, y64;
    DevBuf<zf> x32, y32;
    const size_t cols = (size_t)c->neqns * nrhs;
    if (prec == 0) {
        CK(x64.alloc(cols));
        CK(y64.alloc(cols));
        CK(cudaMemsetAsync(x64.p, 0, sizeof(zd) * cols, c->st));
    } else {
        CK(x32.alloc(cols));
        CK(y32.alloc(cols));
        CK(cudaMemsetAsync(x32.p, 0, sizeof(zf) * cols, c->st));
    }
    auto pass = [&]() -> int {
        if (prec == 0) return translate_many<double>(c, x64.p, y64.p, nrhs, nrhs >= 2 ? 2u : 0u);
        if (prec == 2) return tc_translate(c, x32.p, y32.p, nrhs);   // plain columns on the tensor cores
        return translate_many<float>(c, x32.p, y32.p, nrhs, nrhs >= 2 ? 2u : 0u);
    };
    if ((rc = pass())) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        set_err("mstmg_time_translation: cudaEventCreate failed");
        return MSTMG_ERR_CUDA;
    }
    cudaEventRecord(e0, c->st);
    for (int k = 0; k < reps && rc == 0; k++) rc = pass();
    cudaEventRecord(e1, c->st);
    cudaError_t es = cudaEventSynchronize(e1);
    float t = 0.f;
    if (es == cudaSuccess) es = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    CK(es);
    if (ms) *ms = t / reps;
    return check_kernel_err(c);
}


template int translate<float>(mstmg_ctx*, const zf*, zf*, int, unsigned, int);
template int translate<double>(mstmg_ctx*, const zd*, zd*, int, unsigned, int);
template int translate_many<float>(mstmg_ctx*, const zf*, zf*, int, unsigned);
template int translate_many<double>(mstmg_ctx*, const zd*, zd*, int, unsigned);
