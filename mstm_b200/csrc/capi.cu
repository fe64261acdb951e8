// capi.cu -- the C ABI (include/mstm_b200.h): context set-up (sphere layout,
// Mie coefficients, pair lists and tiles), options, timing and diagnostics.
// The translation passes are in capi_pass.cu, the solvers in capi_solve.cu,
// the cluster-origin post-processing and the T matrix in capi_origin.cu.
#include "ctx.cuh"

static thread_local std::string g_err;
void set_err(const std::string& s) { g_err = s; }
void mstmg_internal_set_error(const std::string& msg) { set_err(msg); }

extern "C" void mstmg_default_opts(mstmg_opts* o)
{
    o->precision = MSTMG_PRECISION_FP64;
    o->device = 0;
    o->medium_re = 1.0;
    o->medium_im = 0.0;
    o->translation_switch_order = 3;
    o->inner_eps = 1.0e-8;
    o->max_outer = 30;
    o->generic_kernel = 0;
    o->tile_ctas_per_sm = 0;
    o->fp32_chunk = 0;
    o->mixed_solver = 2;
    o->gmres_restart = 0;
    o->tile_pairs = 0;
    o->tensor_core = 0;
}

extern "C" const char* mstmg_last_error(void) { return g_err.c_str(); }

// Fold completed translation-kernel event pairs into the running totals.
void resolve_timing(mstmg_ctx* c)
{
    std::vector<mstmg_ctx::Pending> keep;
    for (auto& p : c->pending) {
        if (cudaEventQuery(p.b) == cudaSuccess) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, p.a, p.b);
            c->kt_ms[p.prec] += ms;
            c->kt_n[p.prec] += 1;
            c->ev_pool.push_back(p.a);
            c->ev_pool.push_back(p.b);
        } else {
            keep.push_back(p);
        }
    }
    c->pending.swap(keep);
}

// entry points that treat the context as one cluster refuse an ensemble
int reject_ensemble(const mstmg_ctx* c, const char* fn)
{
    if (c && !c->cfg_start.empty()) {
        set_err(std::string(fn) + ": not available on an ensemble context (mstmg_ensemble_fixed_orientation solves ensembles)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    return MSTMG_OK;
}

// Solvers need the whole H x inside every iteration: a context holding one
// shard of the pairs leaves the iteration to the caller (who sums the parts).
int reject_sharded(const mstmg_ctx* c, const char* fn)
{
    if (c && c->nshards > 1) {
        set_err(std::string(fn) + ": the context translates one shard of the pairs (mstmg_set_pair_shard); iterate over the "
                                  "summed interactions instead");
        return MSTMG_ERR_UNSUPPORTED;
    }
    return MSTMG_OK;
}

// Entry points built for clusters of spheres that all sit in the medium
// refuse a context with spheres inside others.
int reject_hosts(const mstmg_ctx* c, const char* fn)
{
    if (c && c->hs.on()) {
        set_err(std::string(fn) + ": not available for a cluster with spheres inside other spheres (host spheres)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    return MSTMG_OK;
}

// Whether any sphere's centre lies inside a larger sphere (of the same
// configuration), for positions pos (host memory, 3 per sphere).
static bool any_host(const mstmg_ctx* c, const double* pos)
{
    const int n = c->n;
    if (std::all_of(c->radius.begin(), c->radius.end(), [&](double r) { return r == c->radius[0]; })) return false;   // equal spheres
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            if (!(c->radius[j] > c->radius[i])) continue;
            if (!c->cfg_of.empty() && c->cfg_of[j] != c->cfg_of[i]) continue;
            const double d0 = pos[3 * (size_t)j] - pos[3 * (size_t)i], d1 = pos[3 * (size_t)j + 1] - pos[3 * (size_t)i + 1],
                         d2 = pos[3 * (size_t)j + 2] - pos[3 * (size_t)i + 2];
            if (d0 * d0 + d1 * d1 + d2 * d2 <= c->radius[j] * c->radius[j]) return true;
        }
    return false;
}

// findhostspheres (modules:5230-5276): the holder of sphere i is the
// smallest larger sphere whose surface encloses i's centre (the first in
// order among equal radii); exteriorrefindex (modules:5408-5419) gives the
// index around each sphere.
static void find_hosts(mstmg_ctx* c, const std::vector<double>& ri)
{
    const int n = c->n;
    HostSpheres& h = c->hs;
    h.host.assign(n, -1);
    h.vid.assign(n, -1);
    h.rext.assign(2 * (size_t)n, 0.0);
    h.nhosted = h.nv = 0;
    const bool equal = std::all_of(c->radius.begin(), c->radius.end(), [&](double r) { return r == c->radius[0]; });
    for (int i = 0; i < n && !equal; i++) {   // equal spheres hold none
        double xspmin = 1.0e6;
        for (int j = 0; j < n; j++) {
            if (!(c->radius[j] > c->radius[i])) continue;
            if (!c->cfg_of.empty() && c->cfg_of[j] != c->cfg_of[i]) continue;   // an ensemble's configurations do not meet
            const double d0 = c->hpos[3 * (size_t)j] - c->hpos[3 * (size_t)i], d1 = c->hpos[3 * (size_t)j + 1] - c->hpos[3 * (size_t)i + 1],
                         d2 = c->hpos[3 * (size_t)j + 2] - c->hpos[3 * (size_t)i + 2];
            const double rij = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            if (rij <= c->radius[j] && c->radius[j] < xspmin) {
                h.host[i] = j;
                xspmin = c->radius[j];
            }
        }
    }
    for (int i = 0; i < n; i++) {
        const int j = h.host[i];
        if (j >= 0) {
            h.nhosted++;
            if (h.vid[j] < 0) h.vid[j] = 0;
        }
        h.rext[2 * (size_t)i] = j >= 0 ? ri[2 * (size_t)j] : c->opts.medium_re;
        h.rext[2 * (size_t)i + 1] = j >= 0 ? ri[2 * (size_t)j + 1] : c->opts.medium_im;
    }
    for (int i = 0; i < n; i++)
        if (h.vid[i] >= 0) h.vid[i] = n + 1 + h.nv++;
}

// Upload the tiles of this context's shard (all tiles when nshards == 1).
int apply_shard(mstmg_ctx* c)
{
    std::vector<int4> sub;
    sub.reserve(c->tiles_host.size() / (size_t)c->nshards + 1);
    for (size_t t = 0; t < c->tiles_host.size(); t++)
        if ((int)(t % (size_t)c->nshards) == c->shard) sub.push_back(c->tiles_host[t]);
    c->ntiles = (int)sub.size();
    if (!sub.empty()) {
        CK(c->tiles.alloc(sub.size()));
        CK(cudaMemcpyAsync(c->tiles.p, sub.data(), sizeof(int4) * sub.size(), cudaMemcpyHostToDevice, c->st));
        CK(cudaStreamSynchronize(c->st));
    }
    c->layout_gen++;
    return MSTMG_OK;
}

int check_kernel_err(mstmg_ctx* c)
{
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (herr != 0) {
        set_err("device kernel reported status " + std::to_string(herr));
        int z = 0;
        cudaMemcpyAsync(c->err.p, &z, sizeof(int), cudaMemcpyHostToDevice, c->st);
        cudaStreamSynchronize(c->st);
        return herr;
    }
    return MSTMG_OK;
}

// Install a pair list (i < j) and, for the tiled kernel, its tiles: operator
// record offsets, the device copies, and invalidated operators.
int upload_pairs(mstmg_ctx* c, const std::vector<int2>& pr, int np, const std::vector<int4>& tl)
{
    std::vector<long long> off(np > 0 ? np : 1);
    long long u = 0;
    int maxrec = 4, pl = 1, lo = 1 << 30;
    for (int t = 0; t < np; t++) {
        off[t] = u;
        int rec = op_record_units(c->order[pr[t].x], c->order[pr[t].y]);
        maxrec = std::max(maxrec, rec);
        pl = std::max(pl, std::max(c->order[pr[t].x], c->order[pr[t].y]));
        lo = std::min(lo, std::min(c->order[pr[t].x], c->order[pr[t].y]));
        u += rec;
    }
    c->npairs = np;
    c->pair_lmax = pl;
    c->pair_uniform = np > 0 && lo == pl;
    c->tiles_host = tl;
    if (!c->tiled) {   // shards need tiles; a re-layout without them drops the shard
        c->shard = 0;
        c->nshards = 1;
    }
    if (int rs = apply_shard(c)) return rs;
    c->op_units = u;
    c->maxrec = maxrec;
    // FP32 passes of the tiled path run the row kernel on row records unless
    // the rotation-tiled kernel is asked for (tile_pairs 1 or 2)
    c->row32 = (c->tiled && c->opts.tile_pairs == 0 && rows_supported(c->tile_L, 1)) ? row_record_units(c->tile_L) : 0;
    c->layout_gen++;
    if (np > 0) {
        CK(c->pairs.alloc(np));
        CK(c->opoff.alloc(np));
        CK(cudaMemcpyAsync(c->pairs.p, pr.data(), sizeof(int2) * np, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(c->opoff.p, off.data(), sizeof(long long) * np, cudaMemcpyHostToDevice, c->st));
        CK(cudaStreamSynchronize(c->st));   // host vectors are freed on return
    }
    c->ops64_ready = c->ops32_ready = false;
    if (c->tc_state == 1) c->tc_state = 0;
    return MSTMG_OK;
}

// tran_coef constants of gentranmatrix (and the tables its Legendre
// recurrence uses) for orders up to lm, on the device
int ensure_gentran(mstmg_ctx* c, int lm)
{
    if (c->gt_nmax >= lm) return MSTMG_OK;
    std::vector<double> tcv, bd(GT_WMAX + 2);
    gentran_constants(lm, tcv);
    mstmg::Tables tb(6 * GT_WMAX + 6);
    for (int k = 0; k < (int)bd.size(); k++) bd[k] = tb.bc(k, k);
    CK(c->gt_tc.alloc(tcv.size()));
    CK(c->gt_bcd.alloc(bd.size()));
    CK(c->gt_fnr.alloc(tb.fnr.size()));
    CK(cudaMemcpyAsync(c->gt_tc.p, tcv.data(), sizeof(double) * tcv.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->gt_bcd.p, bd.data(), sizeof(double) * bd.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->gt_fnr.p, tb.fnr.data(), sizeof(double) * tb.fnr.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->gt_nmax = lm;
    return MSTMG_OK;
}

// The host-sphere pieces of the pair lists: the medium index of every
// same-host pair (rotation and dense), and the regular translations between
// each host's internal block and the spheres it holds
// (external_to_internal_expansion, modules:6533-6608), with their operator
// record offsets; coincident centres go to the copy list.
static int setup_host_pairs(mstmg_ctx* c, const std::vector<int2>& pr, int np)
{
    HostSpheres& h = c->hs;
    const int n = c->n;
    std::vector<double> pm(2 * (size_t)std::max(np, 1)), dm(2 * (size_t)std::max(c->ndense, 1));
    for (int t = 0; t < np; t++) {
        pm[2 * (size_t)t] = h.rext[2 * (size_t)pr[t].x];
        pm[2 * (size_t)t + 1] = h.rext[2 * (size_t)pr[t].x + 1];
    }
    if (c->ndense > 0) {
        std::vector<int2> dp(c->ndense);
        CK(cudaMemcpy(dp.data(), c->dpairs.p, sizeof(int2) * c->ndense, cudaMemcpyDeviceToHost));
        for (int t = 0; t < c->ndense; t++) {
            dm[2 * (size_t)t] = h.rext[2 * (size_t)dp[t].x];
            dm[2 * (size_t)t + 1] = h.rext[2 * (size_t)dp[t].x + 1];
        }
    }
    CK(h.pmed.alloc(pm.size()));
    CK(h.dmed.alloc(dm.size()));
    CK(cudaMemcpy(h.pmed.p, pm.data(), sizeof(double) * pm.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h.dmed.p, dm.data(), sizeof(double) * dm.size(), cudaMemcpyHostToDevice));
    // positions of the device sphere arrays (the internal blocks at their host's centre)
    std::vector<double> xp(3 * (size_t)(n + 1 + h.nv), 0.0);
    std::copy(c->hpos.begin(), c->hpos.end(), xp.begin());
    for (int i = 0; i < n; i++)
        if (h.vid[i] >= 0)
            for (int k = 0; k < 3; k++) xp[3 * (size_t)h.vid[i] + k] = c->hpos[3 * (size_t)i + k];
    std::vector<int2> hp, zp;
    std::vector<long long> off;
    std::vector<double> hm;
    long long u = 0;
    int maxrec = 4, hl = 0;
    for (int j = 0; j < n; j++) {
        const int i = h.host[j];
        if (i < 0) continue;
        double d2 = 0.0;
        for (int k = 0; k < 3; k++) {
            const double d = c->hpos[3 * (size_t)i + k] - c->hpos[3 * (size_t)j + k];
            d2 += d * d;
        }
        if (d2 < 1.0e-12) {   // zero_translation (modules:6645-6650)
            zp.push_back(make_int2(h.vid[i], j));
            continue;
        }
        hp.push_back(make_int2(h.vid[i], j));
        off.push_back(u);
        const int rec = op_record_units(c->order[i], c->order[j]);
        maxrec = std::max(maxrec, rec);
        hl = std::max(hl, std::max(c->order[i], c->order[j]));
        u += rec;
        hm.push_back(c->ri_host[2 * (size_t)i]);
        hm.push_back(c->ri_host[2 * (size_t)i + 1]);
    }
    h.nhp = (int)hp.size();
    h.nzp = (int)zp.size();
    h.hunits = u;
    h.hmaxrec = maxrec;
    h.hlmax = hl;
    h.hops_ready = h.hops32_ready = false;
    if (h.nhp > 0) {
        CK(h.hpairs.alloc(h.nhp));
        CK(h.hopoff.alloc(h.nhp));
        CK(h.hmed.alloc(hm.size()));
        CK(h.xpos.alloc(xp.size()));
        CK(cudaMemcpy(h.hpairs.p, hp.data(), sizeof(int2) * hp.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h.hopoff.p, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h.hmed.p, hm.data(), sizeof(double) * hm.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h.xpos.p, xp.data(), sizeof(double) * xp.size(), cudaMemcpyHostToDevice));
    }
    if (h.nzp > 0) {
        CK(h.zpairs.alloc(h.nzp));
        CK(cudaMemcpy(h.zpairs.p, zp.data(), sizeof(int2) * zp.size(), cudaMemcpyHostToDevice));
    }
    return MSTMG_OK;
}

int setup_layout(mstmg_ctx* c)
{
    const int n = c->n;
    c->offset.assign(n + 1, 0);
    c->mie_offset.assign(n + 1, 0);
    int lm = 0, lmin = 1 << 30;
    long long ne = 0, nt = 0;
    const HostSpheres& hs = c->hs;
    for (int i = 0; i < n; i++) {
        int L = c->order[i];
        c->offset[i] = (int)ne;
        c->mie_offset[i] = (int)nt;
        // a sphere holding others: its block, then the field inside it (number_field_expansions 2)
        ne += 2LL * L * (L + 2) * (hs.on() && hs.vid[i] >= 0 ? 2 : 1);
        nt += 4LL * L;
        lm = std::max(lm, L);
        lmin = std::min(lmin, L);
    }
    c->offset[n] = (int)ne;
    c->mie_offset[n] = (int)nt;
    if (lm > MSTMG_LMAX) {
        set_err("sphere order " + std::to_string(lm) + " exceeds the kernels' limit " + std::to_string(MSTMG_LMAX));
        return MSTMG_ERR_UNSUPPORTED;
    }
    if (2 * lm > GT_WMAX) {
        set_err("sphere orders above 20 are not supported");
        return MSTMG_ERR_UNSUPPORTED;
    }
    c->neqns = (int)ne;
    c->lmax = lm;
    // device sphere arrays: the spheres, the offset sentinel at n, then the
    // internal blocks of the spheres holding others (index n + 1 + v)
    const int next = n + 1 + hs.nv;
    std::vector<int> xord(next, 0), xoff(next, 0), xmie(next, 0), hoff(hs.on() ? n : 0, -1);
    for (int i = 0; i < n; i++) {
        xord[i] = c->order[i];
        xoff[i] = c->offset[i];
        xmie[i] = c->mie_offset[i];
    }
    xoff[n] = c->offset[n];
    xmie[n] = c->mie_offset[n];
    if (hs.on())
        for (int i = 0; i < n; i++)
            if (hs.vid[i] >= 0) {
                const int v = hs.vid[i], L = c->order[i];
                xord[v] = L;
                xoff[v] = hoff[i] = c->offset[i] + 2 * L * (L + 2);
                xmie[v] = c->mie_offset[i];
            }
    CK(c->d_order.alloc(next));
    CK(c->d_offset.alloc(next));
    CK(c->d_mie_offset.alloc(next));
    CK(cudaMemcpyAsync(c->d_order.p, xord.data(), sizeof(int) * next, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_offset.p, xoff.data(), sizeof(int) * next, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_mie_offset.p, xmie.data(), sizeof(int) * next, cudaMemcpyHostToDevice, c->st));
    // slot maps
    std::vector<int> slot(ne / 2), slotf(ne);
    for (int i = 0; i < next; i++) {
        if (i == n) continue;
        int L = xord[i], hb = L * (L + 2);
        for (int k = 0; k < hb; k++) slot[xoff[i] / 2 + k] = i;
        for (int k = 0; k < 2 * hb; k++) slotf[xoff[i] + k] = i;
    }
    CK(c->slot.alloc(ne / 2));
    CK(c->slot_full.alloc(ne));
    CK(cudaMemcpyAsync(c->slot.p, slot.data(), sizeof(int) * slot.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->slot_full.p, slotf.data(), sizeof(int) * slotf.size(), cudaMemcpyHostToDevice, c->st));
    // Mie coefficients
    CK(c->an.alloc(nt));
    CK(c->an_inv.alloc(nt));
    CK(c->an32.alloc(2 * nt));
    CK(c->qext.alloc(n));
    CK(c->qabs.alloc(n));
    if (hs.on()) {
        HostSpheres& h = c->hs;
        std::vector<int> outside(n);
        for (int i = 0; i < n; i++) outside[i] = h.host[i] < 0 ? 1 : 0;
        CK(h.d_hoff.alloc(n));
        CK(h.d_outside.alloc(n));
        CK(h.d_host.alloc(n));
        CK(h.qv.alloc(3LL * n));
        CK(h.dn.alloc(nt));
        CK(h.un.alloc(nt));
        CK(h.vn.alloc(nt));
        CK(cudaMemcpyAsync(h.d_hoff.p, hoff.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(h.d_outside.p, outside.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(h.d_host.p, h.host.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
        std::vector<int> hst(n + 1, 0), held;
        for (int i = 0; i < n; i++)
            if (h.host[i] >= 0) hst[h.host[i] + 1]++;
        for (int i = 0; i < n; i++) hst[i + 1] += hst[i];
        held.assign(std::max(hst[n], 1), 0);
        std::vector<int> fill(hst.begin(), hst.end() - 1);
        for (int j = 0; j < n; j++)
            if (h.host[j] >= 0) held[fill[h.host[j]]++] = j;
        CK(h.d_hstart.alloc(n + 1));
        CK(h.d_held.alloc(held.size()));
        CK(cudaMemcpy(h.d_hstart.p, hst.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h.d_held.p, held.data(), sizeof(int) * held.size(), cudaMemcpyHostToDevice));
    }
    launch_mie_coefs(n, c->rad.p, c->ri.p, c->opts.medium_re, c->opts.medium_im, hs.on() ? hs.d_rext.p : nullptr, c->d_order.p,
                     c->d_mie_offset.p, hs.on() ? hs.d_hoff.p : nullptr, c->an.p, c->an_inv.p, c->an32.p, c->hs.dn.p, c->hs.un.p,
                     c->hs.vn.p, c->qext.p, c->qabs.p, c->st);
    CK(cudaGetLastError());
    if (hs.on()) {
        HostSpheres& h = c->hs;
        CK(h.dn32.alloc(nt));
        CK(h.un32.alloc(nt));
        CK(h.vn32.alloc(nt));
        launch_d2f((int)nt, h.dn.p, h.dn32.p, c->st);
        launch_d2f((int)nt, h.un.p, h.un32.p, c->st);
        launch_d2f((int)nt, h.vn.p, h.vn32.p, c->st);
        CK(cudaGetLastError());
    }
    // pairs whose smaller order is below translation_switch_order take the
    // reference's dense path (coefficient_translation, rot_op false)
    const int tso = c->opts.translation_switch_order;
    auto dense_pair = [&](int i, int j) { return std::min(c->order[i], c->order[j]) < tso; };
    // an ensemble has no pairs between its configurations; spheres interact
    // directly only inside the same host (modules:6466-6469)
    auto same_cfg = [&](int i, int j) {
        return (c->cfg_of.empty() || c->cfg_of[i] == c->cfg_of[j]) && (!hs.on() || hs.host[i] == hs.host[j]);
    };
    {
        std::vector<int2> dp;
        std::vector<long long> doff;
        long long du = 0;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
                if (same_cfg(i, j) && dense_pair(i, j)) {
                    dp.push_back(make_int2(i, j));
                    doff.push_back(du);
                    du += 2LL * c->order[i] * (c->order[i] + 2) * c->order[j] * (c->order[j] + 2);
                }
        c->ndense = (int)dp.size();
        c->dense_units = du;
        if (c->ndense > 0) {
            CK(c->dpairs.alloc(dp.size()));
            CK(c->doff.alloc(doff.size()));
            CK(cudaMemcpyAsync(c->dpairs.p, dp.data(), sizeof(int2) * dp.size(), cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(c->doff.p, doff.data(), sizeof(long long) * doff.size(), cudaMemcpyHostToDevice, c->st));
            if (int rg = ensure_gentran(c, lm)) return rg;
        }
    }
    // pair list (i < j, the reference's loop order) and operator offsets
    long long np = (long long)n * (n - 1) / 2 - c->ndense;
    if (hs.on()) {
        np = -c->ndense;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++) np += same_cfg(i, j) ? 1 : 0;
    } else if (!c->cfg_of.empty()) {
        np = -c->ndense;
        for (size_t k = 0; k + 1 < c->cfg_start.size(); k++) {
            const long long m = c->cfg_start[k + 1] - c->cfg_start[k];
            np += m * (m - 1) / 2;
        }
    }
    if (np > 2000000000LL) {
        set_err("too many sphere pairs for the direct translation path");
        return MSTMG_ERR_UNSUPPORTED;
    }
    c->npairs = (int)np;
    // Pair order.  Monodisperse clusters of a supported order use tiles of
    // TILE_B x TILE_B sphere blocks (translate_tiled.cu); the block pairs are
    // visited in round-robin tournament order (circle method), so tiles that
    // run at the same time write mostly disjoint spheres.  Otherwise the pairs
    // themselves follow the tournament order: each round holds floor(N/2)
    // pairs with no sphere in common, so concurrent CTAs' atomic adds do not
    // collide.  Pairs keep i < j, the reference's orientation of the operator.
    std::vector<int2> pr(np > 0 ? np : 1);
    std::vector<long long> off(np > 0 ? np : 1);
    long long u = 0;
    int maxrec = 4;
    long long t = 0;
    auto add_pair = [&](int i, int j) {
        pr[t] = make_int2(i, j);
        off[t] = u;
        int rec = op_record_units(c->order[i], c->order[j]);
        maxrec = std::max(maxrec, rec);
        u += rec;
        t++;
    };
    auto tournament = [](int n, std::vector<std::pair<int, int>>& out) {
        int M = (n % 2 == 0) ? n : n + 1;
        for (int r = 0; r < M - 1 && n > 1; r++)
            for (int k = 0; k < M / 2; k++) {
                int a_, b_;
                if (k == 0) { a_ = M - 1; b_ = r; }
                else { a_ = (r + k) % (M - 1); b_ = (r - k + (M - 1)) % (M - 1); }
                if (a_ >= n || b_ >= n) continue;
                out.push_back({std::min(a_, b_), std::max(a_, b_)});
            }
    };
    c->tiled = !c->opts.generic_kernel && !hs.on() && (lm == lmin) && lmin >= tso && tiled_supported(lm, 1) && n > 1 && n < 65536;
    std::vector<int4> tl;
    if (c->tiled) {
        const int B = TILE_B;
        int nb = (n + B - 1) / B;
        std::vector<std::pair<int, int>> bp;
        tournament(nb, bp);
        for (int I = 0; I < nb; I++) bp.push_back({I, I});
        for (auto& IJ : bp) {
            int I = IJ.first, J = IJ.second;
            int i0 = I * B, j0 = J * B;
            int start = (int)t;
            // inside a tile, consecutive pairs (0,1), (2,3), ... share no
            // sphere wherever the tile is whole: an off-diagonal tile runs the
            // diagonals (a, a+s mod B) of its block pair, a diagonal tile the
            // matchings {01, 23}, {02, 13}, {03, 12}; the row kernel takes two
            // such pairs a step
            static_assert(TILE_B == 4, "the diagonal-tile order below is for blocks of 4 spheres");
            static const int dg[6][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {0, 3}, {1, 2}};
            auto try_add = [&](int i, int j) {
                if (i < n && j < n && i < j && same_cfg(i, j)) add_pair(i, j);
            };
            if (I == J) {
                for (const auto& d : dg) try_add(i0 + d[0], i0 + d[1]);
            } else {
                for (int sft = 0; sft < B; sft++)
                    for (int a_ = 0; a_ < B; a_++) try_add(i0 + a_, j0 + (a_ + sft) % B);
            }
            int cnt = (int)t - start;
            if (cnt > 0) tl.push_back(make_int4(start, cnt, (i0 << 16) | j0, I == J ? 1 : 0));
        }
    } else {
        std::vector<std::pair<int, int>> pp;
        tournament(n, pp);
        for (auto& ij : pp)
            if (same_cfg(ij.first, ij.second) && !dense_pair(ij.first, ij.second)) add_pair(ij.first, ij.second);
    }
    if (t != np) {
        set_err("internal error: pair schedule incomplete");
        return MSTMG_ERR_ARG;
    }
    c->tile_L = lm;
    c->tsph.release();   // block tiles
    c->pslot.release();
    if (hs.on() && !c->opts.generic_kernel && np > 0) {
        // host spheres: when the pairs inside the hosts all have one order
        // the tiled kernels take them on grouped tiles (the spheres of each
        // host in groups, each sphere's block at its own offset)
        const int L0 = c->order[pr[0].x];
        bool uni = true;
        for (long long q = 0; q < np && uni; q++) uni = c->order[pr[q].x] == L0 && c->order[pr[q].y] == L0;
        if (uni && L0 >= tso && tiled_supported(L0, 1)) {
            std::vector<char> inp(n, 0);
            for (long long q = 0; q < np; q++) inp[pr[q].x] = inp[pr[q].y] = 1;
            std::vector<std::vector<int>> members(n + 1);   // by host, the spheres outside every other first
            for (int i = 0; i < n; i++)
                if (inp[i]) members[hs.host[i] + 1].push_back(i);
            if (int rg = group_tiles(c, members, pr, tl)) return rg;
            c->tiled = true;
            c->tile_L = L0;
        }
    }
    (void)off;
    (void)maxrec;
    int rc_ = upload_pairs(c, pr, (int)np, tl);
    if (rc_) return rc_;
    if (hs.on()) {
        rc_ = setup_host_pairs(c, pr, (int)np);
        if (rc_) return rc_;
    }
    // constant tables
    mstmg::Tables tb(6 * lm + 6);
    std::vector<double> vcc, f1, f2, f3;
    tb.axial_constants(lm, vcc, f1, f2, f3);
    c->vn = lm;
    std::vector<double> bd(lm + 2, 0.0);
    for (int k = 0; k <= lm + 1; k++) bd[k] = tb.bc(k, k);
    std::vector<double> rf(tb.fnr.size(), 0.0);
    for (size_t k = 1; k < rf.size(); k++) rf[k] = 1.0 / tb.fnr[k];
    CK(c->vcc.alloc(vcc.size()));
    CK(c->fnr.alloc(tb.fnr.size()));
    CK(c->rfnr.alloc(rf.size()));
    CK(c->bcofd.alloc(bd.size()));
    CK(cudaMemcpyAsync(c->vcc.p, vcc.data(), sizeof(double) * vcc.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->fnr.p, tb.fnr.data(), sizeof(double) * tb.fnr.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->rfnr.p, rf.data(), sizeof(double) * rf.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->bcofd.p, bd.data(), sizeof(double) * bd.size(), cudaMemcpyHostToDevice, c->st));
    // work buffers
    CK(c->X64.alloc(4LL * ne));
    CK(c->Y64.alloc(4LL * ne));
    CK(c->X32.alloc(4LL * ne));
    CK(c->Y32.alloc(4LL * ne));
    CK(c->pmnp.alloc(2LL * ne));
    CK(c->amnp.alloc(2LL * ne));
    CK(c->vec64.alloc(2LL * 7 * ne));
    CK(c->bvec64.alloc(2LL * ne));
    CK(c->vec32.alloc(2LL * 7 * ne));
    CK(c->rvec32.alloc(2LL * ne));
    CK(c->pw0.alloc(2LL * 2 * lm * (lm + 2)));
    CK(c->drot.alloc(3LL * (lm * (lm + 2) + 1)));
    CK(c->part.alloc(3LL * c->nsm * 4 + 16));
    CK(c->qeff.alloc(9LL * n));
    CK(c->qtot.alloc(9));
    CK(c->small.alloc(16));
    CK(c->sc.alloc(4));
    // vol_radius as main_calling_program forms it: (sum r^3)**.333333 (single-precision
    // literal) over the spheres outside every other (input:1218-1225)
    double v = 0.0;
    for (int i = 0; i < n; i++)
        if (!hs.on() || hs.host[i] < 0) v = v + c->radius[i] * c->radius[i] * c->radius[i];
    c->xg = std::pow(v, (double)0.333333f);
    if (!c->cfg_start.empty()) {
        const int nc = (int)c->cfg_start.size() - 1;
        c->cfg_xg.assign(nc, 0.0);
        std::vector<int> off(2 * nc), len(2 * nc);
        c->ens_ldv = 0;
        for (int k = 0; k < nc; k++) {
            double vk = 0.0;
            for (int i = c->cfg_start[k]; i < c->cfg_start[k + 1]; i++) vk = vk + c->radius[i] * c->radius[i] * c->radius[i];
            c->cfg_xg[k] = std::pow(vk, (double)0.333333f);
            const int o = c->offset[c->cfg_start[k]], l = c->offset[c->cfg_start[k + 1]] - o;
            off[2 * k] = off[2 * k + 1] = o;
            len[2 * k] = len[2 * k + 1] = l;
            c->ens_ldv = std::max(c->ens_ldv, l);
        }
        c->ens_ldv = ((c->ens_ldv + 3) / 4) * 4;
        CK(c->d_cfg_start.alloc(nc + 1));
        CK(c->d_cfg_xg.alloc(nc));
        CK(c->cfg_qtot.alloc(9LL * nc));
        CK(c->ens_off.alloc(2 * nc));
        CK(c->ens_len.alloc(2 * nc));
        CK(cudaMemcpyAsync(c->d_cfg_start.p, c->cfg_start.data(), sizeof(int) * (nc + 1), cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(c->d_cfg_xg.p, c->cfg_xg.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(c->ens_off.p, off.data(), sizeof(int) * 2 * nc, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(c->ens_len.p, len.data(), sizeof(int) * 2 * nc, cudaMemcpyHostToDevice, c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return MSTMG_OK;
}

static int create_impl(mstmg_ctx** out, int nsphere, const double* pos, const double* radius, const double* ref_index, double mie_epsilon,
                       const mstmg_opts* opts, int nconfig, const int* config_start);

extern "C" int mstmg_ctx_create(mstmg_ctx** out, int nsphere, const double* pos, const double* radius, const double* ref_index,
                                double mie_epsilon, const mstmg_opts* opts)
{
    return create_impl(out, nsphere, pos, radius, ref_index, mie_epsilon, opts, 0, nullptr);
}

extern "C" int mstmg_ensemble_create(mstmg_ctx** out, int nconfig, const int* config_start, int nsphere, const double* pos,
                                     const double* radius, const double* ref_index, double mie_epsilon, const mstmg_opts* opts)
{
    if (out) *out = nullptr;
    if (nconfig < 1 || !config_start || config_start[0] != 0 || config_start[nconfig] != nsphere) {
        set_err("mstmg_ensemble_create: config_start must run from 0 to nsphere over nconfig >= 1 configurations");
        return MSTMG_ERR_ARG;
    }
    for (int k = 0; k < nconfig; k++)
        if (config_start[k + 1] <= config_start[k]) {
            set_err("mstmg_ensemble_create: configuration " + std::to_string(k + 1) + " has no spheres");
            return MSTMG_ERR_ARG;
        }
    return create_impl(out, nsphere, pos, radius, ref_index, mie_epsilon, opts, nconfig, config_start);
}

static int create_impl(mstmg_ctx** out, int nsphere, const double* pos, const double* radius, const double* ref_index, double mie_epsilon,
                       const mstmg_opts* opts, int nconfig, const int* config_start)
{
    if (!out || nsphere < 1 || !pos || !radius || !ref_index) {
        set_err("mstmg_ctx_create: bad arguments");
        return MSTMG_ERR_ARG;
    }
    *out = nullptr;
    if (!is_dev(pos) && !is_dev(radius) && !is_dev(ref_index)) {
        // host inputs are checked before anything reaches the GPU
        for (int i = 0; i < nsphere; i++) {
            bool ok = std::isfinite(radius[i]) && radius[i] > 0.0 && std::isfinite(ref_index[2 * i]) && std::isfinite(ref_index[2 * i + 1]);
            for (int k = 0; k < 3; k++) ok = ok && std::isfinite(pos[3 * (size_t)i + k]);
            if (!ok) {
                set_err("mstmg_ctx_create: sphere " + std::to_string(i + 1) + " has a non-finite position or index, or a radius <= 0");
                return MSTMG_ERR_ARG;
            }
        }
    }
    if (opts && (opts->gmres_restart < 0 || opts->mixed_solver < 0 || opts->mixed_solver > 2 || opts->tensor_core < -1 ||
                 opts->tensor_core > 1 || opts->tile_pairs < 0 || opts->tile_pairs > 2)) {
        set_err("mstmg_ctx_create: gmres_restart must be >= 0, mixed_solver 0, 1 or 2, tensor_core -1, 0 or 1, tile_pairs 0, 1 or 2");
        return MSTMG_ERR_ARG;
    }
    mstmg_ctx* c = new mstmg_ctx();
    if (opts) c->opts = *opts;
    else mstmg_default_opts(&c->opts);
    c->n = nsphere;
    int rc;
    {
        cudaError_t e = cudaSetDevice(c->opts.device);
        if (e != cudaSuccess) {
            set_err(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
            delete c;
            return MSTMG_ERR_CUDA;
        }
        cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->opts.device);
        e = cudaStreamCreateWithFlags(&c->own_st, cudaStreamNonBlocking);
        c->st = c->own_st;
        if (e != cudaSuccess) {
            set_err(std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
            delete c;
            return MSTMG_ERR_CUDA;
        }
        if (cudaMallocHost((void**)&c->h_sc, sizeof(BicgScalars) * 4) != cudaSuccess ||
            cudaMallocHost((void**)&c->h_small, sizeof(double) * 16) != cudaSuccess) {
            set_err("cudaMallocHost failed");
            mstmg_ctx_destroy(c);
            return MSTMG_ERR_CUDA;
        }
    }
    auto fail = [&](int code) {
        mstmg_ctx_destroy(c);
        return code;
    };
    if (c->pos.alloc(3LL * nsphere) || c->rad.alloc(nsphere) || c->ri.alloc(2LL * nsphere) || c->err.alloc(1)) {
        set_err("cudaMalloc failed");
        return fail(MSTMG_ERR_CUDA);
    }
    c->radius.assign(radius, radius + nsphere);
    c->hpos.assign(3 * (size_t)nsphere, 0.0);
    if (is_dev(pos)) {
        if (cudaMemcpy(c->hpos.data(), pos, sizeof(double) * 3 * nsphere, cudaMemcpyDeviceToHost)) return fail(MSTMG_ERR_CUDA);
    } else {
        memcpy(c->hpos.data(), pos, sizeof(double) * 3 * nsphere);
    }
    if (copy_in(c->pos.p, pos, sizeof(double) * 3 * nsphere, c->st) || copy_in(c->rad.p, radius, sizeof(double) * nsphere, c->st) ||
        copy_in(c->ri.p, ref_index, sizeof(double) * 2 * nsphere, c->st) || cudaMemsetAsync(c->err.p, 0, sizeof(int), c->st)) {
        set_err("copy of sphere data failed");
        return fail(MSTMG_ERR_CUDA);
    }
    if (is_dev(radius)) {
        if (cudaMemcpy(c->radius.data(), radius, sizeof(double) * nsphere, cudaMemcpyDeviceToHost)) return fail(MSTMG_ERR_CUDA);
    }
    c->ri_host.assign(2 * (size_t)nsphere, 0.0);
    if (is_dev(ref_index)) {
        if (cudaMemcpy(c->ri_host.data(), ref_index, sizeof(double) * 2 * nsphere, cudaMemcpyDeviceToHost)) return fail(MSTMG_ERR_CUDA);
    } else {
        memcpy(c->ri_host.data(), ref_index, sizeof(double) * 2 * nsphere);
    }
    if (nconfig > 0) {
        c->cfg_start.assign(config_start, config_start + nconfig + 1);
        c->cfg_of.assign(nsphere, 0);
        for (int k = 0; k < nconfig; k++)
            for (int i = config_start[k]; i < config_start[k + 1]; i++) c->cfg_of[i] = k;
    }
    find_hosts(c, c->ri_host);
    if (c->hs.on()) {
        if (nconfig > 0) {
            set_err("mstmg_ensemble_create: configurations with spheres inside other spheres are not supported in ensembles");
            return fail(MSTMG_ERR_UNSUPPORTED);
        }
        if (c->hs.d_rext.alloc(2LL * nsphere) ||
            cudaMemcpyAsync(c->hs.d_rext.p, c->hs.rext.data(), sizeof(double) * 2 * nsphere, cudaMemcpyHostToDevice, c->st)) {
            set_err("copy of the exterior indices failed");
            return fail(MSTMG_ERR_CUDA);
        }
    }
    // sphere orders on the device (mieoa order test, each sphere in the index
    // around it), read back for the layout
    DevBuf<int> ord;
    if (ord.alloc(nsphere)) return fail(MSTMG_ERR_CUDA);
    launch_mie_orders(nsphere, c->rad.p, c->ri.p, c->opts.medium_re, c->opts.medium_im, c->hs.on() ? c->hs.d_rext.p : nullptr, mie_epsilon,
                      ord.p, c->st);
    c->order.assign(nsphere, 0);
    if (cudaMemcpyAsync(c->order.data(), ord.p, sizeof(int) * nsphere, cudaMemcpyDeviceToHost, c->st) ||
        cudaStreamSynchronize(c->st)) {
        set_err("mie order kernel failed");
        ord.release();
        return fail(MSTMG_ERR_CUDA);
    }
    ord.release();
    // a host has at least the order of every sphere inside it (modules:5331-5342)
    if (c->hs.on())
        for (int i = 0; i < nsphere; i++)
            for (int j = c->hs.host[i]; j >= 0; j = c->hs.host[j]) c->order[j] = std::max(c->order[j], c->order[i]);
    rc = setup_layout(c);
    if (rc != MSTMG_OK) return fail(rc);
    *out = c;
    return MSTMG_OK;
}

extern "C" void mstmg_ctx_destroy(mstmg_ctx* c)
{
    if (!c) return;
    DevBuf<double>* d[] = {&c->pos, &c->rad, &c->ri, &c->qext, &c->qabs, &c->op64, &c->vcc, &c->fnr, &c->rfnr,
                           &c->bcofd, &c->part, &c->qeff, &c->qtot, &c->small};
    for (auto* b : d) b->release();
    DevBuf<int>* ib[] = {&c->d_order, &c->d_offset, &c->d_mie_offset, &c->slot, &c->slot_full, &c->err};
    for (auto* b : ib) b->release();
    DevBuf<zd>* zb[] = {&c->an, &c->an_inv, &c->X64, &c->Y64, &c->pmnp, &c->amnp, &c->pw0, &c->drot, &c->vec64, &c->bvec64};
    for (auto* b : zb) b->release();
    DevBuf<zf>* fb[] = {&c->X32, &c->Y32, &c->vec32, &c->rvec32};
    for (auto* b : fb) b->release();
    c->an32.release();
    c->op32.release();
    c->pairs.release();
    c->tiles.release();
    c->opoff.release();
    c->sc.release();
    if (c->h_sc) cudaFreeHost(c->h_sc);
    if (c->h_small) cudaFreeHost(c->h_small);
    for (auto& p : c->pending) { c->ev_pool.push_back(p.a); c->ev_pool.push_back(p.b); }
    for (auto ev : c->ev_pool) cudaEventDestroy(ev);
    if (c->own_st) cudaStreamDestroy(c->own_st);
    delete c;
}

extern "C" int mstmg_ctx_set_positions(mstmg_ctx* c, const double* pos)
{
    if (!c || !pos) return MSTMG_ERR_ARG;
    if (int rh = reject_hosts(c, "mstmg_ctx_set_positions")) return rh;
    if (!is_dev(pos))
        for (int k = 0; k < 3 * c->n; k++)
            if (!std::isfinite(pos[k])) {
                set_err("mstmg_ctx_set_positions: non-finite position of sphere " + std::to_string(k / 3 + 1));
                return MSTMG_ERR_ARG;
            }
    {
        // spheres moved inside others would need the host-sphere layout: a new context
        std::vector<double> hp;
        const double* p = pos;
        if (is_dev(pos)) {
            hp.resize(3 * (size_t)c->n);
            CK(cudaMemcpy(hp.data(), pos, sizeof(double) * 3 * c->n, cudaMemcpyDeviceToHost));
            p = hp.data();
        }
        if (any_host(c, p)) {
            set_err("mstmg_ctx_set_positions: a sphere's centre would lie inside another sphere (host spheres): create a new context");
            return MSTMG_ERR_UNSUPPORTED;
        }
    }
    CK(copy_in(c->pos.p, pos, sizeof(double) * 3 * c->n, c->st));
    if (is_dev(pos)) CK(cudaMemcpy(c->hpos.data(), pos, sizeof(double) * 3 * c->n, cudaMemcpyDeviceToHost));
    else memcpy(c->hpos.data(), pos, sizeof(double) * 3 * c->n);
    c->ops64_ready = c->ops32_ready = false;
    if (c->tc_state == 1) c->tc_state = 0;
    if (c->fft && c->fft->on) {
        c->fft->drop_plans();
        c->fft->on = false;
        return fft_build(c);
    }
    return MSTMG_OK;
}

extern "C" int mstmg_set_pair_shard(mstmg_ctx* c, int shard, int nshards)
{
    if (!c || nshards < 1 || shard < 0 || shard >= nshards) return MSTMG_ERR_ARG;
    if (int rc0 = reject_ensemble(c, "mstmg_set_pair_shard")) return rc0;
    if (nshards > 1)
        if (int rh = reject_hosts(c, "mstmg_set_pair_shard")) return rh;
    if (nshards > 1 && (!c->tiled || c->ndense > 0)) {
        set_err("mstmg_set_pair_shard: shards are tiles of pairs of one sphere order (no dense pairs)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    c->shard = shard;
    c->nshards = nshards;
    if (c->tc_state == 1) c->tc_state = 0;   // the tensor-core images cover every pair
    return apply_shard(c);
}

extern "C" int mstmg_neqns(const mstmg_ctx* c) { return c ? c->neqns : 0; }
extern "C" int mstmg_npairs(const mstmg_ctx* c) { return c ? c->npairs : 0; }
extern "C" double mstmg_vol_radius(const mstmg_ctx* c) { return c ? c->xg : 0.0; }

extern "C" int mstmg_sphere_orders(const mstmg_ctx* c, int* order, int* offset)
{
    if (!c) return MSTMG_ERR_ARG;
    if (order) memcpy(order, c->order.data(), sizeof(int) * c->n);
    if (offset) memcpy(offset, c->offset.data(), sizeof(int) * (c->n + 1));
    return MSTMG_OK;
}

extern "C" int mstmg_mie_coefficients(const mstmg_ctx* c, double* an, double* qext, double* qabs)
{
    if (!c) return MSTMG_ERR_ARG;
    if (an) CK(copy_out(an, c->an.p, sizeof(zd) * c->mie_offset[c->n], c->st));
    if (qext) CK(copy_out(qext, c->qext.p, sizeof(double) * c->n, c->st));
    if (qabs) CK(copy_out(qabs, c->qabs.p, sizeof(double) * c->n, c->st));
    CK(cudaStreamSynchronize(c->st));
    return MSTMG_OK;
}

extern "C" int mstmg_host_spheres(const mstmg_ctx* c, int* host)
{
    if (!c) return MSTMG_ERR_ARG;
    if (host)
        for (int i = 0; i < c->n; i++) host[i] = c->hs.on() ? c->hs.host[i] : -1;
    return c->hs.nhosted;
}

extern "C" int mstmg_host_mie_coefficients(const mstmg_ctx* c, double* dn, double* un, double* vn)
{
    if (!c) return MSTMG_ERR_ARG;
    const size_t nt = (size_t)c->mie_offset[c->n];
    double* out[3] = {dn, un, vn};
    const zd* src[3] = {c->hs.dn.p, c->hs.un.p, c->hs.vn.p};
    for (int k = 0; k < 3; k++) {
        if (!out[k]) continue;
        if (c->hs.on()) CK(copy_out(out[k], src[k], sizeof(zd) * nt, c->st));
        else memset(out[k], 0, sizeof(zd) * nt);
    }
    CK(cudaStreamSynchronize(c->st));
    return MSTMG_OK;
}

extern "C" int mstmg_set_stream(mstmg_ctx* c, void* stream)
{
    if (!c) return MSTMG_ERR_ARG;
    CK(cudaStreamSynchronize(c->st));
    c->st = stream ? (cudaStream_t)stream : c->own_st;
    return MSTMG_OK;
}

extern "C" int mstmg_set_timing(mstmg_ctx* c, int enable)
{
    if (!c) return MSTMG_ERR_ARG;
    CK(cudaStreamSynchronize(c->st));
    resolve_timing(c);
    c->timing = enable != 0;
    for (int k = 0; k < 3; k++) {
        c->kt_ms[k] = 0.0;
        c->kt_n[k] = 0;
    }
    return MSTMG_OK;
}

extern "C" int mstmg_kernel_time(mstmg_ctx* c, double* ms64, int* n64, double* ms32, int* n32)
{
    if (!c) return MSTMG_ERR_ARG;
    CK(cudaStreamSynchronize(c->st));
    resolve_timing(c);
    if (ms64) *ms64 = c->kt_ms[0];
    if (n64) *n64 = c->kt_n[0];
    if (ms32) *ms32 = c->kt_ms[1];
    if (n32) *n32 = c->kt_n[1];
    for (int k = 0; k < 2; k++) {
        c->kt_ms[k] = 0.0;
        c->kt_n[k] = 0;
    }
    return MSTMG_OK;
}

extern "C" int mstmg_kernel_time_tc(mstmg_ctx* c, double* ms, int* n)
{
    if (!c) return MSTMG_ERR_ARG;
    CK(cudaStreamSynchronize(c->st));
    resolve_timing(c);
    if (ms) *ms = c->kt_ms[2];
    if (n) *n = c->kt_n[2];
    c->kt_ms[2] = 0.0;
    c->kt_n[2] = 0;
    return MSTMG_OK;
}

extern "C" long long mstmg_kernel_launches(void) { return launch_counter().load(); }

// One translation pass over nrhs columns laid out as BiCG packs them
// ([p, A^T conj w] pairs, odd columns conjugate-transpose products), timed with
// CUDA events on the context's stream (mean of reps after one warm-up).
extern "C" int mstmg_selftest_bounded_wait(int device, int limit, int* status)
{
    if (!status || limit < 1 || limit > (1 << 22)) {
        set_err("mstmg_selftest_bounded_wait: bad arguments (limit 1..4194304)");
        return MSTMG_ERR_ARG;
    }
    CK(cudaSetDevice(device));
    int* d = nullptr;
    CK(cudaMalloc((void**)&d, sizeof(int)));
    int h = 0;
    cudaError_t e = cudaMemset(d, 0, sizeof(int));
    if (e == cudaSuccess) {
        launch_wait_selftest(limit, d, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    CK(e);
    *status = h;
    return MSTMG_OK;
}

