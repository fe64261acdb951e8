// capi.cu -- the C ABI (include/mstm_b200.h): context set-up, the translation
// matvec driver (sphereinteraction), the device BiCG (cbicg), the
// fixed-orientation solve (fixedorsoln) and its mixed-precision variant.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include "../../include/mstm_b200.h"
#include "common.cuh"
#include "kernels.cuh"
#include "bicg.cuh"
#include "sphere_kernels.cuh"
#include "tables.h"
#include "translate_tiled.cuh"
#include "postproc.cuh"

static thread_local std::string g_err;
static void set_err(const std::string& s) { g_err = s; }
void mstmg_internal_set_error(const std::string& msg) { set_err(msg); }

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            set_err(std::string(#call) + ": " + cudaGetErrorString(e_));                          \
            return MSTMG_ERR_CUDA;                                                                \
        }                                                                                         \
    } while (0)

template <typename T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count)
    {
        if (count <= n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc((void**)&p, sizeof(T) * (count ? count : 1));
        if (e == cudaSuccess) n = count;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

template <typename T> struct BicgVecs {
    cpx<T>*x, *r, *p, *w, *q, *cap, *caw;
};

struct mstmg_ctx {
    int dev = 0, nsm = 148;
    cudaStream_t st = nullptr;
    mstmg_opts opts;
    int n = 0, neqns = 0, lmax = 0, npairs = 0, maxrec = 0;
    long long op_units = 0;
    double xg = 1.0;
    std::vector<int> order, offset, mie_offset;
    std::vector<double> radius;
    std::vector<double> hpos;   // host copy of the positions (cluster origin)
    DevBuf<double> pos, rad, ri, qext, qabs;
    DevBuf<int> d_order, d_offset, d_mie_offset, slot, slot_full;
    DevBuf<zd> an, an_inv;
    DevBuf<float> an32;
    DevBuf<int2> pairs;
    DevBuf<long long> opoff;
    DevBuf<int4> tiles;
    int ntiles = 0;
    bool tiled = false;   // monodisperse cluster: pairs stored in tile order for the fast kernel
    DevBuf<double> op64;
    DevBuf<float> op32;
    bool ops64_ready = false, ops32_ready = false;
    DevBuf<double> vcc, fnm1, fnc, fnp1, fnr, bcofd;
    int vn = 0;
    DevBuf<int> err;
    DevBuf<zd> X64, Y64, pmnp, amnp, pw0, drot, vec64, bvec64;
    DevBuf<zf> X32, Y32, vec32, rvec32;
    DevBuf<double> part, qeff, qtot, small;
    DevBuf<BicgScalars> sc;
    BicgScalars* h_sc = nullptr;
    double* h_small = nullptr;
    int iters[2] = {0, 0}, outer = 0, passes64 = 0, passes32 = 0;
    cudaStream_t own_st = nullptr;
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    struct Pending { cudaEvent_t a, b; int prec; };
    std::vector<Pending> pending;
    double kt_ms[2] = {0.0, 0.0};
    int kt_n[2] = {0, 0};
    SlotMaps sm() const { return SlotMaps{neqns / 2, slot.p, d_order.p, d_offset.p, d_mie_offset.p}; }
};

static bool is_dev(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static cudaError_t copy_in(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
    return cudaMemcpyAsync(dst, src, bytes, is_dev(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
}
static cudaError_t copy_out(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
    return cudaMemcpyAsync(dst, src, bytes, is_dev(dst) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st);
}

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
}

extern "C" const char* mstmg_last_error(void) { return g_err.c_str(); }

// Fold completed translation-kernel event pairs into the running totals.
static void resolve_timing(mstmg_ctx* c)
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

static int check_kernel_err(mstmg_ctx* c)
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

static int setup_layout(mstmg_ctx* c)
{
    const int n = c->n;
    c->offset.assign(n + 1, 0);
    c->mie_offset.assign(n + 1, 0);
    int lm = 0, lmin = 1 << 30;
    long long ne = 0, nt = 0;
    for (int i = 0; i < n; i++) {
        int L = c->order[i];
        c->offset[i] = (int)ne;
        c->mie_offset[i] = (int)nt;
        ne += 2LL * L * (L + 2);
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
    if (n > 1 && lmin < c->opts.translation_switch_order) {
        set_err("pairs with min order below translation_switch_order use MSTM's dense gentranmatrix path, "
                "which this library does not implement");
        return MSTMG_ERR_UNSUPPORTED;
    }
    c->neqns = (int)ne;
    c->lmax = lm;
    CK(c->d_order.alloc(n));
    CK(c->d_offset.alloc(n + 1));
    CK(c->d_mie_offset.alloc(n + 1));
    CK(cudaMemcpyAsync(c->d_order.p, c->order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_offset.p, c->offset.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_mie_offset.p, c->mie_offset.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, c->st));
    // slot maps
    std::vector<int> slot(ne / 2), slotf(ne);
    for (int i = 0; i < n; i++) {
        int L = c->order[i], hb = L * (L + 2);
        for (int k = 0; k < hb; k++) slot[c->offset[i] / 2 + k] = i;
        for (int k = 0; k < 2 * hb; k++) slotf[c->offset[i] + k] = i;
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
    launch_mie_coefs(n, c->rad.p, c->ri.p, c->opts.medium_re, c->opts.medium_im, c->d_order.p, c->d_mie_offset.p, c->an.p,
                     c->an_inv.p, c->an32.p, c->qext.p, c->qabs.p, c->st);
    CK(cudaGetLastError());
    // pair list (i < j, the reference's loop order) and operator offsets
    long long np = (long long)n * (n - 1) / 2;
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
    c->tiled = !c->opts.generic_kernel && (lm == lmin) && tiled_supported(lm, 1) && n > 1 && n < 65536;
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
            for (int i = i0; i < std::min(n, i0 + B); i++)
                for (int j = j0; j < std::min(n, j0 + B); j++)
                    if (i < j) add_pair(i, j);
            int cnt = (int)t - start;
            if (cnt > 0) tl.push_back(make_int4(start, cnt, (i0 << 16) | j0, I == J ? 1 : 0));
        }
    } else {
        std::vector<std::pair<int, int>> pp;
        tournament(n, pp);
        for (auto& ij : pp) add_pair(ij.first, ij.second);
    }
    c->ntiles = (int)tl.size();
    if (c->ntiles > 0) {
        CK(c->tiles.alloc(tl.size()));
        CK(cudaMemcpyAsync(c->tiles.p, tl.data(), sizeof(int4) * tl.size(), cudaMemcpyHostToDevice, c->st));
    }
    if (t != np) {
        set_err("internal error: pair schedule incomplete");
        return MSTMG_ERR_ARG;
    }
    c->op_units = u;
    c->maxrec = maxrec;
    if (np > 0) {
        CK(c->pairs.alloc(np));
        CK(c->opoff.alloc(np));
        CK(cudaMemcpyAsync(c->pairs.p, pr.data(), sizeof(int2) * np, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(c->opoff.p, off.data(), sizeof(long long) * np, cudaMemcpyHostToDevice, c->st));
    }
    // constant tables
    mstmg::Tables tb(6 * lm + 6);
    std::vector<double> vcc, f1, f2, f3;
    tb.axial_constants(lm, vcc, f1, f2, f3);
    c->vn = lm;
    std::vector<double> bd(lm + 2, 0.0);
    for (int k = 0; k <= lm + 1; k++) bd[k] = tb.bc(k, k);
    CK(c->vcc.alloc(vcc.size()));
    CK(c->fnm1.alloc(f1.size()));
    CK(c->fnc.alloc(f2.size()));
    CK(c->fnp1.alloc(f3.size()));
    CK(c->fnr.alloc(tb.fnr.size()));
    CK(c->bcofd.alloc(bd.size()));
    CK(cudaMemcpyAsync(c->vcc.p, vcc.data(), sizeof(double) * vcc.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->fnm1.p, f1.data(), sizeof(double) * f1.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->fnc.p, f2.data(), sizeof(double) * f2.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->fnp1.p, f3.data(), sizeof(double) * f3.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->fnr.p, tb.fnr.data(), sizeof(double) * tb.fnr.size(), cudaMemcpyHostToDevice, c->st));
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
    // vol_radius as main_calling_program forms it: (sum r^3)**.333333 (single-precision literal)
    double v = 0.0;
    for (int i = 0; i < n; i++) v = v + c->radius[i] * c->radius[i] * c->radius[i];
    c->xg = std::pow(v, (double)0.333333f);
    CK(cudaStreamSynchronize(c->st));
    return MSTMG_OK;
}

extern "C" int mstmg_ctx_create(mstmg_ctx** out, int nsphere, const double* pos, const double* radius, const double* ref_index,
                                double mie_epsilon, const mstmg_opts* opts)
{
    if (!out || nsphere < 1 || !pos || !radius || !ref_index) {
        set_err("mstmg_ctx_create: bad arguments");
        return MSTMG_ERR_ARG;
    }
    *out = nullptr;
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
    // sphere orders on the device (mieoa order test), read back for the layout
    DevBuf<int> ord;
    if (ord.alloc(nsphere)) return fail(MSTMG_ERR_CUDA);
    launch_mie_orders(nsphere, c->rad.p, c->ri.p, c->opts.medium_re, c->opts.medium_im, mie_epsilon, ord.p, c->st);
    c->order.assign(nsphere, 0);
    if (cudaMemcpyAsync(c->order.data(), ord.p, sizeof(int) * nsphere, cudaMemcpyDeviceToHost, c->st) ||
        cudaStreamSynchronize(c->st)) {
        set_err("mie order kernel failed");
        ord.release();
        return fail(MSTMG_ERR_CUDA);
    }
    ord.release();
    rc = setup_layout(c);
    if (rc != MSTMG_OK) return fail(rc);
    *out = c;
    return MSTMG_OK;
}

extern "C" void mstmg_ctx_destroy(mstmg_ctx* c)
{
    if (!c) return;
    DevBuf<double>* d[] = {&c->pos, &c->rad, &c->ri, &c->qext, &c->qabs, &c->op64, &c->vcc, &c->fnm1, &c->fnc, &c->fnp1, &c->fnr,
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
    CK(copy_in(c->pos.p, pos, sizeof(double) * 3 * c->n, c->st));
    if (is_dev(pos)) CK(cudaMemcpy(c->hpos.data(), pos, sizeof(double) * 3 * c->n, cudaMemcpyDeviceToHost));
    else memcpy(c->hpos.data(), pos, sizeof(double) * 3 * c->n);
    c->ops64_ready = c->ops32_ready = false;
    return MSTMG_OK;
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

// ---------------------------------------------------------------------------
// operators and the translation pass
// ---------------------------------------------------------------------------
// Generate the stored pair operators.  want64 / want32 select the FP64 and
// FP32 records; both come out of one pass of the generator when both are due.
static int ensure_ops_both(mstmg_ctx* c, bool want64, bool want32, bool force)
{
    if (c->npairs == 0) return MSTMG_OK;
    bool need64 = want64 && (force || !c->ops64_ready);
    bool need32 = want32 && (force || !c->ops32_ready);
    if (!need64 && !need32) return MSTMG_OK;
    if (need64) CK(c->op64.alloc(c->op_units));
    if (need32) CK(c->op32.alloc(c->op_units));
    OpGenArgs a;
    a.npairs = c->npairs;
    a.pairs = c->pairs.p;
    a.pos = c->pos.p;
    a.order = c->d_order.p;
    a.opoff = c->opoff.p;
    a.op64 = need64 ? c->op64.p : nullptr;
    a.op32 = need32 ? c->op32.p : nullptr;
    a.vcc = c->vcc.p;
    a.vnmax = c->vn;
    a.fnm1 = c->fnm1.p;
    a.fnc = c->fnc.p;
    a.fnp1 = c->fnp1.p;
    a.fnr = c->fnr.p;
    a.bcofd = c->bcofd.p;
    a.rimed_re = c->opts.medium_re;
    a.rimed_im = c->opts.medium_im;
    a.err = c->err.p;
    launch_opgen(a, c->nsm, c->st);
    CK(cudaGetLastError());
    if (need64) c->ops64_ready = true;
    if (need32) c->ops32_ready = true;
    return MSTMG_OK;
}
static int ensure_ops(mstmg_ctx* c, int prec, bool force) { return ensure_ops_both(c, prec == 0, prec == 1, force); }

template <typename T> static const T* ops_ptr(mstmg_ctx* c);
template <> const double* ops_ptr<double>(mstmg_ctx* c) { return c->op64.p; }
template <> const float* ops_ptr<float>(mstmg_ctx* c) { return c->op32.p; }

// y[:, 0:nrhs] = H x[:, 0:nrhs]  (y zeroed here)
template <typename T> static int translate(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int nrhs, unsigned contran)
{
    CK(cudaMemsetAsync(y, 0, sizeof(cpx<T>) * (size_t)c->neqns * nrhs, c->st));
    if (c->npairs == 0) return MSTMG_OK;
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
    a.lmax = c->lmax;
    a.maxrec = c->maxrec;
    a.err = c->err.p;
    TiledArgs<T> ta;
    bool use_tiled = c->tiled && tiled_supported(c->lmax, nrhs);
    if (use_tiled) {
        ta.ntiles = c->ntiles;
        ta.tiles = c->tiles.p;
        ta.pairs = c->pairs.p;
        ta.ops = ops_ptr<T>(c);
        ta.x = x;
        ta.y = y;
        ta.ld = c->neqns;
        ta.nrhs = nrhs;
        ta.nsph = c->n;
        ta.contran = contran;
        ta.err = c->err.p;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->timing) {
        for (cudaEvent_t* ev : {&e0, &e1}) {
            if (!c->ev_pool.empty()) { *ev = c->ev_pool.back(); c->ev_pool.pop_back(); }
            else CK(cudaEventCreate(ev));
        }
        CK(cudaEventRecord(e0, c->st));
    }
    if (!use_tiled || launch_translate_tiled<T>(ta, c->lmax, c->nsm, c->st) != 0) launch_translate<T>(a, c->nsm, c->st);
    CK(cudaGetLastError());
    if (c->timing) {
        CK(cudaEventRecord(e1, c->st));
        c->pending.push_back({e0, e1, sizeof(T) == 8 ? 0 : 1});
    }
    if (sizeof(T) == 8) c->passes64++;
    else c->passes32++;
    return MSTMG_OK;
}

extern "C" int mstmg_interaction(mstmg_ctx* c, int nrhs, const double* ain, double* aout, const int* con_tran, const int* mie_mult,
                                 int initial_run)
{
    if (!c || nrhs < 1 || nrhs > 4 || !ain || !aout) {
        set_err("mstmg_interaction: bad arguments (nrhs must be 1..4)");
        return MSTMG_ERR_ARG;
    }
    int rc = ensure_ops(c, 0, initial_run != 0);
    if (rc) return rc;
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    unsigned mask = 0;
    CK(copy_in(c->X64.p, ain, sizeof(zd) * (size_t)ne * nrhs, c->st));
    for (int r = 0; r < nrhs; r++) {
        int ct = con_tran ? con_tran[r] : 0;
        int mm = mie_mult ? mie_mult[r] : 1;
        zd* col = c->X64.p + (size_t)r * ne;
        if (ct) {
            mask |= 1u << r;
            if (mm) launch_mie<double>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, c->an.p, -1, 1, col, col, c->st);
            else launch_conj_copy<double>(ne, col, col, c->st);
        }
    }
    rc = translate<double>(c, c->X64.p, c->Y64.p, nrhs, mask);
    if (rc) return rc;
    for (int r = 0; r < nrhs; r++) {
        int ct = con_tran ? con_tran[r] : 0;
        int mm = mie_mult ? mie_mult[r] : 1;
        zd* col = c->Y64.p + (size_t)r * ne;
        if (!ct) {
            if (mm) launch_mie<double>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, c->an.p, 1, 0, col, col, c->st);
        } else {
            launch_conj_copy<double>(ne, col, col, c->st);
        }
    }
    CK(cudaGetLastError());
    CK(copy_out(aout, c->Y64.p, sizeof(zd) * (size_t)ne * nrhs, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_kernel_err(c);
}

// ---------------------------------------------------------------------------
// Batched BiCG: S independent systems advance in lockstep, sharing one
// translation pass per iteration ([p_1, w_1, p_2, w_2, ...], the w columns as
// conjugate-transpose products).  With S = 1 this is cbicg's single-rank
// iteration (mstm-solver-8.f90:828-947) step for step.
//   have_x0: the initial residual is b - A x0 (one extra pass); otherwise x0 = 0.
// ---------------------------------------------------------------------------
template <typename T>
static int bicg_batched(mstmg_ctx* c, int S, const cpx<T>* const* b, BicgVecs<T>* v, bool have_x0, int niter, const double* eps,
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
    for (int s = 0; s < S; s++) {
        if (!have_x0) CK(cudaMemsetAsync(v[s].x, 0, sizeof(cpx<T>) * ne, c->st));
        launch_init<T>(sm, an, b[s], v[s].x, Y + (size_t)s * ne, have_x0 ? 1 : 0, v[s].r, v[s].p, v[s].w, v[s].q, part, c->sc.p + s, 1,
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
            launch_mie<T>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, an, -1, 1, v[s].w, X + (size_t)(2 * k + 1) * ne, c->st);
            mask |= 2u << (2 * k);
        }
        rc = translate<T>(c, X, Y, 2 * a, mask);
        if (rc) return rc;
        for (int k = 0; k < a; k++) {
            int s = slots[k];
            launch_post<T>(sm, an, v[s].p, v[s].w, Y + (size_t)(2 * k) * ne, Y + (size_t)(2 * k + 1) * ne, v[s].cap, v[s].caw, part,
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

extern "C" int mstmg_bicg(mstmg_ctx* c, int niter, double eps, const double* pnp, double* anp, int initialize, int* iter, double* err)
{
    if (!c || !pnp || !anp) return MSTMG_ERR_ARG;
    int rc = ensure_ops(c, 0, initialize != 0);
    if (rc) return rc;
    const int ne = c->neqns;
    BicgVecs<double> v = vecs_at<double>(c->vec64.p, ne, 0);
    CK(copy_in(c->bvec64.p, pnp, sizeof(zd) * ne, c->st));
    CK(copy_in(v.x, anp, sizeof(zd) * ne, c->st));
    const zd* bb[1] = {c->bvec64.p};
    int it = 0, st = 0;
    double e = 0.0;
    if (niter <= 0) {
        set_err("mstmg_bicg: niter must be positive (MSTM's niter<=0 modes are not on this path)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    rc = bicg_batched<double>(c, 1, bb, &v, true, niter, &eps, &it, &e, &st);
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
    launch_planewave(alpha, sinc, dir, c->lmax, c->neqns, c->slot_full.p, c->d_order.p, c->d_offset.p, c->pos.p, c->pw0.p, c->drot.p,
                     c->pmnp.p, c->st);
    CK(cudaGetLastError());
    CK(copy_out(pmnp, c->pmnp.p, sizeof(zd) * 2 * (size_t)c->neqns, c->st));
    CK(cudaStreamSynchronize(c->st));
    return MSTMG_OK;
}

// Mixed precision: FP64 outer refinement around FP32 inner BiCG, both
// polarisations at once.  x (FP64, 2 systems) starts at the Mie solution.
static int solve_mixed(mstmg_ctx* c, zd* const* b, zd* const* x, double eps, int niter, int* iters, double* errs, int* status)
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

extern "C" int mstmg_fixed_orientation(mstmg_ctx* c, double alpha, double sinc, int dir, double eps, int niter, double* amnp,
                                       double* qeff, double* qtot, double* maxerr, int* maxiter)
{
    if (!c || !amnp) return MSTMG_ERR_ARG;
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
    c->passes64 = c->passes32 = 0;
    c->outer = 0;
    // operators are (re)generated for this configuration: the reference's initial_run
    int rc = ensure_ops_both(c, true, c->opts.precision == MSTMG_PRECISION_MIXED, true);
    if (rc) return rc;
    launch_planewave(alpha, sinc, dir, c->lmax, ne, c->slot_full.p, c->d_order.p, c->d_offset.p, c->pos.p, c->pw0.p, c->drot.p,
                     c->pmnp.p, c->st);
    zd* bvec = c->bvec64.p;   // pmnpan for both polarisations: 2 x ne
    for (int p = 0; p < 2; p++)
        launch_mie<double>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, c->an.p, 1, 0, c->pmnp.p + (size_t)p * ne,
                           bvec + (size_t)p * ne, c->st);
    CK(cudaGetLastError());
    int istat = 0;
    int it[2] = {0, 0}, st[2] = {0, 0};
    double er[2] = {0.0, 0.0};
    if (niter == 0) {
        for (int p = 0; p < 2; p++)
            CK(cudaMemcpyAsync(c->amnp.p + (size_t)p * ne, bvec + (size_t)p * ne, sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
    } else if (c->opts.precision == MSTMG_PRECISION_MIXED) {
        zd* xs[2] = {c->amnp.p, c->amnp.p + ne};
        zd* bs[2] = {bvec, bvec + ne};
        for (int p = 0; p < 2; p++) CK(cudaMemcpyAsync(xs[p], bs[p], sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
        rc = solve_mixed(c, bs, xs, eps, niter, it, er, st);
        if (rc) return rc;
    } else {
        // the reference's order: polarisation 1 then 2, each from x0 = Mie*f
        for (int p = 0; p < 2; p++) {
            BicgVecs<double> v = vecs_at<double>(c->vec64.p, ne, 0);
            CK(cudaMemcpyAsync(v.x, bvec + (size_t)p * ne, sizeof(zd) * ne, cudaMemcpyDeviceToDevice, c->st));
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
    launch_qeff(c->n, c->d_order.p, c->d_offset.p, c->d_mie_offset.p, c->rad.p, mk(c->opts.medium_re, c->opts.medium_im), c->an_inv.p,
                c->amnp.p, c->pmnp.p, ne, c->qeff.p, c->xg, c->qtot.p, c->st);
    CK(cudaGetLastError());
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
    if (stored) *stored = (double)c->op_units * es;
    if (canonical) {
        double s = 0.0;
        for (int i = 0; i < c->n - 1; i++)
            for (int j = i + 1; j < c->n; j++) {
                int a = c->order[i], b = c->order[j], nmn = std::min(a, b), nmx = std::max(a, b);
                s += (2.0 * nmn + 1) * (nmx * (nmx + 2) + 1) * es + atcdim_h(a, b) * 2 * es + (2.0 * nmx + 1) * 2 * es;
            }
        *canonical = s;
    }
    return MSTMG_OK;
}

// ---------------------------------------------------------------------------
// Scattering post-processing of a solution (main_calling_program,
// mstm-input-37.f90:1159-1197 and 1497-1532): translation orders and
// t_matrix_order, merge to the common origin, GSF expansion, azimuth-averaged
// scattering matrix on nangles polar angles 0..180 deg, and g.
// ---------------------------------------------------------------------------
extern "C" int mstmg_scattering(mstmg_ctx* c, const double* amnp, double trans_eps, int max_t_order, int nangles, double* smat,
                                double* g, int* t_matrix_order, double* amnp0, int amnp0_cap)
{
    if (!c || !amnp || nangles < 2 || max_t_order < 1) {
        set_err("mstmg_scattering: bad arguments");
        return MSTMG_ERR_ARG;
    }
    const int n = c->n, L = c->lmax;
    const int NBC = 420;
    // cluster origin: mean position of the external spheres
    double r0[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) r0[k] = r0[k] + c->hpos[3 * (size_t)i + k];
    for (int k = 0; k < 3; k++) r0[k] = r0[k] / (double)n;
    static thread_local mstmg::Tables* big = nullptr;
    if (!big) big = new mstmg::Tables(NBC);
    DevBuf<double> dbc, dfnr;
    CK(dbc.alloc(big->bcof.size()));
    CK(dfnr.alloc(big->fnr.size()));
    CK(cudaMemcpyAsync(dbc.p, big->bcof.data(), sizeof(double) * big->bcof.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(dfnr.p, big->fnr.data(), sizeof(double) * big->fnr.size(), cudaMemcpyHostToDevice, c->st));
    // translation orders (tranordertest) on the device
    DevBuf<int> dtord;
    DevBuf<zd> tscr;
    const int sstride = 3 * (200 + MSTMG_LMAX + 4);
    CK(dtord.alloc(n));
    CK(tscr.alloc((size_t)n * sstride));
    launch_tranorder(n, c->pos.p, c->d_order.p, r0, c->opts.medium_re, trans_eps, max_t_order, dbc.p, dfnr.p, NBC, tscr.p, sstride,
                     dtord.p, c->st);
    std::vector<int> tord(n);
    CK(cudaMemcpyAsync(tord.data(), dtord.p, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int T = std::min(L, max_t_order);
    for (int i = 0; i < n; i++) T = std::max(T, tord[i]);
    if (T > 200) {
        set_err("mstmg_scattering: t_matrix_order above 200 is not supported");
        return MSTMG_ERR_UNSUPPORTED;
    }
    // axial constants for regular translation up to order T (host, FP64)
    std::vector<double> vcc((size_t)T * L * (L + 2) * (T + L + 1), 0.0), f1, f2, f3, vc1(2 * (T + L) + 4), vc2(2 * (T + L) + 4);
    for (int nn = 1; nn <= T; nn++)
        for (int l = 1; l <= L; l++) {
            double c1 = big->fnr[nn + nn + 1] * big->fnr[l + l + 1];
            big->vcfunc(-1, nn, 1, l, vc2.data());
            int wmin = std::abs(nn - l), wmax = nn + l, nlmin = std::min(l, nn);
            for (int m = -nlmin; m <= nlmin; m++) {
                int ml = l * (l + 1) + m;
                double c2 = -c1 * ((m & 1) ? -1.0 : 1.0);
                big->vcfunc(-m, nn, m, l, vc1.data());
                for (int w = wmin; w <= wmax; w++) {
                    int e = ((nn - l + w) % 4 + 4) % 4;
                    double ri = (e == 0 || e == 1) ? 1.0 : -1.0;
                    vcc[(size_t)(nn - 1) + (size_t)T * ((size_t)(ml - 1) + (size_t)L * (L + 2) * w)] = c2 * vc1[w] * vc2[w] * ri;
                }
            }
        }
    int FN = std::max(T, L);
    {
        std::vector<double> tmpv;
        mstmg::Tables small(6 * FN + 6 < NBC ? 6 * FN + 6 : NBC);
        size_t nf = (size_t)(2 * FN + 1) * FN;
        f1.assign(nf, 0.0);
        f2.assign(nf, 0.0);
        f3.assign(nf, 0.0);
        const std::vector<double>& fr = big->fnr;
        for (int m = -FN; m <= FN; m++)
            for (int l = std::max(1, std::abs(m)); l <= FN; l++) {
                size_t ix = (size_t)(m + FN) + (2 * FN + 1) * (size_t)(l - 1);
                int lp1 = l + 1, lm1 = l - 1;
                f1[ix] = fr[lm1] * fr[lp1] * fr[l - m] * fr[l + m] / fr[lm1 + l] / fr[l + lp1] / (double)l;
                f2[ix] = (double)m / (double)l / (double)lp1;
                f3[ix] = fr[l] * fr[l + 2] * fr[lp1 - m] * fr[lp1 + m] / fr[l + lp1] / fr[l + l + 3] / (double)lp1;
            }
    }
    DevBuf<double> dvcc, df1, df2, df3, dbcd;
    CK(dvcc.alloc(vcc.size()));
    CK(df1.alloc(f1.size()));
    CK(df2.alloc(f2.size()));
    CK(df3.alloc(f3.size()));
    std::vector<double> bd(T + L + 4);
    for (int k = 0; k < (int)bd.size(); k++) bd[k] = big->bc(k, k);
    CK(dbcd.alloc(bd.size()));
    CK(cudaMemcpyAsync(dvcc.p, vcc.data(), sizeof(double) * vcc.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(df1.p, f1.data(), sizeof(double) * f1.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(df2.p, f2.data(), sizeof(double) * f2.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(df3.p, f3.data(), sizeof(double) * f3.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(dbcd.p, bd.data(), sizeof(double) * bd.size(), cudaMemcpyHostToDevice, c->st));
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
    MergeArgs ma;
    ma.nsph = n;
    ma.pos = c->pos.p;
    ma.order = c->d_order.p;
    ma.offset = c->d_offset.p;
    ma.tord = dtord.p;
    ma.T = T;
    ma.r0[0] = r0[0];
    ma.r0[1] = r0[1];
    ma.r0[2] = r0[2];
    ma.rimed_re = c->opts.medium_re;
    ma.rimed_im = c->opts.medium_im;
    ma.amnp = dsrc.p;
    ma.ld = ne;
    ma.npol = 2;
    ma.amnp0 = da0.p;
    ma.ld0 = nb0;
    ma.vcc = dvcc.p;
    ma.vcT = T;
    ma.vcML = L * (L + 2);
    ma.fnm1 = df1.p;
    ma.fnc = df2.p;
    ma.fnp1 = df3.p;
    ma.fcN = FN;
    ma.fnr = dfnr.p;
    ma.bcofd = dbcd.p;
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
    launch_fosm(T, da0.p, dbc.p, dfnr.p, NBC, ds.p, ds.p + 16 * W, ds.p + 32 * W, ds.p + 48 * W, fscr.p, c->st);
    CK(cscr.alloc(fosmcalc_scratch_doubles(T, nangles)));
    CK(dsm.alloc(16 * (size_t)nangles));
    launch_fosmcalc(T, nangles, ds.p, ds.p + 16 * W, ds.p + 32 * W, ds.p + 48 * W, dfnr.p, dbcd.p, cscr.p, dsm.p, c->st);
    CK(cudaGetLastError());
    double s0[2];
    CK(cudaMemcpyAsync(&s0[0], ds.p + 0, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&s0[1], ds.p + 16, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    if (smat) CK(copy_out(smat, dsm.p, sizeof(double) * 16 * (size_t)nangles, c->st));
    if (amnp0 && amnp0_cap >= nb0) CK(copy_out(amnp0, da0.p, sizeof(zd) * 2 * (size_t)nb0, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (g) *g = s0[1] / (3.0 * s0[0]);
    if (t_matrix_order) *t_matrix_order = T;
    dbc.release(); dfnr.release(); dtord.release(); tscr.release(); dvcc.release(); df1.release(); df2.release(); df3.release();
    dbcd.release(); dsrc.release(); da0.release(); mscr.release(); ds.release(); fscr.release(); cscr.release(); dsm.release();
    return check_kernel_err(c);
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
    c->kt_ms[0] = c->kt_ms[1] = 0.0;
    c->kt_n[0] = c->kt_n[1] = 0;
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
    c->kt_ms[0] = c->kt_ms[1] = 0.0;
    c->kt_n[0] = c->kt_n[1] = 0;
    return MSTMG_OK;
}

extern "C" long long mstmg_kernel_launches(void) { return launch_counter().load(); }

extern "C" int mstmg_time_translation(mstmg_ctx* c, int prec, int nrhs, int reps, double* ms)
{
    if (!c || nrhs < 1 || nrhs > 4 || reps < 1) return MSTMG_ERR_ARG;
    int rc = ensure_ops(c, prec, false);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    unsigned mask = (nrhs >= 2) ? 0xAu : 0u;
    // warm-up
    if (prec == 0) rc = translate<double>(c, c->X64.p, c->Y64.p, nrhs, mask);
    else rc = translate<float>(c, c->X32.p, c->Y32.p, nrhs, mask);
    if (rc) return rc;
    CK(cudaEventRecord(e0, c->st));
    for (int k = 0; k < reps; k++) {
        if (prec == 0) rc = translate<double>(c, c->X64.p, c->Y64.p, nrhs, mask);
        else rc = translate<float>(c, c->X32.p, c->Y32.p, nrhs, mask);
        if (rc) return rc;
    }
    CK(cudaEventRecord(e1, c->st));
    CK(cudaEventSynchronize(e1));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = t / reps;
    return check_kernel_err(c);
}
