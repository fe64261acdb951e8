// capi.cu -- the C ABI (include/mstm_b200.h): context set-up, the translation
// matvec driver (sphereinteraction), the device BiCG (cbicg), the
// fixed-orientation solve (fixedorsoln) and its mixed-precision variant.
#include <algorithm>
#include <complex>
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
#include "mrhs.cuh"
#include "ranorient.cuh"
#include "fftpath.cuh"
#include "densepair.cuh"
#include "tcpass.cuh"
#include <nvtx3/nvToolsExt.h>
#include <cufft.h>
#include <map>
#include <memory>
#include <type_traits>

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

// Owning device buffer (freed on destruction, not copyable).
template <typename T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
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

// FFT translation state (fft_translation-5.f90): cells, node translations,
// kernel spectra, cuFFT plans and the node work arrays.
struct FftState {
    bool on = false;
    double fv_in = 0.2, d_in = 0.0;
    int no_in = -1, model_in = 2;
    int No = 0, nbN = 0, cd[3] = {0, 0, 0}, nnb = 0, nbv[81] = {0};
    double dcell = 0.0, cb[3] = {0.0, 0.0, 0.0};
    size_t N8 = 0;
    DevBuf<int> snode, slot;
    DevBuf<long long> joff;
    DevBuf<zd> Jsn64, Jns64, A64, G64;
    DevBuf<zf> Jsn32, Jns32, A32, G32;
    DevBuf<float2> H;
    cufftHandle plan[2][5] = {{0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}};   // [FP64, FP32][columns]
    bool have[2][5] = {{false, false, false, false, false}, {false, false, false, false, false}};
    void drop_plans()
    {
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 5; b++)
                if (have[a][b]) {
                    cufftDestroy(plan[a][b]);
                    have[a][b] = false;
                }
    }
    ~FftState() { drop_plans(); }
};

// NVTX range over a C-ABI call or a pass, visible in Nsight timelines (a
// no-op unless a tool is attached)
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// work vectors of the many-system BiCG (mrhs.cu kernels): S systems in columns
template <typename T> struct MultiWork {
    int S = 0;
    DevBuf<cpx<T>> vec, XP, YP;
    DevBuf<double> part, epsv;
    DevBuf<BicgScalars> sc;
    DevBuf<int> act;
    DevBuf<unsigned> cnt;   // per active position: CTAs done with a reduction (the last one finishes it)
    std::vector<BicgScalars> hsc;
    std::vector<int> hact;
    MultiVecs<T> v(int ne) const
    {
        MultiVecs<T> m;
        cpx<T>* b = vec.p;
        size_t cs = (size_t)ne * S;
        m.X = b;
        m.R = b + cs;
        m.P = b + 2 * cs;
        m.W = b + 3 * cs;
        m.Q = b + 4 * cs;
        m.CAP = b + 5 * cs;
        m.CAW = b + 6 * cs;
        return m;
    }
    // vectors = false: only the packed translation buffers (FP64 residuals of the refinement)
    int init(int S_, int ne, int nsm, bool vectors)
    {
        S = S_;
        int spad = S + 3;
        if (vectors) CK(vec.alloc((size_t)7 * ne * S));
        CK(XP.alloc((size_t)2 * ne * spad));
        CK(YP.alloc((size_t)2 * ne * spad));
        CK(part.alloc((size_t)3 * (4 * nsm + spad)));
        CK(epsv.alloc(S));
        CK(sc.alloc(S));
        CK(act.alloc(S));
        CK(cnt.alloc(S));
        CK(cudaMemset(cnt.p, 0, sizeof(unsigned) * S));
        hsc.resize(S);
        hact.resize(S);
        return MSTMG_OK;
    }
};

// work of the many-system restarted GMRES (mrhs.cu gm_* kernels): basis
// vector i of system s at V + (s (m + 1) + i) ne, up to m steps per cycle
struct GmresWork {
    int S = 0, m = 0, ne = 0;
    DevBuf<zf> V, W, XP, Y, R;
    // h: S squared norms (padded to even), then two Gram-Schmidt passes of (m + 1) S complex
    DevBuf<double> h, rr;
    DevBuf<int> act;
    double* hh = nullptr;   // pinned host copy of the norms and the first pass
    std::vector<std::complex<double>> Rm, g, sn;   // per system: rotated Hessenberg (m x (m + 1)), rhs, rotations
    std::vector<double> cs, target, ybuf;
    std::vector<int> kk;
    std::vector<char> frozen;
    // Arnoldi steps captured as CUDA graphs, keyed by (step j, active
    // systems): kernel launches and passes they hold, replayed with them
    struct StepGraph {
        cudaGraphExec_t exec;
        long long launches;
        int passes32;
    };
    std::map<long long, StepGraph> graphs;
    unsigned long long graph_gen = ~0ull;   // the context's layout generation the graphs were captured at
    bool graphs_ok = true;                  // false once a capture failed: plain launches from then on
    // Arnoldi cycles driven on the device (two-column solves): the state of
    // the rotations in device memory and one graph per active-system count,
    // the step under a conditional WHILE node (mrhs.cu, gm_givens_kernel)
    DevBuf<int> dj, djmax, dalive, dkk, dstatus, dkmax;
    DevBuf<double> dtarget, dcs;
    DevBuf<double2> dsn, dg, dRm;
    int* hkk = nullptr;   // pinned: kk, status of every system and the steps of the last device cycle
    struct CycleGraph {
        cudaGraphExec_t exec;
        long long launches_per_step;
        int passes32_per_step;
    };
    std::map<int, CycleGraph> cycles;
    GmDevState dev() { return GmDevState{dj.p, djmax.p, dalive.p, dkk.p, dstatus.p, dtarget.p, dcs.p, dsn.p, dg.p, dRm.p}; }
    void drop_graphs()
    {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
        graphs.clear();
        for (auto& kv : cycles) cudaGraphExecDestroy(kv.second.exec);
        cycles.clear();
    }
    GmresWork() = default;
    GmresWork(const GmresWork&) = delete;
    GmresWork& operator=(const GmresWork&) = delete;
    ~GmresWork()
    {
        drop_graphs();
        if (hh) cudaFreeHost(hh);
        if (hkk) cudaFreeHost(hkk);
    }
    size_t off1() const { return (size_t)(S + (S & 1)); }
    size_t hpass() const { return (size_t)(m + 1) * S * 2; }
    // basis length from the free device memory: at most `cap` vectors a
    // system (200 when cap is 0), the basis within a quarter of the free memory
    static int pick_m(int S, int ne, int cap)
    {
        const int mmax = cap > 0 ? cap : 200;
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return 0;
        const size_t per = sizeof(zf) * (size_t)S * ne;
        const size_t fit = fr / 4 / (per ? per : 1);
        return (int)std::min<size_t>(mmax, fit > 1 ? fit - 1 : 0);
    }
    // allocate for S systems of ne elements with the basis length pick_m
    // allows (an error when it is below 8 steps, or below the cap when smaller)
    int setup(int S_, int ne_, int cap, const char* who)
    {
        V.release();   // the old basis does not count against the new one's memory
        const int m_ = pick_m(S_, ne_, cap);
        if (m_ < (cap > 0 ? std::min(cap, 8) : 8)) {
            set_err(std::string(who) + ": no device memory for the GMRES basis");
            return MSTMG_ERR_CUDA;
        }
        return init(S_, ne_, m_);
    }
    int init(int S_, int ne_, int m_)
    {
        if (S_ == S && ne_ == ne && m_ == m && hh && V.p) return MSTMG_OK;
        drop_graphs();   // they hold this work's buffers
        V.release();
        S = S_;
        ne = ne_;
        m = m_;
        const int spad = ((S + 3) / 4) * 4;
        CK(V.alloc((size_t)(m + 1) * S * ne));
        CK(W.alloc((size_t)S * ne));
        CK(XP.alloc((size_t)spad * ne));
        CK(Y.alloc((size_t)spad * ne));
        CK(R.alloc((size_t)S * ne));
        CK(h.alloc(off1() + 2 * hpass()));
        CK(rr.alloc(2 * (size_t)S));
        CK(act.alloc(S));
        if (hh) cudaFreeHost(hh);
        hh = nullptr;
        CK(cudaMallocHost((void**)&hh, sizeof(double) * (off1() + hpass())));
        dRm.release();
        CK(dj.alloc(1));
        CK(djmax.alloc(1));
        CK(dkmax.alloc(1));
        CK(dalive.alloc(S));
        CK(dkk.alloc(S));
        CK(dstatus.alloc(S));
        CK(dtarget.alloc(S));
        CK(dcs.alloc((size_t)S * m));
        CK(dsn.alloc((size_t)S * m));
        CK(dg.alloc((size_t)S * (m + 1)));
        CK(dRm.alloc((size_t)S * m * (m + 1)));
        if (hkk) cudaFreeHost(hkk);
        hkk = nullptr;
        CK(cudaMallocHost((void**)&hkk, sizeof(int) * (2 * (size_t)S + 1)));
        Rm.assign((size_t)S * m * (m + 1), 0.0);
        g.assign((size_t)S * (m + 1), 0.0);
        sn.assign((size_t)S * m, 0.0);
        cs.assign((size_t)S * m, 0.0);
        target.assign(S, 0.0);
        ybuf.assign(hpass(), 0.0);
        kk.assign(S, 0);
        frozen.assign(S, 0);
        return MSTMG_OK;
    }
};

struct mstmg_ctx {
    int dev = 0, nsm = 148;
    cudaStream_t st = nullptr;
    mstmg_opts opts;
    // bumped whenever the pair lists, tiles or operator buffers may move:
    // CUDA graphs captured before hold the old pointers
    unsigned long long layout_gen = 0;
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
    // grouped tiles (the FFT path's near pairs): spheres of each tile by slot
    // and the slots of each pair; empty for block tiles
    DevBuf<int> tsph;
    DevBuf<short2> pslot;
    bool tiled = false;   // monodisperse cluster: pairs stored in tile order for the fast kernel
    DevBuf<double> op64;
    DevBuf<float> op32;
    bool ops64_ready = false, ops32_ready = false;
    // mixed fixed-orientation solve: the two polarisations as a many-system
    // residual-replacement solve, its work kept across solves
    MultiWork<double> fo64;
    MultiWork<float> fo32;
    DevBuf<double> fo_rr;
    DevBuf<int> fo_idx;
    bool fo_ready = false;
    GmresWork fo_gm;   // mixed_solver 2
    bool fo_gm_ready = false;
    GmresWork tm_gm;   // mixed_solver 2, T-matrix columns: kept across calls (sized for the largest order)
    // ensembles (mstmg_ensemble_create): configuration c holds spheres
    // cfg_start[c] .. cfg_start[c+1]-1; no pairs between configurations
    std::vector<int> cfg_start, cfg_of;
    std::vector<double> cfg_xg;   // volume-equivalent radius of each configuration
    DevBuf<int> d_cfg_start, ens_off, ens_len;
    DevBuf<double> d_cfg_xg, cfg_qtot;
    GmresWork ens_gm;
    int ens_ldv = 0;
    int chunk32 = 0;   // FP32 columns per tiled chunk chosen by timing (0: not yet)
    DevBuf<double> vcc, fnr, rfnr, bcofd;
    DevBuf<zd> opgen_xi;   // Hankel functions of every pair while the operators are generated
    int vn = 0;
    DevBuf<int> err;
    DevBuf<zd> X64, Y64, pmnp, amnp, pw0, drot, vec64, bvec64;
    DevBuf<zf> X32, Y32, vec32, rvec32;
    DevBuf<double> part, qeff, qtot, small;
    DevBuf<BicgScalars> sc;
    BicgScalars* h_sc = nullptr;
    double* h_small = nullptr;
    int iters[2] = {0, 0}, outer = 0, passes64 = 0, passes32 = 0;
    int host_syncs = 0;   // host synchronisations of the last mixed GMRES solve
    std::vector<int> tord;   // translation order of each sphere to the cluster origin (mstmg_t_matrix_order)
    std::unique_ptr<FftState> fft;   // set by mstmg_fft_setup
    // pairs below translation_switch_order: dense gentranmatrix records (densepair.cu)
    int ndense = 0;
    long long dense_units = 0;
    DevBuf<int2> dpairs;
    DevBuf<long long> doff;
    DevBuf<zd> dop64;
    DevBuf<zf> dop32;
    DevBuf<double> gt_tc, gt_bcd, gt_fnr;
    int gt_nmax = 0;
    // dense operators of every ordered pair for the tensor-core pass of many
    // FP32 columns (tcpass.cu): images, ordered pairs by target, column images
    int tc_state = 0;   // 0 not built, 1 built, -1 not available for this context
    DevBuf<float> tc_h, tc_a;
    DevBuf<int> tc_rstart, tc_rsrc;
    DevBuf<int2> tc_ent;
    int tc_nent = 0;
    int tc_passes = 0;
    cudaStream_t own_st = nullptr;
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    struct Pending { cudaEvent_t a, b; int prec; };
    std::vector<Pending> pending;
    double kt_ms[3] = {0.0, 0.0, 0.0};   // FP64, FP32 rotation passes; FP32 tensor-core passes
    int kt_n[3] = {0, 0, 0};
    SlotMaps sm() const { return SlotMaps{neqns / 2, slot.p, d_order.p, d_offset.p, d_mie_offset.p}; }
};

template <typename T> static int fft_far(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int ncols, unsigned contran);
static int fft_build(mstmg_ctx* c);

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
    o->tile_ctas_per_sm = 0;
    o->fp32_chunk = 0;
    o->mixed_solver = 2;
    o->gmres_restart = 0;
    o->tensor_core = 0;
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

// entry points that treat the context as one cluster refuse an ensemble
static int reject_ensemble(const mstmg_ctx* c, const char* fn)
{
    if (c && !c->cfg_start.empty()) {
        set_err(std::string(fn) + ": not available on an ensemble context (mstmg_ensemble_fixed_orientation solves ensembles)");
        return MSTMG_ERR_UNSUPPORTED;
    }
    return MSTMG_OK;
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

// Install a pair list (i < j) and, for the tiled kernel, its tiles: operator
// record offsets, the device copies, and invalidated operators.
static int upload_pairs(mstmg_ctx* c, const std::vector<int2>& pr, int np, const std::vector<int4>& tl)
{
    std::vector<long long> off(np > 0 ? np : 1);
    long long u = 0;
    int maxrec = 4;
    for (int t = 0; t < np; t++) {
        off[t] = u;
        int rec = op_record_units(c->order[pr[t].x], c->order[pr[t].y]);
        maxrec = std::max(maxrec, rec);
        u += rec;
    }
    c->npairs = np;
    c->ntiles = (int)tl.size();
    if (c->ntiles > 0) {
        CK(c->tiles.alloc(tl.size()));
        CK(cudaMemcpyAsync(c->tiles.p, tl.data(), sizeof(int4) * tl.size(), cudaMemcpyHostToDevice, c->st));
    }
    c->op_units = u;
    c->maxrec = maxrec;
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
static int ensure_gentran(mstmg_ctx* c, int lm)
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
    if (2 * lm > GT_WMAX) {
        set_err("sphere orders above 20 are not supported");
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
    // pairs whose smaller order is below translation_switch_order take the
    // reference's dense path (coefficient_translation, rot_op false)
    const int tso = c->opts.translation_switch_order;
    auto dense_pair = [&](int i, int j) { return std::min(c->order[i], c->order[j]) < tso; };
    // an ensemble has no pairs between its configurations
    auto same_cfg = [&](int i, int j) { return c->cfg_of.empty() || c->cfg_of[i] == c->cfg_of[j]; };
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
    if (!c->cfg_of.empty()) {
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
    c->tiled = !c->opts.generic_kernel && (lm == lmin) && lmin >= tso && tiled_supported(lm, 1) && n > 1 && n < 65536;
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
                    if (i < j && same_cfg(i, j)) add_pair(i, j);
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
    c->tsph.release();   // block tiles
    c->pslot.release();
    (void)off;
    (void)maxrec;
    int rc_ = upload_pairs(c, pr, (int)np, tl);
    if (rc_) return rc_;
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
    // vol_radius as main_calling_program forms it: (sum r^3)**.333333 (single-precision literal)
    double v = 0.0;
    for (int i = 0; i < n; i++) v = v + c->radius[i] * c->radius[i] * c->radius[i];
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
                 opts->tensor_core > 1)) {
        set_err("mstmg_ctx_create: gmres_restart must be >= 0, mixed_solver 0, 1 or 2 and tensor_core -1, 0 or 1");
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
    if (nconfig > 0) {
        c->cfg_start.assign(config_start, config_start + nconfig + 1);
        c->cfg_of.assign(nsphere, 0);
        for (int k = 0; k < nconfig; k++)
            for (int i = config_start[k]; i < config_start[k + 1]; i++) c->cfg_of[i] = k;
    }
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
    if (!is_dev(pos))
        for (int k = 0; k < 3 * c->n; k++)
            if (!std::isfinite(pos[k])) {
                set_err("mstmg_ctx_set_positions: non-finite position of sphere " + std::to_string(k / 3 + 1));
                return MSTMG_ERR_ARG;
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
static DenseArgs dense_args(mstmg_ctx* c)
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
    d.g.tc = c->gt_tc.p;
    d.g.nmax = c->gt_nmax;
    d.g.nd = c->gt_nmax * (c->gt_nmax + 2);
    d.g.fnr = c->gt_fnr.p;
    d.g.bcd = c->gt_bcd.p;
    return d;
}

static int ensure_ops_both(mstmg_ctx* c, bool want64, bool want32, bool force)
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
        if (need32) CK(c->op32.alloc(c->op_units));
        if (was[0] != c->op64.p || was[1] != c->op32.p) c->layout_gen++;
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
    a.vcc = c->vcc.p;
    a.vnmax = c->vn;
    a.fnr = c->fnr.p;
    a.rfnr = c->rfnr.p;
    a.bcofd = c->bcofd.p;
    a.rimed_re = c->opts.medium_re;
    a.rimed_im = c->opts.medium_im;
    a.err = c->err.p;
    CK(c->opgen_xi.alloc(opgen_xi_scratch(c->npairs)));
    a.xi = c->opgen_xi.p;
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


// y[:, 0:nrhs*nchunk] = H x[:, 0:nrhs*nchunk]  (y zeroed here).  nchunk > 1
// only on the tiled path: contran then applies to column r of every chunk.
template <typename T> static int translate(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int nrhs, unsigned contran, int nchunk = 1)
{
    NvtxRange nvtx_(sizeof(T) == 8 ? "translation pass FP64" : "translation pass FP32");
    CK(cudaMemsetAsync(y, 0, sizeof(cpx<T>) * (size_t)c->neqns * nrhs * nchunk, c->st));
    if (c->ndense > 0) {
        if (nchunk > 1) return MSTMG_ERR_UNSUPPORTED;
        const T* drec = sizeof(T) == 8 ? (const T*)c->dop64.p : (const T*)c->dop32.p;
        launch_dense_apply<T>(dense_args(c), drec, x, y, c->neqns, nrhs, contran, c->st);
        CK(cudaGetLastError());
    }
    if (c->npairs == 0) return (c->fft && c->fft->on) ? fft_far<T>(c, x, y, nrhs * nchunk, contran) : MSTMG_OK;
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
        ta.nchunk = nchunk;
        ta.nsph = c->n;
        ta.contran = contran;
        ta.err = c->err.p;
        ta.ctas_per_sm = c->opts.tile_ctas_per_sm;
        ta.tsph = c->tsph.p;
        ta.pslot = c->pslot.p;
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
    if (!use_tiled || launch_translate_tiled<T>(ta, c->lmax, c->nsm, c->st) != 0) {
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
    if (c->fft && c->fft->on) return fft_far<T>(c, x, y, nrhs * nchunk, contran);
    return MSTMG_OK;
}

// Columns per chunk of FP32 tiled passes: opts.fp32_chunk when set (2 or 4),
// otherwise chosen once per context by timing one pass over the caller's
// columns in chunks of 4 and of 2 (each run twice, the second timed), which
// depends on the order and the cluster size (4 wins at L = 9, 2 at L = 8 and
// for small column counts).  The timing passes write y, which the caller's
// own pass then overwrites.
static int fp32_chunk(mstmg_ctx* c, const zf* x, zf* y, int ncols, unsigned pattern2)
{
    if (c->opts.fp32_chunk == 2 || c->opts.fp32_chunk == 4) return c->opts.fp32_chunk;
    if (c->chunk32 > 0) return c->chunk32;
    if (!c->tiled || ncols < 4 || ncols % 4 != 0 || !tiled_supported(c->lmax, 2) || !tiled_supported(c->lmax, 4)) return 4;
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
static bool tc_eligible(const mstmg_ctx* c)
{
    if (c->opts.tensor_core < 0 || c->tc_state < 0) return false;
    if (!c->tiled || c->ndense > 0 || (c->fft && c->fft->on) || c->npairs == 0) return false;
    return c->lmax >= 5 && tc_geom(c->lmax).NP <= 128;
}

// Build the dense operator images of every ordered pair (both directions of
// each pair of the context's list), unless they would take more than a third
// of the free device memory (the context then keeps the rotation kernels).
static int ensure_tc(mstmg_ctx* c)
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
static int tc_translate(mstmg_ctx* c, const zf* x, zf* y, int ncols)
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
template <typename T> static int translate_many(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int ncols, unsigned pattern2)
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
    if (c->tiled && ncols > NR && ncols % NR == 0 && tiled_supported(c->lmax, NR)) {
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

static int interaction_impl(mstmg_ctx* c, int nrhs, const double* ain, double* aout, const int* con_tran, const int* mie_mult,
                            int initial_run, const int* rhs_list, int skip_external)
{
    if (!c || nrhs < 1 || nrhs > 4 || !ain || !aout) {
        set_err("mstmg_interaction: bad arguments (nrhs must be 1..4)");
        return MSTMG_ERR_ARG;
    }
    int rc = skip_external ? MSTMG_OK : ensure_ops(c, 0, initial_run != 0);
    if (rc) return rc;
    const int ne = c->neqns;
    SlotMaps sm = c->sm();
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
            if (mm) launch_mie<double>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, c->an.p, -1, 1, col, col, c->st);
            else launch_conj_copy<double>(ne, col, col, c->st);
        }
    }
    if (skip_external) {
        // no pair translation (and, on this path, no host spheres or plane
        // boundaries): the interaction is zero
        CK(cudaMemsetAsync(c->Y64.p, 0, sizeof(zd) * (size_t)ne * nrhs, c->st));
    } else {
        rc = translate<double>(c, c->X64.p, c->Y64.p, nrhs, mask);
        if (rc) return rc;
    }
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

// cbicg with niter < 0: the order-of-scattering iteration (mstm-solver-8.f90:787-822),
// x += M H p, p = M H p, until ||M H p||^2 / ||b||^2 < eps or -niter steps.
// *err keeps the reference's value: the error at the exit, 0 when the count ran out.
static int oos_solve(mstmg_ctx* c, const zd* b, zd* x, int niter, double eps, int* iter, double* err)
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
        launch_mie<double>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, c->an.p, 1, 0, c->Y64.p, cr, c->st);
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

static int solve_multi_rr(mstmg_ctx* c, MultiWork<double>& w64, MultiWork<float>& w32, DevBuf<double>& rr, DevBuf<int>& idx, int S,
                          const zd* B, zd* X, double eps, int niter, std::vector<int>& iters, std::vector<double>& errs,
                          std::vector<int>& status, int* outer_count);
// systems of an ensemble: segment offsets and lengths per system (device),
// vectors of ldv elements in the GMRES work
struct EnsSeg {
    const int* off;
    const int* len;
    int ldv;
};
static int solve_multi_gmres(mstmg_ctx* c, MultiWork<double>& w64, GmresWork& gw, int S, const zd* B, zd* X, double eps, int niter,
                             std::vector<int>& iters, std::vector<double>& errs, std::vector<int>& status, int* outer_count,
                             const EnsSeg* seg = nullptr, bool x_zero = false);


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
    launch_planewave(alpha, sinc, dir, c->lmax, ne, c->slot_full.p, c->d_order.p, c->d_offset.p, c->pos.p, c->pw0.p, c->drot.p, c->pmnp.p,
                     c->st);
    zd* bvec = c->bvec64.p;
    for (int p = 0; p < 2; p++)
        launch_mie<double>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, c->an.p, 1, 0, c->pmnp.p + (size_t)p * ne,
                           bvec + (size_t)p * ne, c->st);
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
// ---------------------------------------------------------------------------
// Cluster-origin post-processing and the T matrix
// ---------------------------------------------------------------------------

static mstmg::Tables& big_tables()
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
    r0[0] = r0[1] = r0[2] = 0.0;
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) r0[k] = r0[k] + c->hpos[3 * (size_t)i + k];
    for (int k = 0; k < 3; k++) r0[k] = r0[k] / (double)n;
    DevBuf<zd> tscr;
    const int sstride = 3 * (200 + MSTMG_LMAX + 4);
    CK(dtord.alloc(n));
    CK(tscr.alloc((size_t)n * sstride));
    launch_tranorder(n, c->pos.p, c->d_order.p, r0, c->opts.medium_re, trans_eps, max_t_order, bt.bc.p, bt.fnr.p, bt.nbc, tscr.p, sstride,
                     dtord.p, c->st);
    tord.resize(n);
    CK(cudaMemcpyAsync(tord.data(), dtord.p, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int t = std::min(c->lmax, max_t_order);
    for (int i = 0; i < n; i++) t = std::max(t, tord[i]);
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

// ---- many systems at once ----


// cbicg for the systems listed in sys (columns of B and of the work vectors),
// all advanced together; system s stops where cbicg would stop it.  X (w.v().X)
// holds the initial guesses when have_x0.  iters/errs/status are indexed by
// system; status 2 = breakdown.
template <typename T>
static int bicg_multi(mstmg_ctx* c, MultiWork<T>& w, const cpx<T>* B, const std::vector<int>& sys, bool have_x0, int niter,
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
    launch_m_init<T>(sm, an, ne, a, w.act.p, B, v, w.YP.p, have_x0 ? 1 : 0, w.part.p, w.sc.p, c->nsm, c->st);
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
        launch_m_pack<T>(sm, an, ne, a, apad, w.act.p, v.P, v.W, w.XP.p, c->nsm, c->st);
        if ((rc = translate_many<T>(c, w.XP.p, w.YP.p, 2 * apad, 2u))) return rc;
        launch_m_post<T>(sm, an, ne, a, w.act.p, v, w.YP.p, w.part.p, w.sc.p, c->nsm, c->st, w.cnt.p);
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
static int solve_multi_mixed(mstmg_ctx* c, MultiWork<double>& w64, MultiWork<float>& w32, DevBuf<zf>& B32, DevBuf<double>& rr,
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
static int solve_multi_rr(mstmg_ctx* c, MultiWork<double>& w64, MultiWork<float>& w32, DevBuf<double>& rr, DevBuf<int>& idx, int S,
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
static int solve_multi_gmres(mstmg_ctx* c, MultiWork<double>& w64, GmresWork& gw, int S, const zd* B, zd* X, double eps, int niter,
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
            launch_m_resid<float>(sm, c->an.p, ne, a, w64.act.p, B, X, w64.YP.p, gw.R.p, w64.part.p, gw.rr.p, c->nsm, c->st, 1);
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
                            launch_gm_apply(sm, an32, ne, na, gw.XP.p, gw.Y.p, gw.W.p, c->nsm, c->st);
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
                    launch_gm_apply(sm, an32, ne, na, gw.XP.p, gw.Y.p, gw.W.p, c->nsm, c->st);
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
    double r0[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) r0[k] = r0[k] + c->hpos[3 * (size_t)i + k];
    for (int k = 0; k < 3; k++) r0[k] = r0[k] / (double)n;
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
    CK(mscr.alloc((size_t)grid * std::max(strm, strd)));
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
            // per-sphere efficiencies of every column, summed
            launch_tm_qeff(n, S, c->d_order.p, c->d_offset.p, c->d_mie_offset.p, c->rad.p, rimed, c->an_inv.p, Xq, PK.p + (size_t)col0 * ne,
                           ne, qcol.p, c->st);
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
template <typename T> static int fft_far(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int ncols, unsigned contran)
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
static int fft_build(mstmg_ctx* c)
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
    c->tsph.release();
    c->pslot.release();
    std::vector<int4> tl;
    {
        const int B = TILE_B;
        const int lmin = *std::min_element(c->order.begin(), c->order.end());
        c->tiled = !c->opts.generic_kernel && lmin == c->lmax && lmin >= c->opts.translation_switch_order && tiled_supported(c->lmax, 1) &&
                   !pr.empty();
        if (c->tiled) {
            std::vector<int> grp(n), gs(n);
            int k = 0;
            for (const auto& cm : members)
                for (int i : cm) {
                    grp[i] = k / B;
                    gs[i] = k % B;
                    k++;
                }
            const long long ng = (n + B - 1) / B;
            std::vector<int> gmem((size_t)ng * B, -1);
            for (int i = 0; i < n; i++) gmem[(size_t)grp[i] * B + gs[i]] = i;
            std::vector<long long> key(pr.size());
            std::vector<int> idx(pr.size());
            for (size_t q = 0; q < pr.size(); q++) {
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
                tl.push_back(make_int4((int)start, (int)(q - start), 0, ga == gb ? 1 : 0));
            }
            pr.swap(pr2);
            CK(c->tsph.alloc(ts.size()));
            CK(c->pslot.alloc(ps.size()));
            CK(cudaMemcpyAsync(c->tsph.p, ts.data(), sizeof(int) * ts.size(), cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(c->pslot.p, ps.data(), sizeof(short2) * ps.size(), cudaMemcpyHostToDevice, c->st));
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
