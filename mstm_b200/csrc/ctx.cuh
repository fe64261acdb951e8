// ctx.cuh -- the context of the C ABI (include/mstm_b200.h) and the host-side
// helpers its implementation files share:
//   capi.cu         context set-up, sphere layout, options, timing, diagnostics
//   capi_pass.cu    pair operators, the translation passes (rotation kernels,
//                   tensor-core pass, FFT path), sphereinteraction
//   capi_solve.cu   cbicg, the fixed-orientation solves and the many-system
//                   solvers (BiCG, residual replacement, restarted GMRES)
//   capi_origin.cu  cluster-origin post-processing (scattering matrix, GSF
//                   expansion) and the T matrix (tmatrix_solution, random
//                   orientation)
#pragma once
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
#include "translate_rows.cuh"
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

// message for mstmg_last_error (this thread)
void set_err(const std::string& s);

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

// Spheres inside other spheres (MSTM's host spheres, spheredata
// findhostspheres, december2023/mstm-modules-33.f90:5230-5276).  A sphere
// that holds others has a second block of equations right after its own,
// the regular field inside it; the kernels see that block as a sphere of
// its own at index n + 1 + v (after the offset sentinel at n), with the
// host's order, so that slot maps and pair lists address it like any other.
struct HostSpheres {
    int nhosted = 0;             // spheres with a host (number_host_spheres)
    int nv = 0;                  // spheres holding others
    std::vector<int> host;       // per sphere: the sphere holding it, -1 none
    std::vector<int> vid;        // per sphere: the index of its internal block, -1 none
    std::vector<double> rext;    // per sphere: re, im of the index around it (exteriorrefindex)
    DevBuf<double> d_rext, qv, xpos;   // xpos: positions of the device sphere arrays (internal blocks at their host's centre)
    DevBuf<int> d_host, d_hoff, d_outside;   // holding sphere; offset of the internal block (-1 none); 1 outside every sphere
    DevBuf<int> d_hstart, d_held;            // the spheres each sphere holds: held[hstart[i] .. hstart[i+1])
    DevBuf<zd> dn, un, vn;       // the holding spheres' D, U, V Mie coefficients (mie_offset)
    DevBuf<zf> dn32, un32, vn32; // the same in FP32 (the mixed solver's passes)
    DevBuf<double> pmed, dmed;   // the index of each same-host pair's medium: rotation pairs, dense pairs
    // external_to_internal_expansion: (internal block, held sphere) pairs
    // translated by regular operators in the host's index; coincident
    // centres copy the common orders instead
    int nhp = 0, hmaxrec = 4, hlmax = 0;
    long long hunits = 0;
    DevBuf<int2> hpairs, zpairs;
    int nzp = 0;
    DevBuf<long long> hopoff;
    DevBuf<double> hop64, hmed;
    DevBuf<float> hop32;
    bool hops_ready = false, hops32_ready = false;
    bool on() const { return nhosted > 0; }
};

struct mstmg_ctx {
    int dev = 0, nsm = 148;
    cudaStream_t st = nullptr;
    mstmg_opts opts;
    // bumped whenever the pair lists, tiles or operator buffers may move:
    // CUDA graphs captured before hold the old pointers
    unsigned long long layout_gen = 0;
    int n = 0, neqns = 0, lmax = 0, npairs = 0, maxrec = 0;
    int pair_lmax = 0;   // largest order among the spheres of the rotation pairs (the order-generic kernel's strides)
    bool pair_uniform = false;   // every rotation pair has both orders pair_lmax
    long long op_units = 0;
    double xg = 1.0;
    std::vector<int> order, offset, mie_offset;
    std::vector<double> radius;
    std::vector<double> hpos;   // host copy of the positions (cluster origin)
    std::vector<double> ri_host;   // host copy of the refractive indices (re, im)
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
    int tile_L = 0;       // the sphere order of the tiled pairs (the cluster's; with host spheres, the held spheres')
    int row32 = 0;        // tiled: floats per FP32 row record (translate_rows.cuh); 0: FP32 records as FP64
    // pair shard (mstmg_set_pair_shard): this context translates the tiles
    // t with t % nshards == shard; all tiles kept on the host
    int shard = 0, nshards = 1;
    std::vector<int4> tiles_host;
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
    HostSpheres hs;                  // spheres inside others (empty when none)
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

inline bool is_dev(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

inline cudaError_t copy_in(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
    return cudaMemcpyAsync(dst, src, bytes, is_dev(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
}
inline cudaError_t copy_out(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
    return cudaMemcpyAsync(dst, src, bytes, is_dev(dst) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st);
}

// ---- shared between the implementation files ----
struct EnsSeg {
    const int* off;
    const int* len;
    int ldv;
};
// capi.cu
void resolve_timing(mstmg_ctx* c);
int reject_ensemble(const mstmg_ctx* c, const char* fn);
int reject_sharded(const mstmg_ctx* c, const char* fn);
int reject_hosts(const mstmg_ctx* c, const char* fn);
int apply_shard(mstmg_ctx* c);
int check_kernel_err(mstmg_ctx* c);
int upload_pairs(mstmg_ctx* c, const std::vector<int2>& pr, int np, const std::vector<int4>& tl);
int ensure_gentran(mstmg_ctx* c, int lm);
int setup_layout(mstmg_ctx* c);
// capi_pass.cu
DenseArgs dense_args(mstmg_ctx* c);
int ensure_ops_both(mstmg_ctx* c, bool want64, bool want32, bool force);
int ensure_ops(mstmg_ctx* c, int prec, bool force);
template <typename T> int translate(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int nrhs, unsigned contran, int nchunk = 1);
int fp32_chunk(mstmg_ctx* c, const zf* x, zf* y, int ncols, unsigned pattern2);
bool tc_eligible(const mstmg_ctx* c);
int ensure_tc(mstmg_ctx* c);
int tc_translate(mstmg_ctx* c, const zf* x, zf* y, int ncols);
template <typename T> int translate_many(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int ncols, unsigned pattern2);
int interaction_impl(mstmg_ctx* c, int nrhs, const double* ain, double* aout, const int* con_tran, const int* mie_mult, int initial_run,
                     const int* rhs_list, int skip_external);
// host spheres: y[:, 0:nrhs] += the regular translations between hosts and
// the spheres they hold (external_to_internal_expansion)
template <typename T> int translate_hosts(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int nrhs, unsigned contran);
// the Mie multiply of every sphere (host spheres' blocks included)
template <typename T> void mie_all(mstmg_ctx* c, int idir, int conj_in, const cpx<T>* x, cpx<T>* y);
template <typename T> int fft_far(mstmg_ctx* c, const cpx<T>* x, cpx<T>* y, int ncols, unsigned contran);
int fft_build(mstmg_ctx* c);
int group_tiles(mstmg_ctx* c, const std::vector<std::vector<int>>& members, std::vector<int2>& pr, std::vector<int4>& tl);
// capi_origin.cu
mstmg::Tables& big_tables();   // the reference's large constant tables (this thread's copy)
// capi_solve.cu
template <typename T>
int bicg_batched(mstmg_ctx* c, int S, const cpx<T>* const* b, BicgVecs<T>* v, bool have_x0, int niter, const double* eps, int* iters,
                 double* errs, int* status);
int oos_solve(mstmg_ctx* c, const zd* b, zd* x, int niter, double eps, int* iter, double* err);
int solve_mixed(mstmg_ctx* c, zd* const* b, zd* const* x, double eps, int niter, int* iters, double* errs, int* status);
template <typename T>
int bicg_multi(mstmg_ctx* c, MultiWork<T>& w, const cpx<T>* B, const std::vector<int>& sys, bool have_x0, int niter,
               const std::vector<double>& eps, std::vector<int>& iters, std::vector<double>& errs, std::vector<int>& status);
int solve_multi_mixed(mstmg_ctx* c, MultiWork<double>& w64, MultiWork<float>& w32, DevBuf<zf>& B32, DevBuf<double>& rr, DevBuf<int>& idx,
                      int S, const zd* B, zd* X, double eps, int niter, std::vector<int>& iters, std::vector<double>& errs,
                      std::vector<int>& status, int* outer_count);
int solve_multi_rr(mstmg_ctx* c, MultiWork<double>& w64, MultiWork<float>& w32, DevBuf<double>& rr, DevBuf<int>& idx, int S, const zd* B,
                   zd* X, double eps, int niter, std::vector<int>& iters, std::vector<double>& errs, std::vector<int>& status,
                   int* outer_count);
int solve_multi_gmres(mstmg_ctx* c, MultiWork<double>& w64, GmresWork& gw, int S, const zd* B, zd* X, double eps, int niter,
                      std::vector<int>& iters, std::vector<double>& errs, std::vector<int>& status, int* outer_count,
                      const EnsSeg* seg = nullptr, bool x_zero = false);

