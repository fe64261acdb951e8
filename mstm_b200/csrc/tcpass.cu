// tcpass.cu -- the pair translation pass of many columns on the tensor cores.
//
// Same operator as the rotation kernels (MSTM's external_to_external_expansion,
// december2023/mstm-modules-33.f90:6390-6525, i.e. y_i += H(r_i - r_j) x_j over
// every ordered pair), with each pair's translation stored as the dense
// mode-diagonal matrix of gentranmatrix (modules:1762-1888, the form
// coefficient_translation uses below translation_switch_order,
// modules:6669-6674) instead of the rotation/axial factors.  With many columns
// (the 2(2l+1) right-hand sides of a T-matrix order, or several orders at
// once) the pass is a dense contraction, done here with tcgen05.mma:
//
//   for target sphere i, mode p, M tile of 128 columns:
//     Y_i^T (128 x NP, complex) = sum_j X_j^T (128 x NP) H_ij^T (NP x NP)
//
// in real arithmetic [Yr | Yi] += Xr [Hr | Hi]^T, Yr -= Xi Hi^T, Yi += Xi Hr^T,
// with every operand split into TF32 hi + lo parts and three products per
// real product (hi hi + hi lo + lo hi): FP32-level accuracy with FP32
// accumulation in tensor memory.
//
// Data layout: both operands are stored in HBM as images of the shared-memory
// tiles the MMA reads (K-major, no swizzle: core matrices of 8 rows x 16 bytes),
// chunk by chunk of 8 sources (one MMA K step), so one bulk copy
// (cp.async.bulk) moves a chunk into a pipeline stage:
//   * operator images (built once per cluster by tc_gen_kernel): per ordered
//     pair (i <- j), mode p, chunk kc: [Hr; Hi] hi plane and lo plane, 2NP rows
//     (targets) x 8 sources;
//   * column images (built every pass by tc_pack_kernel): per M tile, source
//     sphere j, mode p, chunk kc: Xr hi, Xr lo, Xi hi, Xi lo, 128 rows (columns)
//     x 8 sources.
//
// The pass is a persistent kernel, one CTA per SM: the work is the list of
// (target, mode, source) units, cut into equal ranges, one range per CTA.  A
// CTA carries up to two M tiles (256 columns), so every operator chunk is
// read from HBM once per pass.  Inside a CTA, warp 4 streams the chunks into
// a ring of stages (bulk copies + mbarriers), warp 5 issues the MMAs (one
// thread) into the tensor-memory accumulators, and warps 0-3 read a finished
// accumulator out (tcgen05.ld) and add it into y with vector atomics; with
// one M tile there are two accumulators, so the next target accumulates
// while the last one is read out.  Every wait is bounded: a wait that gives up records
// MSTMG_ERR_CUDA and ends the CTA's work.
#include "common.cuh"
#include "tcpass.cuh"

namespace {

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mb_init(uint32_t bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mb_expect(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mb_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mb_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}
#define TC_WAIT_LIMIT (1 << 22)
// bounded wait; gives up after TC_WAIT_LIMIT polls or when another role of
// the CTA has given up
__device__ __forceinline__ bool mb_wait(uint32_t bar, uint32_t parity, volatile int* abort)
{
    for (int it = 0; it < TC_WAIT_LIMIT; ++it) {
        if (mb_try(bar, parity)) return true;
        if ((it & 255) == 255 && *abort) return false;
    }
    return false;
}
// bounded wait that does not give up early when the CTA aborts (used to
// drain the MMAs before the tensor memory is released)
__device__ __forceinline__ bool mb_wait_all(uint32_t bar, uint32_t parity)
{
    for (int it = 0; it < TC_WAIT_LIMIT; ++it)
        if (mb_try(bar, parity)) return true;
    return false;
}
// bulk copy global -> shared with an L2 eviction-priority hint for the lines it reads
__device__ __forceinline__ void bulk_g2s_hint(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar, uint64_t policy)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar), "l"(policy)
                 : "memory");
}
__device__ __forceinline__ uint64_t l2_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// shared-memory matrix descriptor: K-major, no swizzle (core matrices of 8
// rows x 16 bytes), lbo = byte distance of the two core matrices along K of
// one MMA step, sbo = byte distance between groups of 8 rows
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           (1ull << 46);
}
// instruction descriptor of kind::tf32: D FP32, A and B TF32, both K-major,
// M = 128, N = n; neg: negate A
__host__ __device__ constexpr uint32_t idesc_tf32(int n, int neg)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)neg << 13) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}
__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ float tf32_rna(float v)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return __uint_as_float(r);
}
// float offset of element (row r, source k) inside a K-major plane of 8
// sources: core matrices of 8 rows x 4 sources (128 bytes), the two of a row
// group adjacent (LBO 128 bytes), row groups 256 bytes apart (SBO)
__host__ __device__ __forceinline__ int img_off(int r, int k) { return (r >> 3) * 64 + (k >> 2) * 32 + (r & 7) * 4 + (k & 3); }
#define TC_LBO 128u
#define TC_SBO 256u

// unit u of the flat list (target i, mode p, entry e): i-major, then p, then e
struct UnitIt {
    int i, p, e;
};
__device__ __forceinline__ UnitIt unit_at(const int* rstart, int nsph, long long u)
{
    int lo = 0, hi = nsph - 1;
    while (lo < hi) {   // largest i with 2 rstart[i] <= u
        const int mid = (lo + hi + 1) >> 1;
        if (2LL * rstart[mid] <= u) lo = mid;
        else hi = mid - 1;
    }
    UnitIt it;
    it.i = lo;
    const int ns = rstart[lo + 1] - rstart[lo];
    const long long rem = u - 2LL * rstart[lo];
    it.p = (int)(rem / ns);
    it.e = rstart[lo] + (int)(rem - (long long)it.p * ns);
    return it;
}
__device__ __forceinline__ void unit_next(const int* rstart, UnitIt& it)
{
    if (++it.e < rstart[it.i + 1]) return;
    if (it.p == 0) {
        it.p = 1;
        it.e = rstart[it.i];
        return;
    }
    do { it.i++; } while (rstart[it.i + 1] == rstart[it.i]);
    it.p = 0;
    it.e = rstart[it.i];
}

}  // namespace

// ---------------------------------------------------------------------------
// operator images: one CTA per ordered pair (i <- j), H(r_i - r_j) of
// gentranmatrix (outgoing, source order L, target order L, both modes)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) tc_gen_kernel(TcGenArgs a)
{
    __shared__ GtShared gs;
    const int q = blockIdx.x;
    if (q >= a.nent) return;
    const int i = a.ent[q].x, j = a.ent[q].y;
    const TcGeom G = a.geo;
    double xp[3] = {a.pos[3 * i] - a.pos[3 * j], a.pos[3 * i + 1] - a.pos[3 * j + 1], a.pos[3 * i + 2] - a.pos[3 * j + 2]};
    gt_prepare(gs, a.g, xp, 3, mk(a.rimed_re, a.rimed_im), 2 * G.L);
    float* base = a.himg + (size_t)q * tc_himg_floats(G);
    const int plane = 2 * G.NP * TC_KC;
    for (int el = threadIdx.x; el < G.nb * G.nb; el += blockDim.x) {
        const int t = el / G.nb, s = el - t * G.nb;   // target row, source column
        int m, n, k, l;
        gt_mn(s, G.L, m, n);
        gt_mn(t, G.L, k, l);
        zd e[2];
        gt_element(gs, a.g, 3, 2 * G.L, n, m, l, k, e[0], e[1]);
        const int kc = s / TC_KC, kk = s % TC_KC;
#pragma unroll
        for (int p = 0; p < 2; p++) {
            float* img = base + ((size_t)p * G.NKC + kc) * 2 * plane;
            const double v[2] = {e[p].x, e[p].y};
#pragma unroll
            for (int c = 0; c < 2; c++) {   // Hr rows 0..NP-1, Hi rows NP..2NP-1
                const float hi = tf32_rna((float)v[c]);
                const float lo = tf32_rna((float)(v[c] - (double)hi));
                const int o = img_off(t + c * G.NP, kk);
                img[o] = hi;
                img[plane + o] = lo;
            }
        }
    }
}

void launch_tc_gen(const TcGenArgs& a, cudaStream_t st)
{
    if (a.nent == 0) return;
    tc_gen_kernel<<<a.nent, 128, 0, st>>>(a);
    launch_counter() += 1;
}

// ---------------------------------------------------------------------------
// column images: one CTA per (M tile, sphere, mode, chunk), a thread per
// (row, group of 4 sources)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) tc_pack_kernel(TcPassArgs a)
{
    const TcGeom G = a.geo;
    int b = blockIdx.x;
    const int kc = b % G.NKC;
    b /= G.NKC;
    const int p = b & 1;
    b >>= 1;
    const int j = b % a.nsph, mt = b / a.nsph;
    const int r = threadIdx.x >> 1, k4 = threadIdx.x & 1;
    const int c = mt * TC_M + r;
    float4 v[4];
    float* pv = reinterpret_cast<float*>(v);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int s = kc * TC_KC + k4 * 4 + q;
        zf x = mk(0.f, 0.f);
        if (c < a.ncols && s < G.nb) x = a.x[(size_t)c * a.ld + (size_t)j * 2 * G.nb + (size_t)p * G.nb + s];
        const float rh = tf32_rna(x.x), ih = tf32_rna(x.y);
        pv[0 * 4 + q] = rh;
        pv[1 * 4 + q] = tf32_rna(x.x - rh);
        pv[2 * 4 + q] = ih;
        pv[3 * 4 + q] = tf32_rna(x.y - ih);
    }
    float* base = a.aimg + ((((size_t)mt * a.nsph + j) * 2 + p) * G.NKC + kc) * (4 * TC_M * TC_KC);
    const int o = img_off(r, k4 * 4);
#pragma unroll
    for (int pl = 0; pl < 4; pl++) *reinterpret_cast<float4*>(base + pl * (TC_M * TC_KC) + o) = v[pl];
}

// ---------------------------------------------------------------------------
// the pass
// ---------------------------------------------------------------------------
#define TC_SA (4 * TC_M * TC_KC * 4)   // bytes of one M tile's column images in a stage
#define TC_MAXST 8

template <int MTN>
__global__ void __launch_bounds__(192, 1) tc_pass_kernel(TcPassArgs a, int nstage, long long nunit, int ngroup)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    const TcGeom G = a.geo;
    const int NP = G.NP, NKC = G.NKC;
    const uint32_t SB = 2u * 2u * NP * TC_KC * 4u;   // bytes of a stage's operator images (hi, lo)
    const uint32_t SA = MTN * TC_SA;
    const uint32_t STG = SA + SB;
    // tensor memory: per segment MTN accumulators of 2NP columns ([Yr | Yi]);
    // two segments' worth (double buffering) when they fit in 256 columns
    const int RS = MTN * 2 * NP;
    const int nbuf = RS <= 256 ? 2 : 1;
    const uint32_t sbase = su32(sm);
    auto bar_full = [&](int s) { return sbase + 8u * s; };
    auto bar_empty = [&](int s) { return sbase + 8u * (TC_MAXST + s); };
    auto bar_tfull = [&](int b) { return sbase + 8u * (2 * TC_MAXST + b); };
    auto bar_tempty = [&](int b) { return sbase + 8u * (2 * TC_MAXST + 2 + b); };
    const uint32_t bar_drain = sbase + 8u * (2 * TC_MAXST + 4);
    uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(sm + 256);
    volatile int* abort = reinterpret_cast<volatile int*>(sm + 260);
    const uint32_t stage0 = sbase + 1024u;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < nstage; s++) {
            mb_init(bar_full(s), 1);
            mb_init(bar_empty(s), 1);
        }
        for (int b = 0; b < 2; b++) {
            mb_init(bar_tfull(b), 1);
            mb_init(bar_tempty(b), 4);
        }
        mb_init(bar_drain, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_holder)), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tmem_holder;

    const int ntp = (a.nmt + MTN - 1) / MTN;
    const int tp = blockIdx.x % ntp, grp = blockIdx.x / ntp;
    const int mt0 = tp * MTN;
    const long long u0 = nunit * grp / ngroup, u1 = nunit * (grp + 1) / ngroup;

    if (u0 < u1) {
        if (warp == 4) {
            // ---- producer: column and operator chunks into the stages ----
            if (lane == 0) {
                // the column images are read by every CTA and should stay in
                // L2; the operator images stream through once
                const uint64_t keep = l2_evict_last(), stream = l2_evict_first();
                UnitIt it = unit_at(a.rstart, a.nsph, u0);
                long long q = 0;
                for (long long u = u0; u < u1; u++) {
                    const int j = a.rsrc[it.e];
                    for (int kc = 0; kc < NKC; kc++, q++) {
                        const int s = (int)(q % nstage);
                        const uint32_t ph = (uint32_t)((q / nstage) & 1);
                        if (!mb_wait(bar_empty(s), ph ^ 1u, abort)) {
                            atomicExch(a.err, MSTMG_ERR_CUDA);
                            *abort = 1;
                            u = u1;
                            break;
                        }
                        const uint32_t dst = stage0 + (uint32_t)s * STG;
                        mb_expect(bar_full(s), STG);
#pragma unroll
                        for (int t = 0; t < MTN; t++)
                            bulk_g2s_hint(dst + t * TC_SA,
                                          a.aimg + ((((size_t)(mt0 + t) * a.nsph + j) * 2 + it.p) * NKC + kc) * (4 * TC_M * TC_KC),
                                          TC_SA, bar_full(s), keep);
                        bulk_g2s_hint(dst + SA, a.himg + (((size_t)it.e * 2 + it.p) * NKC + kc) * (2 * 2 * NP * TC_KC), SB, bar_full(s),
                                      stream);
                    }
                    if (u + 1 < u1) unit_next(a.rstart, it);
                }
            }
        } else if (warp == 5) {
            // ---- MMA issuer ----
            if (lane == 0) {
                const uint32_t id2 = idesc_tf32(2 * NP, 0), id1 = idesc_tf32(NP, 0), id1n = idesc_tf32(NP, 1);
                const uint32_t hoff = (uint32_t)(NP / 8) * TC_SBO;   // the Hi half of an operator plane
                UnitIt it = unit_at(a.rstart, a.nsph, u0);
                long long q = 0;
                int seg = 0;
                bool first = true, ok = true;
                for (long long u = u0; u < u1 && ok; u++) {
                    const int b = seg % nbuf;
                    if (first) {
                        if (!mb_wait(bar_tempty(b), (uint32_t)(((seg / nbuf) & 1) ^ 1), abort)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                    }
                    const uint32_t dbuf = tbase + (uint32_t)b * 256u;
                    for (int kc = 0; kc < NKC; kc++, q++) {
                        const int s = (int)(q % nstage);
                        if (!mb_wait(bar_full(s), (uint32_t)((q / nstage) & 1), abort)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t st = stage0 + (uint32_t)s * STG;
                        const uint32_t bh = st + SA, bl = bh + SB / 2u;
                        const uint32_t acc = (first && kc == 0) ? 0u : 1u;
#pragma unroll
                        for (int t = 0; t < MTN; t++) {
                            const uint32_t d0 = dbuf + (uint32_t)(t * 2 * NP), dy = d0 + (uint32_t)NP;
                            const uint32_t at = st + t * TC_SA;
                            const uint32_t arh = at, arl = at + 1u * TC_M * TC_KC * 4u, aih = at + 2u * TC_M * TC_KC * 4u,
                                           ail = at + 3u * TC_M * TC_KC * 4u;
                            mma_tf32(d0, sdesc(arh, TC_LBO, TC_SBO), sdesc(bh, TC_LBO, TC_SBO), id2, acc);
                            mma_tf32(d0, sdesc(arh, TC_LBO, TC_SBO), sdesc(bl, TC_LBO, TC_SBO), id2, 1u);
                            mma_tf32(d0, sdesc(arl, TC_LBO, TC_SBO), sdesc(bh, TC_LBO, TC_SBO), id2, 1u);
                            mma_tf32(d0, sdesc(aih, TC_LBO, TC_SBO), sdesc(bh + hoff, TC_LBO, TC_SBO), id1n, 1u);
                            mma_tf32(d0, sdesc(aih, TC_LBO, TC_SBO), sdesc(bl + hoff, TC_LBO, TC_SBO), id1n, 1u);
                            mma_tf32(d0, sdesc(ail, TC_LBO, TC_SBO), sdesc(bh + hoff, TC_LBO, TC_SBO), id1n, 1u);
                            mma_tf32(dy, sdesc(aih, TC_LBO, TC_SBO), sdesc(bh, TC_LBO, TC_SBO), id1, 1u);
                            mma_tf32(dy, sdesc(aih, TC_LBO, TC_SBO), sdesc(bl, TC_LBO, TC_SBO), id1, 1u);
                            mma_tf32(dy, sdesc(ail, TC_LBO, TC_SBO), sdesc(bh, TC_LBO, TC_SBO), id1, 1u);
                        }
                        mma_commit(bar_empty(s));   // the stage is free once these MMAs are done
                    }
                    if (!ok) break;
                    UnitIt nx = it;
                    bool last = (u + 1 == u1);
                    if (!last) {
                        unit_next(a.rstart, nx);
                        last = (nx.i != it.i || nx.p != it.p);
                    }
                    if (last) {
                        mma_commit(bar_tfull(b));   // accumulator b complete
                        seg++;
                    }
                    first = last;
                    it = nx;
                }
                if (!ok) {
                    atomicExch(a.err, MSTMG_ERR_CUDA);
                    *abort = 1;
                }
                // every MMA issued by this thread has completed before the
                // tensor memory is released
                mma_commit(bar_drain);
                if (!mb_wait_all(bar_drain, 0u)) atomicExch(a.err, MSTMG_ERR_CUDA);
            }
        } else {
            // ---- epilogue: warps 0-3, accumulator rows 32 w .. 32 w + 31 ----
            const int row = warp * 32 + lane;
            UnitIt it = unit_at(a.rstart, a.nsph, u0);
            int seg = 0;
            for (long long u = u0; u < u1; u++) {
                UnitIt nx = it;
                bool last = (u + 1 == u1);
                if (!last) {
                    unit_next(a.rstart, nx);
                    last = (nx.i != it.i || nx.p != it.p);
                }
                if (last) {
                    const int b = seg % nbuf;
                    if (!mb_wait(bar_tfull(b), (uint32_t)((seg / nbuf) & 1), abort)) {
                        atomicExch(a.err, MSTMG_ERR_CUDA);
                        *abort = 1;
                        break;
                    }
                    tc_fence_after();
#pragma unroll
                    for (int t = 0; t < MTN; t++) {
                        const int c = (mt0 + t) * TC_M + row;
                        const uint32_t tr = tbase + (uint32_t)b * 256u + (uint32_t)(t * 2 * NP) + ((uint32_t)(warp * 32) << 16);
                        zf* yo = a.y + (size_t)c * a.ld + (size_t)it.i * 2 * G.nb + (size_t)it.p * G.nb;
                        for (int t0 = 0; t0 < NP; t0 += 16) {
                            float vr[16], vi[16];
                            tmem_ld16(tr + (uint32_t)t0, vr);
                            tmem_ld16(tr + (uint32_t)(NP + t0), vi);
                            if (c < a.ncols) {
#pragma unroll
                                for (int k = 0; k < 16; k++)
                                    if (t0 + k < G.nb) atomicAdd(reinterpret_cast<float2*>(yo + t0 + k), make_float2(vr[k], vi[k]));
                            }
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mb_arrive(bar_tempty(b));
                    seg++;
                }
                it = nx;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 5) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(512));
}

template <int MTN> static int launch_pass(const TcPassArgs& a, int nsm, cudaStream_t st)
{
    const TcGeom& G = a.geo;
    const size_t stg = (size_t)MTN * TC_SA + (size_t)2 * 2 * G.NP * TC_KC * 4;
    int nstage = (int)((220 * 1024 - 1024) / stg);
    if (nstage > TC_MAXST) nstage = TC_MAXST;
    if (nstage < 2) return -1;
    const size_t smem = 1024 + (size_t)nstage * stg;
    cudaFuncSetAttribute(tc_pass_kernel<MTN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long long nunit = 2LL * a.nent;
    const int ntp = (a.nmt + MTN - 1) / MTN;
    int ngroup = nsm / ntp;
    if (ngroup < 1) ngroup = 1;
    if (ngroup > nunit) ngroup = (int)nunit;
    tc_pass_kernel<MTN><<<(unsigned)(ngroup * ntp), 192, smem, st>>>(a, nstage, nunit, ngroup);
    launch_counter() += 1;
    return 0;
}

int launch_tc_pass(const TcPassArgs& a, int nsm, cudaStream_t st)
{
    const TcGeom& G = a.geo;
    if (G.NP > 128 || G.NP < 16 || a.nmt < 1 || a.nent < 1) return -1;
    const int mtn = tc_tiles_per_cta(G, a.nmt);
    const int ntile = (a.nmt + mtn - 1) / mtn * mtn;   // column images of every tile the CTAs read
    tc_pack_kernel<<<(unsigned)(ntile * a.nsph * 2 * G.NKC), 256, 0, st>>>(a);
    launch_counter() += 1;
    return mtn == 2 ? launch_pass<2>(a, nsm, st) : launch_pass<1>(a, nsm, st);
}
