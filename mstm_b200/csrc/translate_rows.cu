// translate_rows.cu -- the FP32 pair translation pass of monodisperse
// clusters, with operator rows broadcast from shared memory into
// register-resident columns.
//
// Same operator as translate_tiled.cu (MSTM's coefficient_translation,
// december2023/mstm-modules-33.f90:6610-6787, applied in both directions per
// pair as in external_to_external_expansion, modules:6390-6525), on the same
// tiles, with the work of a pair laid out so that every multiply-accumulate
// reads an operator value shared by all columns of the pair:
//   * a step takes PP pairs of a tile whose output spheres are disjoint.  A
//     lane owns one column (direction x rhs x mode) of one pair and one of H
//     interleaved row sets, and holds that column's input of the current
//     degree in registers;
//   * the three products are row sweeps: the lane streams operator rows from
//     shared memory four floats at a time (one address per pair and row set,
//     broadcast to the pair's columns) into packed FP32x2 FMAs:
//        AB  shift/phase/even-odd split of the sources and the forward
//            rotation a'(k) = E_n(k,:) s + O_n(k,:) t            per degree n
//        C   axial translation g = Z_m a' (rows n; the H lanes of a column
//            split each row and add their parts by shuffles)     per degree m
//        D   back rotation, phase and shift, accumulated into the tile's
//            outputs in shared memory                            per degree n
//   * the transposes of the reference's product (the back rotation uses
//     D^T, and the i -> j direction Z^T) are row sweeps too, through the
//     symmetries d^n_{mk} = (-1)^{m+k} d^n_{km} of the Wigner functions, which
//     give E_n(m,k) c_m = (-1)^{m+k} E_n(k,m) c_k (c_0 = 1/2, else 1) and
//     O_n(m,k) = (-1)^{m+k} O_n(k,m) for the folded blocks, and
//     Z_m(l,n) = (-1)^{n+l} Z_m(n,l) for the axial blocks: sign flips of
//     inputs and outputs replace strided reads;
//   * units of work (a degree and a range of its rows) are spread over the 8
//     warps by a schedule made on the host, longest first, so each phase ends
//     at one CTA barrier: three barriers per step of PP pairs;
//   * the operator records and the two source blocks of every pair stream in
//     two steps ahead with cp.async.bulk (two buffers each, mbarrier
//     completion, bounded waits); records use the row layout of
//     translate_rows.cuh, whose rows pair up as the packed FMA's operands and
//     whose header holds the pair's e^{i m phi}.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>
#include "common.cuh"
#include "kernels.cuh"
#include "pairpipe.cuh"
#include "translate_rows.cuh"

using namespace pairpipe;

namespace {

constexpr int RS_MAXU = 64;
// Work units of the three phases: warp w runs unit[ph][first[ph][w] ..
// first[ph][w + 1]), each packed as degree | j0 << 8 | j1 << 16 (row sets
// j0..j1-1 of the degree in AB and D, rows n = j0..j1-1 in C).
struct RowSched {
    int first[3][9];
    unsigned int unit[3][RS_MAXU];
    int fits;   // every phase's units fit unit[][] (checked on the host before a launch)
};

__host__ __device__ constexpr size_t al128(size_t v) { return (v + 127) & ~(size_t)127; }

// the axial products' (s', t') by degree m: entries n = max(1, m)..L of m
// after those of 0..m-1, so the rows of one m are consecutive
template <int L> __host__ __device__ constexpr int goff(int m) { return m == 0 ? 0 : L + (m - 1) * (L + 1) - (m - 1) * m / 2; }
template <int L> __host__ __device__ constexpr int gidx(int m, int n) { return goff<L>(m) + n - (m < 1 ? 1 : m); }

// strides padded for the shared-memory banks: (s', t') columns an odd number
// of 16-byte units apart, tile-output slots an odd number of complex values.
// A column of sources, of a' or of a tile output holds L(L+2) complex values;
// for even L that is a multiple of 16 words and the 8 columns a lane group
// reads at once would share one bank, so their stride gets 2 more (still
// 16-byte aligned for the bulk copies: 4 words apart in the banks)
__host__ __device__ constexpr int rows_cs(int L) { return (L & 1) ? L * (L + 2) : L * (L + 2) + 2; }
__host__ __device__ constexpr int rows_gs(int L) { return (L * (L + 3) / 2) | 1; }
__host__ __device__ constexpr int rows_ss(int L, int NR) { return NR * 2 * rows_cs(L) + 1; }

template <int L, int NR, int PP> __host__ __device__ constexpr size_t rows_smem_pp()
{
    constexpr int C = 4 * NR;
    size_t off = 128;                                                   // mbarriers, step descriptors
    off = al128(off + sizeof(float) * 2 * PP * row_record_units(L));    // records, two steps
    off += sizeof(zf) * 3 * (size_t)PP * C * rows_cs(L);               // sources (two steps), a'
    off += sizeof(float4) * (size_t)PP * C * rows_gs(L);               // (s', t') of the axial products
    off += sizeof(zf) * (size_t)2 * TILE_B * rows_ss(L, NR);           // tile outputs
    return off;
}
// pairs per step: two while two CTAs of that size fit an SM
template <int L, int NR> __host__ __device__ constexpr int rows_pp() { return (NR <= 2 && rows_smem_pp<L, NR, 2>() <= 112 * 1024) ? 2 : 1; }
template <int L, int NR> __host__ __device__ constexpr size_t rows_smem() { return rows_smem_pp<L, NR, rows_pp<L, NR>()>(); }

__device__ __forceinline__ zf cpos(zf a, float s) { return mk(s * a.x, s * a.y); }
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// One row of a rotation block against a register-resident column held as
// pairs X[m] = (s_m.x, t_m.x), Y[m] = (s_m.y, t_m.y): with the row's pairs
// (E(k,m), O(k,m)) every packed FMA takes both operands as they lie.
// Returns P = sum_m E(k,m) s_m and Q = sum_m O(k,m) t_m; with ALT the odd m
// enter with the sign -1.
template <int N, bool ALT>
__device__ __forceinline__ void row_dot(const float* row, const float2 (&X)[N + 1], const float2 (&Y)[N + 1], zf& P, zf& Q)
{
    constexpr int RW = rr_rw(N);
    const float4* r4 = reinterpret_cast<const float4*>(row);
    float2 ax0 = f2(0.f, 0.f), ay0 = ax0, ax1 = ax0, ay1 = ax0;
#pragma unroll
    for (int u = 0; u < RW / 4; u++) {
        const float4 z = r4[u];
        if (2 * u <= N) {
            ax0 = __ffma2_rn(f2(z.x, z.y), X[2 * u], ax0);
            ay0 = __ffma2_rn(f2(z.x, z.y), Y[2 * u], ay0);
        }
        if (2 * u + 1 <= N) {
            ax1 = __ffma2_rn(f2(z.z, z.w), X[2 * u + 1], ax1);
            ay1 = __ffma2_rn(f2(z.z, z.w), Y[2 * u + 1], ay1);
        }
    }
    const float2 sx = ALT ? f2(ax0.x - ax1.x, ax0.y - ax1.y) : f2(ax0.x + ax1.x, ax0.y + ax1.y);
    const float2 sy = ALT ? f2(ay0.x - ay1.x, ay0.y - ay1.y) : f2(ay0.x + ay1.x, ay0.y + ay1.y);
    P = mk(sx.x, sy.x);
    Q = mk(sx.y, sy.y);
}

// Per-lane view of the step: this lane's pair record and columns.
struct Lane {
    const float* rec;   // the pair's record in shared memory
    const zf* src;      // the column's sources (one mode of one sphere block)
    zf* ap;             // the column's a' (rotated sources)
    float4* g;          // the column's (s', t') pairs, packed-S order
    zf* acc;            // the column's output block in the tile accumulators
    int h, p, dir;
    float dsg, sig;     // dir ? -1 : 1 (conjugate phases), swp ? -1 : 1
    bool swp, act;      // shifted column; the lane's pair is part of the step
};

// ---- AB: shift, phase, even/odd split and forward rotation of degree N ----
template <int L, int N, int H> __device__ __forceinline__ void ab_unit(const Lane& ln, int j0, int j1)
{
    const zf* eh = reinterpret_cast<const zf*>(ln.rec);   // e^{i m phi}
    float2 X[N + 1], Y[N + 1];
    {
        const zf U = ln.src[hidx<L>(0, N)];
        X[0] = f2(2.f * U.x, 0.f);
        Y[0] = f2(2.f * U.y, 0.f);
    }
#pragma unroll
    for (int m = 1; m <= N; m++) {
        const int hp = hidx<L>(m, N), hm = hidx<L>(-m, N);
        // with the shift the +m and -m sources trade places; the odd-m sign
        // (-1)^m of the shift and of the fold go into the phase factor
        const zf U = ln.src[ln.swp ? hm : hp], V = ln.src[ln.swp ? hp : hm];
        const zf e = eh[m];
        const float c = (m & 1) ? ln.sig * e.x : e.x;
        const float sn = (m & 1) ? ln.sig * ln.dsg * e.y : ln.dsg * e.y;
        // s = U e + V e*, t = U e - V e* (even m); odd m: s = sig (U e - V e*), t = sig (U e + V e*)
        zf u = U + V, w = U - V;
        if (m & 1) {
            const zf tt = u;
            u = w;
            w = tt;
        }
        X[m] = f2(c * u.x - sn * w.y, c * w.x - sn * u.y);
        Y[m] = f2(c * u.y + sn * w.x, c * w.y + sn * u.x);
    }
    // i -> j: the axial product Z^T a' = S Z S a' (S = diag((-1)^n)); S here
    const float sd = (ln.dir && (N & 1)) ? -1.f : 1.f;
    const float* rows = ln.rec + rr_rot_off(N, L);
    for (int j = j0; j < j1; j++) {
        const int k = H * j + ln.h;
        if (k > N) continue;
        zf P, Q;
        row_dot<N, false>(rows + k * rr_rw(N), X, Y, P, Q);
        if (!ln.act) continue;
        if (k == 0) {
            ln.ap[hidx<L>(0, N)] = cpos(P, sd);
        } else {
            ln.ap[hidx<L>(k, N)] = cpos(P + Q, sd);
            ln.ap[hidx<L>(-k, N)] = cpos(P - Q, (k & 1) ? -sd : sd);
        }
    }
}

// sum over the H lanes of a column (lanes C * PP apart)
template <int H, int STRIDE> __device__ __forceinline__ zf hsum(zf v)
{
#pragma unroll
    for (int o = STRIDE; o < STRIDE * H; o *= 2) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// complex z times v as packed FMAs with z's pair as it lies:
// a += (z.x, z.y) (v.x, v.x), b += (z.x, z.y) (v.y, -v.y); z v = (a.x + b.y, a.y + b.x)
struct CIn {
    float2 a, b;
};
__device__ __forceinline__ CIn cin(zf v) { return CIn{f2(v.x, v.x), f2(v.y, -v.y)}; }

// ---- C: axial translation of degree M, rows (lines) l0..l1-1 ----
template <int L, int M, int H, int STRIDE> __device__ __forceinline__ void c_unit(const Lane& ln, int l0, int l1)
{
    constexpr int m1 = M < 1 ? 1 : M, dim = L - m1 + 1;
    if constexpr (M == 0) {
        // quads (2 complex) per row in the record and per lane; with H = 2 the
        // even row length splits exactly and no lane needs a bounds test
        constexpr int Q0 = rr_zw0(L) / 4, QH = (Q0 + H - 1) / H;
        constexpr bool PRED = QH * H > Q0;
        CIn in[2 * QH];
#pragma unroll
        for (int t = 0; t < 2 * QH; t++) {
            const int v = 2 * QH * ln.h + t;
            in[t] = cin((v < dim) ? ln.ap[hidx<L>(0, 1 + v)] : mk(0.f, 0.f));
        }
        for (int line = l0; line < l1; line++) {
            const float4* rw = reinterpret_cast<const float4*>(ln.rec + rr_z_off(0, L) + (line - 1) * rr_zw0(L)) + QH * ln.h;
            float2 a0 = f2(0.f, 0.f), b0 = a0, a1 = a0, b1 = a0;
#pragma unroll
            for (int t = 0; t < QH; t++) {
                if (!PRED || QH * ln.h + t < Q0) {
                    const float4 z = rw[t];
                    a0 = __ffma2_rn(f2(z.x, z.y), in[2 * t].a, a0);
                    b0 = __ffma2_rn(f2(z.x, z.y), in[2 * t].b, b0);
                    a1 = __ffma2_rn(f2(z.z, z.w), in[2 * t + 1].a, a1);
                    b1 = __ffma2_rn(f2(z.z, z.w), in[2 * t + 1].b, b1);
                }
            }
            const zf g = hsum<H, STRIDE>(mk(a0.x + b0.y + a1.x + b1.y, a0.y + b0.x + a1.y + b1.x));
            // m = 0: s'(0) = g, t'(0) = 0
            if (ln.act && ln.h == 0) ln.g[gidx<L>(0, line)] = make_float4(g.x, 0.f, g.y, 0.f);
        }
    } else {
        constexpr int ZQ = rr_zq(dim), QH = (ZQ + H - 1) / H;   // quads (Z0, Z1 of one l) per row, per lane
        constexpr bool PRED = QH * H > ZQ;
        CIn in0[QH], in1[QH];
#pragma unroll
        for (int t = 0; t < QH; t++) {
            const int v = QH * ln.h + t;
            zf ap = mk(0.f, 0.f), am = ap;
            if (v < dim) {
                ap = ln.ap[hidx<L>(M, m1 + v)];
                am = ln.ap[hidx<L>(-M, m1 + v)];
            }
            // mode 0: Z0 on +m, Z1 on -m; mode 1: Z1 on +m, Z0 on -m
            in0[t] = cin(ln.p ? am : ap);
            in1[t] = cin(ln.p ? ap : am);
        }
        const float sg = (M & 1) ? -1.f : 1.f;
        for (int line = l0; line < l1; line++) {
            const float4* rw = reinterpret_cast<const float4*>(ln.rec + rr_z_off(M, L) + (line - m1) * 4 * ZQ) + QH * ln.h;
            float2 a0 = f2(0.f, 0.f), b0 = a0, a1 = a0, b1 = a0;
#pragma unroll
            for (int t = 0; t < QH; t++) {
                if (!PRED || QH * ln.h + t < ZQ) {
                    const float4 z = rw[t];
                    a0 = __ffma2_rn(f2(z.x, z.y), in0[t].a, a0);
                    b0 = __ffma2_rn(f2(z.x, z.y), in0[t].b, b0);
                    a1 = __ffma2_rn(f2(z.z, z.w), in1[t].a, a1);
                    b1 = __ffma2_rn(f2(z.z, z.w), in1[t].b, b1);
                }
            }
            const zf o0 = hsum<H, STRIDE>(mk(a0.x + b0.y, a0.y + b0.x));
            const zf o1 = hsum<H, STRIDE>(mk(a1.x + b1.y, a1.y + b1.x));
            const zf gp = ln.p ? o1 : o0, gm = ln.p ? o0 : o1;
            // s'(m) = g(m) + (-1)^m g(-m), t'(m) = g(m) - (-1)^m g(-m), stored as (s'.x, t'.x, s'.y, t'.y)
            float* gs = reinterpret_cast<float*>(ln.g + gidx<L>(M, line));
            if (ln.act && ln.h == 0) {
                const zf sv = gp + cpos(gm, sg);
                gs[0] = sv.x;
                gs[2] = sv.y;
            }
            if (ln.act && ln.h == 1) {
                const zf tv = gp - cpos(gm, sg);
                gs[1] = tv.x;
                gs[3] = tv.y;
            }
        }
    }
}

// ---- D: back rotation of degree N, phase, shift, accumulate ----
template <int L, int N, int H> __device__ __forceinline__ void d_unit(const Lane& ln, int j0, int j1)
{
    // hat s(m) = (-1)^m s'(m) / c_m, hat t(m) = (-1)^m t'(m): the (-1)^m by
    // row_dot's alternating sum, 1 / c_0 = 2 here
    float2 X[N + 1], Y[N + 1];
#pragma unroll
    for (int m = 0; m <= N; m++) {
        const float4 g = ln.g[gidx<L>(m, N)];
        X[m] = m ? f2(g.x, g.y) : f2(2.f * g.x, 0.f);
        Y[m] = m ? f2(g.z, g.w) : f2(2.f * g.z, 0.f);
    }
    // i -> j: the output half of S Z S
    const float sd = (ln.dir && (N & 1)) ? -1.f : 1.f;
    const zf* eh = reinterpret_cast<const zf*>(ln.rec);
    const float* rows = ln.rec + rr_rot_off(N, L);
    for (int j = j0; j < j1; j++) {
        const int k = H * j + ln.h;
        if (k > N) continue;
        zf P, Q;
        row_dot<N, true>(rows + k * rr_rw(N), X, Y, P, Q);
        if (!ln.act) continue;
        if (k == 0) {
            zf* o = ln.acc + hidx<L>(0, N);
            *o = *o + cpos(P, sd);
        } else {
            const float sk = (k & 1) ? -1.f : 1.f;
            const zf e = eh[k];
            // e^{-i im phi} and e^{i im phi}, im = k (j -> i) or -k (i -> j)
            const zf em = ln.dir ? e : cj(e), epl = ln.dir ? cj(e) : e;
            zf outk = cpos((P + Q) * em, sk * sd);
            zf outmk = cpos((P - Q) * epl, sd);
            if (ln.swp) {
                const zf tt = outk;
                outk = cpos(outmk, sk);
                outmk = cpos(tt, sk);
            }
            zf* o = ln.acc + hidx<L>(k, N);
            zf* om = ln.acc + hidx<L>(-k, N);
            *o = *o + outk;
            *om = *om + outmk;
        }
    }
}

template <int L, int H, int N = 1> __device__ __forceinline__ void ab_any(int n, const Lane& ln, int j0, int j1)
{
    if constexpr (N <= L) {
        if (n == N) ab_unit<L, N, H>(ln, j0, j1);
        else ab_any<L, H, N + 1>(n, ln, j0, j1);
    }
}
template <int L, int H, int STRIDE, int M = 0> __device__ __forceinline__ void c_any(int m, const Lane& ln, int l0, int l1)
{
    if constexpr (M <= L) {
        if (m == M) c_unit<L, M, H, STRIDE>(ln, l0, l1);
        else c_any<L, H, STRIDE, M + 1>(m, ln, l0, l1);
    }
}
template <int L, int H, int N = 1> __device__ __forceinline__ void d_any(int n, const Lane& ln, int j0, int j1)
{
    if constexpr (N <= L) {
        if (n == N) d_unit<L, N, H>(ln, j0, j1);
        else d_any<L, H, N + 1>(n, ln, j0, j1);
    }
}

// A step's descriptor, written by the thread that streams the step in.
struct StepMeta {
    int q;      // first pair
    int np;     // pairs (1..PP)
    int item;   // work item (tile, chunk)
    int last;   // last step of the tile
    int slots;  // output slots: pair u's (i, j) slots in bytes 2u, 2u + 1
    int i0, j0, diag;   // the tile's block starts and diagonal flag
};

// CTAs per SM the register budget is set for: three for the small orders,
// whose steps are short enough that a third CTA's warps hide the copies' and
// barriers' latency; two otherwise (the larger orders' register tiles)
template <int L> __host__ __device__ constexpr int rows_minb() { return L <= 5 ? 3 : 2; }

template <int L, int NR, bool SO, int MB>
__global__ void __launch_bounds__(256, MB) translate_rows_kernel(TiledArgs<float> a, RowSched sc)
{
    constexpr int NT = 256;
    constexpr int C = 4 * NR, PP = rows_pp<L, NR>(), H = 32 / (PP * C);
    static_assert(PP * C * H == 32, "a warp holds PP pairs x C columns x H row sets");
    constexpr int NB2 = L * (L + 2), NB = 2 * NB2, GS = rows_gs(L), SS = rows_ss(L, NR), CS = rows_cs(L);
    constexpr int REC = row_record_units(L);
    constexpr int NSLOT = 2 * TILE_B;
    constexpr uint32_t RECB = (uint32_t)(REC * sizeof(float));
    constexpr uint32_t XB = (uint32_t)(NB * sizeof(zf));
    constexpr uint32_t XB2 = (uint32_t)(NB2 * sizeof(zf));
    constexpr int CW = PP * C * CS;

    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm);   // [0],[1] records, [2],[3] sources of steps t, t + 1
    StepMeta* meta = reinterpret_cast<StepMeta*>(sm + 64);   // descriptors of steps t, t + 1
    size_t off = 128;
    float* recs = reinterpret_cast<float*>(sm + off);
    off = al128(off + sizeof(float) * 2 * PP * REC);
    zf* SRC = reinterpret_cast<zf*>(sm + off);   // two buffers
    zf* AP = SRC + 2 * CW;
    float4* GB = reinterpret_cast<float4*>(AP + CW);
    zf* ACC = reinterpret_cast<zf*>(GB + PP * C * GS);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int c = lane % C, qq = (lane / C) % PP;
    Lane ln;
    ln.h = lane / (C * PP);
    ln.p = c & 1;
    const int r = (c >> 1) % NR;
    ln.dir = (c >> 1) / NR;
    ln.swp = (ln.dir != (int)((a.contran >> r) & 1u));
    ln.dsg = ln.dir ? -1.f : 1.f;
    ln.sig = ln.swp ? -1.f : 1.f;
    ln.ap = AP + (size_t)(qq * C + c) * CS;
    ln.g = GB + (size_t)(qq * C + c) * GS;

    for (int e = tid; e < NSLOT * SS; e += NT) ACC[e] = mk(0.f, 0.f);
    if (tid == 0) {
        mb_init(&bar[0], 1);
        mb_init(&bar[1], 1);
        mb_init(&bar[2], 1);
        mb_init(&bar[3], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int G = gridDim.x;
    const int NI = a.ntiles * a.nchunk;   // work items (tile, chunk), chunk fastest
    if ((int)blockIdx.x >= NI) return;
    auto tile_of = [&](int it) { return it / a.nchunk; };
    auto col0 = [&](int it) { return (size_t)(it % a.nchunk) * NR * (size_t)a.ld; };

    // Thread 0 streams the step two ahead.  Its tile entry and first two
    // pairs are loaded when the previous step has been issued, a phase
    // before they are used, so their latency stays off the barriers.
    int pf_t = blockIdx.x, pf_q = 0;
    int4 pf_ti = make_int4(0, 0, 0, 0);
    int2 pf_p0 = make_int2(0, 0), pf_p1 = pf_p0;
    short2 pf_s0 = make_short2(0, 0), pf_s1 = pf_s0;
    bool pf_ok = true;
    auto pf_fetch = [&]() {
        pf_p0 = a.pairs[pf_q];
        if (PP == 2 && pf_q + 1 < pf_ti.x + pf_ti.y) pf_p1 = a.pairs[pf_q + 1];
        if (a.pslot) {
            pf_s0 = a.pslot[pf_q];
            if (PP == 2 && pf_q + 1 < pf_ti.x + pf_ti.y) pf_s1 = a.pslot[pf_q + 1];
        }
    };
    // the prefetch step's descriptor: pairs, output slots, end of tile
    auto pf_meta = [&]() {
        auto slots = [&](int2 pr, short2 ps, int& s_i, int& s_j) {
            if (a.pslot) {
                s_i = ps.x;
                s_j = ps.y;
            } else {
                s_i = pr.x - (pf_ti.z >> 16);
                s_j = pf_ti.w ? (pr.y - (pf_ti.z >> 16)) : (TILE_B + pr.y - (pf_ti.z & 0xffff));
            }
        };
        int si0, sj0, si1 = 0, sj1 = 0, np = 1;
        slots(pf_p0, pf_s0, si0, sj0);
        if (PP == 2 && pf_q + 1 < pf_ti.x + pf_ti.y) {
            slots(pf_p1, pf_s1, si1, sj1);
            if (si0 != si1 && si0 != sj1 && sj0 != si1 && sj0 != sj1) np = 2;
        }
        StepMeta m;
        m.q = pf_q;
        m.np = np;
        m.item = pf_t;
        m.last = (pf_q + np == pf_ti.x + pf_ti.y) ? 1 : 0;
        m.slots = si0 | (sj0 << 8) | (si1 << 16) | (sj1 << 24);
        m.i0 = pf_ti.z >> 16;
        m.j0 = pf_ti.z & 0xffff;
        m.diag = pf_ti.w;
        return m;
    };
    auto pf_start = [&]() {
        pf_ti = a.tiles[tile_of(pf_t)];
        pf_q = pf_ti.x;
        pf_fetch();
    };
    auto pf_adv = [&](int np) {
        pf_q += np;
        if (pf_q >= pf_ti.x + pf_ti.y) {
            pf_t += G;
            if (pf_t >= NI) {
                pf_ok = false;
                return;
            }
            pf_start();
        } else {
            pf_fetch();
        }
    };
    auto load_sources = [&](int bb, const StepMeta& m) {
        const zf* xs = a.x + col0(m.item);
        mb_expect(&bar[2 + bb], (uint32_t)m.np * 2u * NR * XB);
        for (int u = 0; u < m.np; u++) {
            const int2 pr = u ? pf_p1 : pf_p0;
            zf* w = SRC + (size_t)bb * CW + (size_t)u * C * CS;
            for (int rr = 0; rr < NR; rr++) {
                const zf* sj = xs + (size_t)rr * a.ld + tile_sphere_base<SO>(a, pr.y, NB);   // source of j -> i
                const zf* si = xs + (size_t)rr * a.ld + tile_sphere_base<SO>(a, pr.x, NB);   // source of i -> j
                if (CS == NB2) {   // both modes' columns in one copy
                    bulk_copy(w + (size_t)(0 * NR + rr) * NB, sj, XB, &bar[2 + bb]);
                    bulk_copy(w + (size_t)(1 * NR + rr) * NB, si, XB, &bar[2 + bb]);
                } else {           // a copy per mode, columns CS apart
                    for (int pm2 = 0; pm2 < 2; pm2++) {
                        bulk_copy(w + (size_t)((0 * NR + rr) * 2 + pm2) * CS, sj + (size_t)pm2 * NB2, XB2, &bar[2 + bb]);
                        bulk_copy(w + (size_t)((1 * NR + rr) * 2 + pm2) * CS, si + (size_t)pm2 * NB2, XB2, &bar[2 + bb]);
                    }
                }
            }
        }
    };
    // records of the prefetch step; its descriptor goes to the ring slot
    // the step uses (read there after the records' mbarrier completes)
    auto load_ops = [&](int bb, const StepMeta& m) {
        meta[bb] = m;
        mb_expect(&bar[bb], (uint32_t)m.np * RECB);
        bulk_copy(recs + (size_t)bb * PP * REC, a.ops + (size_t)m.q * REC, (uint32_t)m.np * RECB, &bar[bb]);   // consecutive records
    };
    if (tid == 0) {
        pf_start();
        for (int bb = 0; bb < 2 && pf_ok; bb++) {
            const StepMeta m = pf_meta();
            load_sources(bb, m);
            load_ops(bb, m);
            pf_adv(m.np);
        }
    }
    for (int t = 0;; t++) {
        const int b = t & 1;
        if (!mb_wait(&bar[b], (t >> 1) & 1) || !mb_wait(&bar[2 + b], (t >> 1) & 1)) {
            // give up; first let the copies in flight land (bounded waits)
            if (tid == 0) atomicExch(a.err, MSTMG_ERR_CUDA);
            mb_wait(&bar[b], (t >> 1) & 1);
            mb_wait(&bar[2 + b], (t >> 1) & 1);
            mb_wait(&bar[b ^ 1], ((t + 1) >> 1) & 1);
            mb_wait(&bar[2 + (b ^ 1)], ((t + 1) >> 1) & 1);
            return;
        }
        const StepMeta cm = meta[b];
        ln.act = qq < cm.np;
        {
            const int sl = (cm.slots >> (16 * qq + (ln.dir ? 8 : 0))) & 255;
            ln.acc = ACC + (size_t)(ln.act ? sl : 0) * SS + (size_t)(r * 2 + ln.p) * CS;
        }
        ln.rec = recs + ((size_t)b * PP + qq) * REC;
        ln.src = SRC + (size_t)b * CW + (size_t)(qq * C + c) * CS;
        // the prefetch step's descriptor (thread 0; its loads were issued a phase ago)
        StepMeta pm;
        if (tid == 0 && pf_ok) pm = pf_meta();

        for (int u = sc.first[0][warp]; u < sc.first[0][warp + 1]; u++) {
            const unsigned un = sc.unit[0][u];
            ab_any<L, H>((int)(un & 255u), ln, (int)((un >> 8) & 255u), (int)(un >> 16));
        }
        __syncthreads();

        // the sources of the step after next stream into this step's buffer
        if (tid == 0 && pf_ok) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            load_sources(b, pm);
        }

        for (int u = sc.first[1][warp]; u < sc.first[1][warp + 1]; u++) {
            const unsigned un = sc.unit[1][u];
            c_any<L, H, C * PP>((int)(un & 255u), ln, (int)((un >> 8) & 255u), (int)(un >> 16));
        }
        __syncthreads();

        for (int u = sc.first[2][warp]; u < sc.first[2][warp + 1]; u++) {
            const unsigned un = sc.unit[2][u];
            d_any<L, H>((int)(un & 255u), ln, (int)((un >> 8) & 255u), (int)(un >> 16));
        }
        __syncthreads();

        // ---- refill this record buffer with the step after next, then
        //      start the loads of the descriptor of the one after it ----
        if (tid == 0 && pf_ok) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            load_ops(b, pm);
            pf_adv(pm.np);
        }
        // ---- end of tile: flush the tile's outputs with coalesced atomics
        //      (the next writes to ACC come two barriers later) ----
        if (cm.last) {
            zf* yc = a.y + col0(cm.item);
            for (int idx = tid; idx < NSLOT * NR * NB; idx += NT) {
                const int slot = idx / (NR * NB);
                const int rem = idx - slot * (NR * NB);
                const int rr = rem / NB, el = rem - rr * NB;
                // grouped tiles carry their sphere-list row in z (i0 << 16 | j0 here)
                const int sph = a.tsph ? a.tsph[(size_t)((cm.i0 << 16) | cm.j0) * NSLOT + slot] : ((slot < TILE_B) ? (cm.i0 + slot) : (cm.j0 + slot - TILE_B));
                zf* av;
                if constexpr (CS == NB2) {
                    av = ACC + (size_t)slot * SS + rem;
                } else {
                    const int pe = el >= NB2 ? 1 : 0;
                    av = ACC + (size_t)slot * SS + (size_t)(rr * 2 + pe) * CS + (el - pe * NB2);
                }
                if (a.tsph ? sph >= 0 : (!(cm.diag && slot >= TILE_B) && sph < a.nsph)) {
                    const size_t sb = tile_sphere_base<SO>(a, sph, NB);
                    red_add<float>(yc + (size_t)rr * a.ld + sb + el, *av);
                }
                *av = mk(0.f, 0.f);
            }
            if (cm.item + G >= NI) break;
        }
    }
}

// ---------------------------------------------------------------------------
// host: the work schedule of one (L, H)
// ---------------------------------------------------------------------------
struct Unit {
    int deg, j0, j1;
    double cost;
};

// Per-lane cost estimates (FMA instructions and their overheads) of a unit:
// a fixed part (loading the column's inputs) and a part per row set / row.
static void unit_costs(int ph, int deg, int L, int H, int& j0, int& j1, double& fix, double& per)
{
    if (ph == 1) {   // C: rows n = m1..L
        const int m1 = std::max(1, deg), dim = L - m1 + 1;
        const int qn = deg == 0 ? (dim + 1) / 2 : dim, qh = (qn + H - 1) / H;
        int lg = 0;
        while ((1 << lg) < H) lg++;
        j0 = m1;
        j1 = L + 1;
        fix = 6.0 * qh + 8.0;
        per = 4.0 * qh + 1.5 + (deg == 0 ? 2.0 : 4.0) * lg + 3.0;
    } else {         // AB / D: row sets j of degree n, rows k = H j + h
        const int n = deg, w = 2 * n + 1;
        j0 = 0;
        j1 = (n + H) / H;
        fix = (ph == 0 ? 5.0 : 3.0) * w + 8.0;
        per = (double)rr_rw(n) + (ph == 0 ? 8.0 : 16.0);
    }
}

static RowSched make_sched(int L, int H)
{
    RowSched s{};
    s.fits = 1;
    for (int ph = 0; ph < 3; ph++) {
        std::vector<Unit> us;
        double total = 0.0;
        const int d0 = ph == 1 ? 0 : 1;
        for (int d = d0; d <= L; d++) {
            int j0, j1;
            double fix, per;
            unit_costs(ph, d, L, H, j0, j1, fix, per);
            total += fix + per * (j1 - j0);
        }
        const double target = total / 8.0;
        for (int d = d0; d <= L; d++) {
            int j0, j1;
            double fix, per;
            unit_costs(ph, d, L, H, j0, j1, fix, per);
            const int J = j1 - j0;
            int pieces = (int)std::lround((fix + per * J) / (0.6 * target));
            pieces = std::max(1, std::min(J, pieces));
            for (int k = 0; k < pieces; k++) {
                const int a0 = j0 + (J * k) / pieces, a1 = j0 + (J * (k + 1)) / pieces;
                us.push_back({d, a0, a1, fix + per * (a1 - a0)});
            }
        }
        std::stable_sort(us.begin(), us.end(), [](const Unit& x, const Unit& y) { return x.cost > y.cost; });
        std::vector<std::vector<Unit>> per_warp(8);
        double load[8] = {0};
        for (const Unit& u : us) {
            int w = (int)(std::min_element(load, load + 8) - load);
            load[w] += u.cost;
            per_warp[w].push_back(u);
        }
        int k = 0;
        for (int w = 0; w < 8; w++) {
            s.first[ph][w] = k;
            for (const Unit& u : per_warp[w]) {
                if (k < RS_MAXU) s.unit[ph][k] = (unsigned)u.deg | ((unsigned)u.j0 << 8) | ((unsigned)u.j1 << 16);
                k++;
            }
        }
        s.first[ph][8] = k;
        if (k > RS_MAXU) s.fits = 0;
    }
    return s;
}

static const RowSched& sched_for(int L, int H)
{
    static std::mutex mu;
    static std::map<int, RowSched> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(L * 64 + H);
    if (it == cache.end()) it = cache.emplace(L * 64 + H, make_sched(L, H)).first;
    return it->second;
}

template <int L, int NR, int MB> static int launch_mb(const TiledArgs<float>& a, int nsm, cudaStream_t st)
{
    constexpr size_t smem = rows_smem<L, NR>();
    if (smem > 227 * 1024) return -1;
    constexpr int H = 32 / (rows_pp<L, NR>() * 4 * NR);
    const RowSched& sc = sched_for(L, H);
    if (!sc.fits) return -1;
    auto kern = a.soff ? translate_rows_kernel<L, NR, true, MB> : translate_rows_kernel<L, NR, false, MB>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = (int)((228 * 1024) / (smem + 1024));
    per_sm = std::max(1, std::min(MB, per_sm));
    if (a.ctas_per_sm >= 1 && a.ctas_per_sm < per_sm) per_sm = a.ctas_per_sm;
    int blocks = std::min(nsm * per_sm, a.ntiles * a.nchunk);
    if (blocks < 1) return 0;
    kern<<<blocks, 256, smem, st>>>(a, sc);
    launch_counter() += 1;
    return 0;
}

// a pass whose work items do not fill one wave of three CTAs per SM runs the
// two-CTA instance, faster per CTA without the small orders' spills (30
// spheres of order 5, 2 columns: 33.3 us with the three-CTA instance, 29.2 us
// with this one)
template <int L, int NR> static int launch_LN(const TiledArgs<float>& a, int nsm, cudaStream_t st)
{
    constexpr int MB = rows_minb<L>();
    if constexpr (MB == 3) {
        if (a.ntiles * a.nchunk < 3 * nsm || (a.ctas_per_sm >= 1 && a.ctas_per_sm < 3)) return launch_mb<L, NR, 2>(a, nsm, st);
    }
    return launch_mb<L, NR, MB>(a, nsm, st);
}

template <int L> static int launch_L(const TiledArgs<float>& a, int nsm, cudaStream_t st)
{
    switch (a.nrhs) {
    case 1: return launch_LN<L, 1>(a, nsm, st);
    case 2: return launch_LN<L, 2>(a, nsm, st);
    case 4: return launch_LN<L, 4>(a, nsm, st);
    default: return -1;
    }
}

}  // namespace

bool rows_supported(int L, int nrhs) { return L >= 3 && L <= 10 && (nrhs == 1 || nrhs == 2 || nrhs == 4); }

int launch_translate_rows(const TiledArgs<float>& a, int L, int nsm, cudaStream_t st)
{
    switch (L) {
    case 3: return launch_L<3>(a, nsm, st);
    case 4: return launch_L<4>(a, nsm, st);
    case 5: return launch_L<5>(a, nsm, st);
    case 6: return launch_L<6>(a, nsm, st);
    case 7: return launch_L<7>(a, nsm, st);
    case 8: return launch_L<8>(a, nsm, st);
    case 9: return launch_L<9>(a, nsm, st);
    case 10: return launch_L<10>(a, nsm, st);
    default: return -1;
    }
}
