// opgen.cu -- FP64 generation of the per-pair VSWF translation operators on the
// device, in the folded layout the translation kernel streams.
//
// A pair (i, j), i < j, gets one operator record, computed once per cluster
// (MSTM's store_translation_matrix=.true. mode, december2023/mstm-modules-33.f90:6390-6525):
//   - e^{i phi} of the pair vector r_i - r_j                (cartosphere/ephicoef, modules:1986-2004, 2075-2085)
//   - Wigner-d d^n_{km}(theta) for |k| <= min(n,nmin), folded
//     by the symmetry d_{-k,-m} = (-1)^{k+m} d_{k,m} into
//     E_n(k,m) = (d_{k,m} + (-1)^m d_{k,-m})/2  (0<=k<=kk, 0<=m<=n) and
//     O_n(k,m) = (d_{k,m} - (-1)^m d_{k,-m})/2  (1<=k<=kk, 1<=m<=n)   (rotcoef, modules:1098-1175)
//   - axial translation blocks Z_m(n,l), m = 0..nmin, both modes for m>0 and
//     one mode for m=0; the -m block equals the +m block with modes swapped
//     (axialtrancoefrecurrence, modules:1566-1676; constants axialtrancoefinit, modules:1680-1722).
//     Every element is the vector-coupling sum over the Hankel orders w that the
//     reference uses for the first row and the last column of each block,
//     Z_m(n,l) = sum_w vcc(n, l(l+1)+m, w) xi_w / z with the odd-offset terms
//     times +-i for the two modes; the reference fills the interior by a
//     three-term recurrence in n instead, the same quantity up to rounding.
//     The sums are independent.
// Three launches, each shaped for its own parallelism: the per-pair scalars and
// the Riccati-Hankel functions xi_w / z (serial in w) one thread per pair,
// into a scratch of 2 LMAX + 1 complex per pair; the Wigner-d rows (serial in
// the degree and the restricted index, parallel over the other index) one
// warp per pair; the axial blocks one CTA per pair, a thread per (m, n, l).
// Record layout (units of the storage type T, double or float):
//   [0,2)            e^{i phi}
//   [2, 2+R)         E_1, O_1, E_2, O_2, ...   (row-major, restricted index first)
//   [2+R, 2+R+2Z)    Z_0[p=0], Z_1[p=0], Z_1[p=1], Z_2[p=0], ... complex, [row n][col l]
//   padding to a multiple of 4 units.
// FP32 records of clusters of one sphere order (the tiled passes) use the row
// layout of translate_rows.cuh instead: the same values, rows 16-byte aligned.
#include "common.cuh"
#include "special.cuh"
#include "kernels.cuh"
#include "translate_rows.cuh"

#define DW (2 * MSTMG_LMAX + 1)
#define XIW (2 * MSTMG_LMAX + 1)   // Hankel orders w = 0 .. nt + ns <= 2 LMAX per pair

static_assert(2 * MSTMG_LMAX - 1 <= 32, "the m = 0 recurrence gives each lane one k");

struct PairGeom {
    int i, j, nt, ns, nmin, nmax;
    double r, ct;
    zd ephi;
    bool ok;
};

// cartosphere (modules:1986-2004) of r_i - r_j; ok is false for coincident centres
__device__ __forceinline__ PairGeom pair_geom(const OpGenArgs& a, int q)
{
    PairGeom g;
    g.i = a.pairs[q].x;
    g.j = a.pairs[q].y;
    g.nt = a.order[g.i];
    g.ns = a.order[g.j];
    g.nmin = g.nt < g.ns ? g.nt : g.ns;
    g.nmax = g.nt > g.ns ? g.nt : g.ns;
    const double rv0 = a.pos[3 * g.i] - a.pos[3 * g.j], rv1 = a.pos[3 * g.i + 1] - a.pos[3 * g.j + 1],
                 rv2 = a.pos[3 * g.i + 2] - a.pos[3 * g.j + 2];
    const double rr = rv0 * rv0 + rv1 * rv1 + rv2 * rv2;
    if (rr == 0.0) {
        g.r = 0.0;
        g.ct = 1.0;
        g.ephi = mk(1.0, 0.0);
    } else {
        g.r = sqrt(rr);
        g.ct = rv2 / g.r;
        if (rv0 == 0.0 && rv1 == 0.0) g.ephi = mk(1.0, 0.0);
        else {
            const double h = sqrt(rv0 * rv0 + rv1 * rv1);
            g.ephi = mk(rv0 / h, rv1 / h);
        }
    }
    g.ok = rr >= 1.0e-12;
    return g;
}

// e^{i phi} into the record and xi_w(z) / z, z = r m_medium, w = 0 .. nt + ns
// into the scratch (psi_w(z) / z for regular translations): one thread per pair
__global__ void __launch_bounds__(128) opgen_pair_kernel(OpGenArgs a)
{
    zd hs[2 * (XIW + 1)];   // spherical Bessel scratch of the complex-argument branch
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < a.npairs; q += gridDim.x * blockDim.x) {
        const PairGeom g = pair_geom(a, q);
        if (!g.ok) {
            atomicExch(a.err, MSTMG_ERR_UNSUPPORTED);
            continue;
        }
        const long long off = a.opoff[q];
        if (a.op64) {
            a.op64[off] = g.ephi.x;
            a.op64[off + 1] = g.ephi.y;
        }
        if (a.op32 && a.row32) {
            // row records: the powers e^{i m phi}, m = 0..nt, by the recurrence in FP64
            float* h = a.op32 + (long long)q * a.row32;
            zd e = mk(1.0, 0.0);
            for (int m = 0; m <= g.nt; m++) {
                h[2 * m] = (float)e.x;
                h[2 * m + 1] = (float)e.y;
                e = e * g.ephi;
            }
        } else if (a.op32) {
            a.op32[off] = (float)g.ephi.x;
            a.op32[off + 1] = (float)g.ephi.y;
        }
        zd* xi = a.xi + (size_t)q * XIW;
        const int nl = g.nt + g.ns;
        const zd z = a.pmed ? mk(g.r * a.pmed[2 * q], g.r * a.pmed[2 * q + 1]) : mk(g.r * a.rimed_re, g.r * a.rimed_im);
        if (a.regular) mstm_cricbessel(nl, z, xi, hs);
        else mstm_crichankel(nl, z, xi, hs);
        for (int k = 0; k <= nl; k++) xi[k] = cdiv(xi[k], z);
    }
}

// rotcoef(ct, nmin, nmax) (modules:1098-1175), degree by degree, folded into
// E_n, O_n: one warp per pair.  Per-warp shared scratch: D, rows k = 0..kk of
// (2 LMAX + 1) doubles (restricted index first), and the m = 0 columns dk0,
// dk01 of the degree recurrence (index -LMAX-1 .. LMAX+1).
#define ROT_WARP_DOUBLES ((MSTMG_LMAX + 1) * DW + 2 * (2 * MSTMG_LMAX + 3))
__global__ void __launch_bounds__(128) opgen_rot_kernel(OpGenArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* D = reinterpret_cast<double*>(smem_raw) + (size_t)warp * ROT_WARP_DOUBLES;
    double* dk0 = D + (MSTMG_LMAX + 1) * DW + (MSTMG_LMAX + 1);
    double* dk01 = dk0 + (2 * MSTMG_LMAX + 3);
    const int nwarps = blockDim.x >> 5;
    const double* fnr = a.fnr;
    const double* rfnr = a.rfnr;
    for (int q = blockIdx.x * nwarps + warp; q < a.npairs; q += gridDim.x * nwarps) {
        const PairGeom g = pair_geom(a, q);
        if (!g.ok) continue;
        const int nmin = g.nmin, nmax = g.nmax;
        const double ct = g.ct;
        const long long off = a.opoff[q];
        double* rec64 = a.op64 ? a.op64 + off : nullptr;
        float* rec32 = (a.op32 && !a.row32) ? a.op32 + off : nullptr;
        float* row32 = (a.op32 && a.row32) ? a.op32 + (size_t)q * a.row32 : nullptr;
        const double sbe = (fabs(ct) >= 1.0) ? 0.0 : sqrt(fabs((1.0 + ct) * (1.0 - ct)));
        const double cbe2 = 0.5 * (1.0 + ct), sbe2 = 0.5 * (1.0 - ct);
        for (int k = lane; k < 2 * MSTMG_LMAX + 3; k += 32) {
            dk0[k - (MSTMG_LMAX + 1)] = 0.0;
            dk01[k - (MSTMG_LMAX + 1)] = 0.0;
        }
        __syncwarp();
        if (lane == 0) {
            dk0[0] = 1.0;
            dk01[0] = 0.0;
        }
        __syncwarp();
        int sgn = 1;
        double sben = 1.0;
        for (int n = 1; n <= nmax; n++) {
            const int kk = n < nmin ? n : nmin;
            sgn = -sgn;
            sben = sben * sbe / 2.0;
            if (sben < 1.0e-30) sben = 0.0;
            // m = 0 column by the three-term recurrence in n (lane k + n - 1 takes
            // k = -n+1 .. n-1: at most 2 LMAX - 1 <= 31 lanes)
            {
                const int k = -n + 1 + lane;
                const bool on = k <= n - 1;
                double newv = 0.0;
                if (on)
                    newv = (ct * (double)(n + n - 1) * dk0[k] - fnr[n - k - 1] * fnr[n + k - 1] * dk01[k]) * (rfnr[n + k] * rfnr[n - k]);
                __syncwarp();
                if (on) {
                    dk01[k] = dk0[k];
                    dk0[k] = newv;
                }
            }
            if (lane == 0) {
                dk0[n] = sgn * sben * a.bcofd[n];
                dk0[-n] = sgn * dk0[n];
                dk01[n] = 0.0;
                dk01[-n] = 0.0;
            }
            __syncwarp();
            for (int k = -n + lane; k <= n; k += 32) D[k + MSTMG_LMAX] = dk0[k];
            __syncwarp();
            for (int m = 1; m <= kk; m++) {
                const double fmn = rfnr[n - m + 1] * rfnr[n + m];
                const int m1 = m - 1;
                // rows with a negative restricted index are never read (the
                // fold below takes rows 0..kk), so only row m is written
                for (int k = -n + lane; k <= n; k += 32) {
                    const double dkm1 = (k == -n) ? 0.0 : D[m1 * DW + (k - 1 + MSTMG_LMAX)];
                    const double dkn1 = (k == n) ? 0.0 : D[m1 * DW + (k + 1 + MSTMG_LMAX)];
                    const double v = (fnr[n + k] * fnr[n - k + 1] * cbe2 * dkm1 - fnr[n - k] * fnr[n + k + 1] * sbe2 * dkn1
                                      - (double)k * sbe * D[m1 * DW + (k + MSTMG_LMAX)]) * fmn;
                    D[m * DW + (k + MSTMG_LMAX)] = v;
                }
                __syncwarp();
            }
            // fold into E_n, O_n
            const int roff = 2 + op_rot_offset(n, nmin);
            const int ne = (kk + 1) * (n + 1), no = kk * n;
            // row and column of flat element e by a float reciprocal: e < 2^10 and
            // e / (n + 1) sits at least 1 / (2 (n + 1)) from the next integer
            const float rn1 = 1.0f / (float)(n + 1), rn = 1.0f / (float)n;
            for (int e = lane; e < ne + no; e += 32) {
                double v;
                if (e < ne) {
                    const int rr_ = (int)(((float)e + 0.5f) * rn1), f = e - rr_ * (n + 1);
                    const double dp = D[rr_ * DW + (f + MSTMG_LMAX)];
                    v = (f == 0) ? 0.5 * dp : 0.5 * (dp + pm1(f) * D[rr_ * DW + (-f + MSTMG_LMAX)]);
                } else {
                    const int e2 = e - ne;
                    const int qq = (int)(((float)e2 + 0.5f) * rn);
                    const int rr_ = 1 + qq, f = 1 + e2 - qq * n;
                    const double dp = D[rr_ * DW + (f + MSTMG_LMAX)];
                    v = 0.5 * (dp - pm1(f) * D[rr_ * DW + (-f + MSTMG_LMAX)]);
                }
                if (rec64) rec64[roff + e] = v;
                if (rec32) rec32[roff + e] = (float)v;
                if (row32) {
                    // row layout: row k of degree n is [E(k,0), 0, E(k,1), O(k,1), ..., E(k,n), O(k,n)]
                    int k, slot;
                    if (e < ne) {
                        k = (int)(((float)e + 0.5f) * rn1);
                        slot = 2 * (e - k * (n + 1));
                    } else {
                        const int qq = (int)(((float)(e - ne) + 0.5f) * rn);
                        k = 1 + qq;
                        slot = 2 * (1 + (e - ne) - qq * n) + 1;
                    }
                    row32[rr_rot_off(n, nmax) + k * rr_rw(n) + slot] = (float)v;
                }
            }
            __syncwarp();
        }
    }
}

// axial translation blocks (itype 3, outgoing; itype 1, regular, with the
// Bessel functions in the scratch), one CTA per pair: the
// pair's xi_w / z staged in shared memory, thread t takes the mode-0
// elements t, t + 128, ... of the concatenated blocks Z_0, Z_1, ...
__global__ void __launch_bounds__(128) opgen_axial_kernel(OpGenArgs a)
{
    __shared__ zd xs[XIW];
    const int vn = a.vnmax;
    for (int q = blockIdx.x; q < a.npairs; q += gridDim.x) {
        const PairGeom g = pair_geom(a, q);
        if (!g.ok) continue;   // uniform over the CTA
        const int nt = g.nt, ns = g.ns, nmin = g.nmin;
        __syncthreads();   // the previous pair's reads of xs are done
        for (int k = threadIdx.x; k <= nt + ns; k += blockDim.x) xs[k] = a.xi[(size_t)q * XIW + k];
        __syncthreads();
        const long long off = a.opoff[q];
        double* rec64 = a.op64 ? a.op64 + off : nullptr;
        float* rec32 = (a.op32 && !a.row32) ? a.op32 + off : nullptr;
        float* row32 = (a.op32 && a.row32) ? a.op32 + (size_t)q * a.row32 : nullptr;
        const int zbase = 2 + op_rot_size(g.nmax, nmin);
        // walk the blocks forward: block m holds rc(m) elements, mode-1 copies
        // after the mode-0 ones for m > 0 (op_z_offset)
        int m = 0, e = threadIdx.x, zoff = 0;
        while (m <= nmin) {
            const int m1 = m < 1 ? 1 : m;
            const int cols = ns - m1 + 1, rc = (nt - m1 + 1) * cols;
            if (e >= rc) {
                e -= rc;
                zoff += (m == 0 ? 1 : 2) * rc;
                m++;
                continue;
            }
            const int qn = (int)(((float)e + 0.5f) * (1.0f / (float)cols));   // e / cols (e < 2^10)
            const int n = m1 + qn, l = m1 + e - qn * cols;
            const int wmin = n > l ? n - l : l - n, wmax = n + l, ml = l * (l + 1) + m;
            const double* vc = a.vcc + (size_t)(n - 1) + (size_t)vn * (size_t)(ml - 1);
            const size_t ws = (size_t)vn * vn * (vn + 2);
            zd s1 = mk(0.0, 0.0), s2 = mk(0.0, 0.0);
            for (int w = wmin; w <= wmax; w += 2) s1 = s1 + vc[ws * w] * xs[w];
            for (int w = wmin + 1; w <= wmax - 1; w += 2) s2 = s2 + vc[ws * w] * xs[w];
            s2 = imul(s2);
            const zd v0 = s1 + s2, v1 = s1 - s2;
            const int zo = zbase + 2 * (zoff + e);
            if (rec64) {
                rec64[zo] = v0.x;
                rec64[zo + 1] = v0.y;
                if (m > 0) {
                    rec64[zo + 2 * rc] = v1.x;
                    rec64[zo + 2 * rc + 1] = v1.y;
                }
            }
            if (row32) {
                // row layout: m = 0 rows of Z_0(n, .); m > 0 rows of (Z_m^0, Z_m^1)(n, l) pairs
                if (m == 0) {
                    float* z = row32 + rr_z_off(0, nt) + (n - 1) * rr_zw0(nt) + 2 * (l - 1);
                    z[0] = (float)v0.x;
                    z[1] = (float)v0.y;
                } else {
                    float* z = row32 + rr_z_off(m, nt) + (n - m1) * 4 * rr_zq(cols) + 4 * (l - m1);
                    z[0] = (float)v0.x;
                    z[1] = (float)v0.y;
                    z[2] = (float)v1.x;
                    z[3] = (float)v1.y;
                }
            }
            if (rec32) {
                rec32[zo] = (float)v0.x;
                rec32[zo + 1] = (float)v0.y;
                if (m > 0) {
                    rec32[zo + 2 * rc] = (float)v1.x;
                    rec32[zo + 2 * rc + 1] = (float)v1.y;
                }
            }
            e += blockDim.x;
        }
    }
}

size_t opgen_xi_scratch(int npairs) { return (size_t)npairs * XIW; }

void launch_opgen(const OpGenArgs& a, int nsm, cudaStream_t st)
{
    if (a.npairs <= 0) return;
    int b1 = (a.npairs + 127) / 128;
    if (b1 > nsm * 16) b1 = nsm * 16;
    opgen_pair_kernel<<<b1, 128, 0, st>>>(a);
    const int warps = 4;
    const size_t smem = sizeof(double) * ROT_WARP_DOUBLES * warps;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(opgen_rot_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    int b2 = (a.npairs + warps - 1) / warps;
    if (b2 > nsm * 16) b2 = nsm * 16;
    opgen_rot_kernel<<<b2, warps * 32, smem, st>>>(a);
    int b3 = a.npairs < nsm * 16 ? a.npairs : nsm * 16;
    opgen_axial_kernel<<<b3, 128, 0, st>>>(a);
    launch_counter() += 3;
}
