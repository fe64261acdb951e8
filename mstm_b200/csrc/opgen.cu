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
//     The sums are independent, so the lanes of a warp take one element each.
// Record layout (units of the storage type T, double or float):
//   [0,2)            e^{i phi}
//   [2, 2+R)         E_1, O_1, E_2, O_2, ...   (row-major, restricted index first)
//   [2+R, 2+R+2Z)    Z_0[p=0], Z_1[p=0], Z_1[p=1], Z_2[p=0], ... complex, [row n][col l]
//   padding to a multiple of 4 units.
#include "common.cuh"
#include "special.cuh"
#include "kernels.cuh"

// per-warp scratch in shared memory:
//   D    (LMAX+1) x (2 LMAX+1) doubles: D[k*DW + (m+LMAX)], restricted index k = 0..kk
//   dk0, dk01   2 LMAX+3 doubles each (index -LMAX-1 .. LMAX+1)
//   xi   2 LMAX+2 complex: Riccati-Hankel xi_w / z
//   hs   2 (2 LMAX+2) complex: Hankel scratch
#define DW (2 * MSTMG_LMAX + 1)
#define OPGEN_WARP_BYTES (sizeof(double) * ((MSTMG_LMAX + 1) * DW + 2 * (2 * MSTMG_LMAX + 3)) + sizeof(zd) * ((2 * MSTMG_LMAX + 2) * 3))

static_assert(2 * MSTMG_LMAX - 1 <= 32, "the m = 0 recurrence gives each lane one k");

// 6 CTAs of 4 warps per SM (80 registers): the warps' serial recurrences
// and table loads need the resident warps to hide their latencies
__global__ void __launch_bounds__(128, 6) opgen_kernel(OpGenArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* base = smem_raw + warp * ((OPGEN_WARP_BYTES + 15) & ~15);
    double* D = (double*)base;
    double* dk0 = D + (MSTMG_LMAX + 1) * DW + (MSTMG_LMAX + 1);      // index -LMAX-1..LMAX+1
    double* dk01 = dk0 + (2 * MSTMG_LMAX + 3);
    zd* xi = (zd*)(D + (MSTMG_LMAX + 1) * DW + 2 * (2 * MSTMG_LMAX + 3));
    zd* hs = xi + (2 * MSTMG_LMAX + 2);
    const int nwarps = blockDim.x >> 5;
    const double* fnr = a.fnr;
    const double* rfnr = a.rfnr;
    const int vn = a.vnmax;
#define VCC(n, ml, w) a.vcc[((n) - 1) + (size_t)vn * (((ml) - 1) + (size_t)vn * (vn + 2) * (w))]

    for (int q = blockIdx.x * nwarps + warp; q < a.npairs; q += gridDim.x * nwarps) {
        int i = a.pairs[q].x, j = a.pairs[q].y;
        int nt = a.order[i], ns = a.order[j];
        int nmin = nt < ns ? nt : ns, nmax = nt > ns ? nt : ns;
        double rv0 = a.pos[3 * i] - a.pos[3 * j], rv1 = a.pos[3 * i + 1] - a.pos[3 * j + 1], rv2 = a.pos[3 * i + 2] - a.pos[3 * j + 2];
        // cartosphere
        double rr = rv0 * rv0 + rv1 * rv1 + rv2 * rv2, r, ct;
        zd ephi;
        if (rr == 0.0) { r = 0.0; ct = 1.0; ephi = mk(1.0, 0.0); }
        else {
            r = sqrt(rr);
            ct = rv2 / r;
            if (rv0 == 0.0 && rv1 == 0.0) ephi = mk(1.0, 0.0);
            else { double h = sqrt(rv0 * rv0 + rv1 * rv1); ephi = mk(rv0 / h, rv1 / h); }
        }
        if (rr < 1.0e-12) { if (lane == 0) atomicExch(a.err, MSTMG_ERR_UNSUPPORTED); continue; }
        const long long off = a.opoff[q];
        double* rec64 = a.op64 ? a.op64 + off : nullptr;
        float* rec32 = a.op32 ? a.op32 + off : nullptr;
        if (lane == 0) {
            if (rec64) { rec64[0] = ephi.x; rec64[1] = ephi.y; }
            if (rec32) { rec32[0] = (float)ephi.x; rec32[1] = (float)ephi.y; }
        }
        // ---------------- rotcoef(ct, nmin, nmax), degree by degree ----------------
        double sbe = (fabs(ct) >= 1.0) ? 0.0 : sqrt(fabs((1.0 + ct) * (1.0 - ct)));
        double cbe2 = 0.5 * (1.0 + ct), sbe2 = 0.5 * (1.0 - ct);
        for (int k = lane; k < 2 * MSTMG_LMAX + 3; k += 32) { dk0[k - (MSTMG_LMAX + 1)] = 0.0; dk01[k - (MSTMG_LMAX + 1)] = 0.0; }
        __syncwarp();
        if (lane == 0) { dk0[0] = 1.0; dk01[0] = 0.0; }
        __syncwarp();
        int sgn = 1;
        double sben = 1.0;
        for (int n = 1; n <= nmax; n++) {
            int kk = n < nmin ? n : nmin;
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
            int im = 1;
            for (int m = 1; m <= kk; m++) {
                im = -im;
                const double fmn = rfnr[n - m + 1] * rfnr[n + m];
                int m1 = m - 1;
                // rows with a negative restricted index are never read (the
                // fold below takes rows 0..kk), so only row m is written
                for (int k = -n + lane; k <= n; k += 32) {
                    double dkm1 = (k == -n) ? 0.0 : D[m1 * DW + (k - 1 + MSTMG_LMAX)];
                    double dkn1 = (k == n) ? 0.0 : D[m1 * DW + (k + 1 + MSTMG_LMAX)];
                    double v = (fnr[n + k] * fnr[n - k + 1] * cbe2 * dkm1 - fnr[n - k] * fnr[n + k + 1] * sbe2 * dkn1
                                - (double)k * sbe * D[m1 * DW + (k + MSTMG_LMAX)]) * fmn;
                    D[m * DW + (k + MSTMG_LMAX)] = v;
                }
                __syncwarp();
            }
            // fold into E_n, O_n
            int roff = 2 + op_rot_offset(n, nmin);
            const int ne = (kk + 1) * (n + 1), no = kk * n;
            // row and column of flat element e by a float reciprocal: e < 2^10 and
            // e / (n + 1) sits at least 1 / (2 (n + 1)) from the next integer
            const float rn1 = 1.0f / (float)(n + 1), rn = 1.0f / (float)n;
            for (int e = lane; e < ne + no; e += 32) {
                double v;
                if (e < ne) {
                    const int rr_ = (int)(((float)e + 0.5f) * rn1), f = e - rr_ * (n + 1);
                    double dp = D[rr_ * DW + (f + MSTMG_LMAX)];
                    v = (f == 0) ? 0.5 * dp : 0.5 * (dp + pm1(f) * D[rr_ * DW + (-f + MSTMG_LMAX)]);
                } else {
                    const int e2 = e - ne;
                    const int q = (int)(((float)e2 + 0.5f) * rn);
                    const int rr_ = 1 + q, f = 1 + e2 - q * n;
                    double dp = D[rr_ * DW + (f + MSTMG_LMAX)];
                    v = 0.5 * (dp - pm1(f) * D[rr_ * DW + (-f + MSTMG_LMAX)]);
                }
                if (rec64) rec64[roff + e] = v;
                if (rec32) rec32[roff + e] = (float)v;
            }
            __syncwarp();
        }
        // ---------------- axial coefficients (itype 3, outgoing) ----------------
        const int nl = nt + ns;
        if (lane == 0) {
            zd z = mk(r * a.rimed_re, r * a.rimed_im);
            mstm_crichankel(nl, z, xi, hs);
        }
        __syncwarp();
        {
            const zd z = mk(r * a.rimed_re, r * a.rimed_im);
            for (int k = lane; k <= nl; k += 32) xi[k] = cdiv(xi[k], z);
        }
        __syncwarp();
        const int zbase = 2 + op_rot_size(nmax, nmin);
        for (int m = 0; m <= nmin; m++) {
            const int m1 = m < 1 ? 1 : m;
            const int rows = nt - m1 + 1, cols = ns - m1 + 1, rc = rows * cols;
            const int zo = zbase + 2 * op_z_offset(m, nt, ns);
            const float rcols = 1.0f / (float)cols;
            for (int e = lane; e < rc; e += 32) {
                const int qn = (int)(((float)e + 0.5f) * rcols);   // e / cols, exact as in the fold above
                const int n = m1 + qn, l = m1 + e - qn * cols;
                const int wmin = n > l ? n - l : l - n, wmax = n + l, ml = l * (l + 1) + m;
                zd s1 = mk(0.0, 0.0), s2 = mk(0.0, 0.0);
                for (int w = wmin; w <= wmax; w += 2) s1 = s1 + VCC(n, ml, w) * xi[w];
                for (int w = wmin + 1; w <= wmax - 1; w += 2) s2 = s2 + VCC(n, ml, w) * xi[w];
                s2 = imul(s2);
                const zd v0 = s1 + s2, v1 = s1 - s2;
                if (rec64) {
                    rec64[zo + 2 * e] = v0.x;
                    rec64[zo + 2 * e + 1] = v0.y;
                    if (m > 0) {
                        rec64[zo + 2 * (rc + e)] = v1.x;
                        rec64[zo + 2 * (rc + e) + 1] = v1.y;
                    }
                }
                if (rec32) {
                    rec32[zo + 2 * e] = (float)v0.x;
                    rec32[zo + 2 * e + 1] = (float)v0.y;
                    if (m > 0) {
                        rec32[zo + 2 * (rc + e)] = (float)v1.x;
                        rec32[zo + 2 * (rc + e) + 1] = (float)v1.y;
                    }
                }
            }
        }
        __syncwarp();
    }
#undef VCC
}

size_t opgen_smem_bytes(int warps)
{
    return (size_t)warps * ((OPGEN_WARP_BYTES + 15) & ~15);
}

void launch_opgen(const OpGenArgs& a, int nsm, cudaStream_t st)
{
    int warps = 4;
    size_t smem = opgen_smem_bytes(warps);
    static bool attr = false;
    if (!attr) { cudaFuncSetAttribute(opgen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); attr = true; }
    int blocks = (a.npairs + warps - 1) / warps;
    int cap = nsm * 16;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    opgen_kernel<<<blocks, warps * 32, smem, st>>>(a);
    launch_counter() += 1;
}
