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
//     (axialtrancoefrecurrence, modules:1566-1676; constants axialtrancoefinit, modules:1680-1722)
// Record layout (units of the storage type T, double or float):
//   [0,2)            e^{i phi}
//   [2, 2+R)         E_1, O_1, E_2, O_2, ...   (row-major, restricted index first)
//   [2+R, 2+R+2Z)    Z_0[p=0], Z_1[p=0], Z_1[p=1], Z_2[p=0], ... complex, [row n][col l]
//   padding to a multiple of 4 units.
#include "common.cuh"
#include "special.cuh"
#include "kernels.cuh"

struct OpGenScratch {
    double* D;      // (2*LMAX+1)^2 : D[(k+LMAX)*(2LMAX+1) + (m+LMAX)], first index restricted
    double* dk0;    // 2*LMAX+3
    double* dk01;
    zd* xi;         // 2*LMAX+2
    zd* hs;         // Hankel scratch 2*(2*LMAX+2)
    zd* act;        // 2 * LMAX * LMAX
};

#define DW (2 * MSTMG_LMAX + 1)

__global__ void __launch_bounds__(128) opgen_kernel(OpGenArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int per_warp_bytes = sizeof(double) * (DW * DW + 2 * (2 * MSTMG_LMAX + 3)) + sizeof(zd) * ((2 * MSTMG_LMAX + 2) * 3 + 2 * MSTMG_LMAX * MSTMG_LMAX);
    unsigned char* base = smem_raw + warp * ((per_warp_bytes + 15) & ~15);
    double* D = (double*)base;
    double* dk0 = D + DW * DW + (MSTMG_LMAX + 1);      // index -LMAX-1..LMAX+1
    double* dk01 = dk0 + (2 * MSTMG_LMAX + 3);
    zd* xi = (zd*)(D + DW * DW + 2 * (2 * MSTMG_LMAX + 3));
    zd* hs = xi + (2 * MSTMG_LMAX + 2);
    zd* act = hs + 2 * (2 * MSTMG_LMAX + 2);
    const int nwarps = blockDim.x >> 5;
    const double* fnr = a.fnr;
    const int vn = a.vnmax;
#define VCC(n, ml, w) a.vcc[((n) - 1) + (size_t)vn * (((ml) - 1) + (size_t)vn * (vn + 2) * (w))]
#define FCI(arr, m, l) arr[((m) + vn) + (2 * vn + 1) * ((l) - 1)]

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
            // m = 0 column by the three-term recurrence in n (lanes over k)
            double newv[2];
            int cnt = 0;
            for (int k = -n + 1 + lane; k <= n - 1; k += 32) {
                double dkt = dk01[k];
                double old = dk0[k];
                newv[cnt & 1] = (ct * (double)(n + n - 1) * old - fnr[n - k - 1] * fnr[n + k - 1] * dkt) / (fnr[n + k] * fnr[n - k]);
                cnt++;
            }
            __syncwarp();
            cnt = 0;
            for (int k = -n + 1 + lane; k <= n - 1; k += 32) {
                dk01[k] = dk0[k];
                dk0[k] = newv[cnt & 1];
                cnt++;
            }
            if (lane == 0) {
                dk0[n] = sgn * sben * a.bcofd[n];
                dk0[-n] = sgn * dk0[n];
                dk01[n] = 0.0;
                dk01[-n] = 0.0;
            }
            __syncwarp();
            for (int k = -n + lane; k <= n; k += 32) D[(0 + MSTMG_LMAX) * DW + (k + MSTMG_LMAX)] = dk0[k];
            __syncwarp();
            int im = 1;
            for (int m = 1; m <= kk; m++) {
                im = -im;
                double fmn = 1.0 / fnr[n - m + 1] / fnr[n + m];
                int m1 = m - 1;
                for (int k = -n + lane; k <= n; k += 32) {
                    double dkm1 = (k == -n) ? 0.0 : D[(m1 + MSTMG_LMAX) * DW + (k - 1 + MSTMG_LMAX)];
                    double dkn1 = (k == n) ? 0.0 : D[(m1 + MSTMG_LMAX) * DW + (k + 1 + MSTMG_LMAX)];
                    double v = (fnr[n + k] * fnr[n - k + 1] * cbe2 * dkm1 - fnr[n - k] * fnr[n + k + 1] * sbe2 * dkn1
                                - (double)k * sbe * D[(m1 + MSTMG_LMAX) * DW + (k + MSTMG_LMAX)]) * fmn;
                    D[(m + MSTMG_LMAX) * DW + (k + MSTMG_LMAX)] = v;
                    D[(-m + MSTMG_LMAX) * DW + (-k + MSTMG_LMAX)] = v * pm1(k) * im;
                }
                __syncwarp();
            }
            // fold into E_n, O_n
            int roff = 2 + op_rot_offset(n, nmin);
            int ne = (kk + 1) * (n + 1), no = kk * n;
            for (int e = lane; e < ne + no; e += 32) {
                double v;
                if (e < ne) {
                    int rr_ = e / (n + 1), f = e % (n + 1);
                    double dp = D[(rr_ + MSTMG_LMAX) * DW + (f + MSTMG_LMAX)];
                    v = (f == 0) ? 0.5 * dp : 0.5 * (dp + pm1(f) * D[(rr_ + MSTMG_LMAX) * DW + (-f + MSTMG_LMAX)]);
                } else {
                    int e2 = e - ne;
                    int rr_ = 1 + e2 / n, f = 1 + e2 % n;
                    double dp = D[(rr_ + MSTMG_LMAX) * DW + (f + MSTMG_LMAX)];
                    v = 0.5 * (dp - pm1(f) * D[(rr_ + MSTMG_LMAX) * DW + (-f + MSTMG_LMAX)]);
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
            for (int k = 0; k <= nl; k++) xi[k] = cdiv(xi[k], z);
        }
        __syncwarp();
        const int zbase = 2 + op_rot_size(nmax, nmin);
        for (int m = 0; m <= nmin; m++) {
            int m1 = m < 1 ? 1 : m;
            int rows = nt - m1 + 1, cols = ns - m1 + 1;
#define ACT(n, l, p) act[(((p) * MSTMG_LMAX) + ((n) - 1)) * MSTMG_LMAX + ((l) - 1)]
            // first row n = m1, l = m1..ns ; last column l = ns, n = m1+1..nt
            for (int e = lane; e < cols + (rows - 1); e += 32) {
                int n, l;
                if (e < cols) { n = m1; l = m1 + e; }
                else { n = m1 + 1 + (e - cols); l = ns; }
                int wmin = n > l ? n - l : l - n, wmax = n + l, ml = l * (l + 1) + m;
                zd s1 = mk(0.0, 0.0), s2 = mk(0.0, 0.0);
                for (int w = wmin; w <= wmax; w += 2) s1 = s1 + VCC(n, ml, w) * xi[w];
                for (int w = wmin + 1; w <= wmax - 1; w += 2) s2 = s2 + VCC(n, ml, w) * xi[w];
                s2 = imul(s2);
                ACT(n, l, 0) = s1 + s2;
                ACT(n, l, 1) = s1 - s2;
            }
            __syncwarp();
            int nlmin = nt < ns ? nt : ns;
            if (m1 < nlmin) {
                for (int n = m1; n <= nt - 1; n++) {
                    for (int e = lane; e < 2 * (ns - m1); e += 32) {
                        int p = e / (ns - m1), l = m1 + e % (ns - m1);
                        double sp = (p == 0) ? 1.0 : -1.0;
                        zd v = -(ACT(n, l + 1, p) * FCI(a.fnp1, m, l))
                               + imul(sp * (FCI(a.fnc, m, l) - FCI(a.fnc, m, n)) * ACT(n, l, p));
                        if (l >= m1 + 1) v = v + ACT(n, l - 1, p) * FCI(a.fnm1, m, l);
                        if (n > m1) v = v + ACT(n - 1, l, p) * FCI(a.fnm1, m, n);
                        { double dd = FCI(a.fnp1, m, n); ACT(n + 1, l, p) = mk(v.x / dd, v.y / dd); }
                    }
                    __syncwarp();
                }
            }
            int nmodes = (m == 0) ? 1 : 2;
            int zo = zbase + 2 * op_z_offset(m, nt, ns);
            for (int e = lane; e < nmodes * rows * cols; e += 32) {
                int p = e / (rows * cols), rem = e % (rows * cols);
                int n = m1 + rem / cols, l = m1 + rem % cols;
                zd v = ACT(n, l, p);
                if (rec64) { rec64[zo + 2 * e] = v.x; rec64[zo + 2 * e + 1] = v.y; }
                if (rec32) { rec32[zo + 2 * e] = (float)v.x; rec32[zo + 2 * e + 1] = (float)v.y; }
            }
            __syncwarp();
#undef ACT
        }
    }
#undef VCC
#undef FCI
}

size_t opgen_smem_bytes(int warps)
{
    int per_warp_bytes = sizeof(double) * (DW * DW + 2 * (2 * MSTMG_LMAX + 3)) + sizeof(zd) * ((2 * MSTMG_LMAX + 2) * 3 + 2 * MSTMG_LMAX * MSTMG_LMAX);
    return (size_t)warps * ((per_warp_bytes + 15) & ~15);
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
