// ranorient.cu -- orientation-averaged scattering matrix from the cluster T
// matrix (ranorientscatmatrix, december2023/mstm-scatprops-26.f90:1963-2530,
// and ranorienscatmatrixcalc, :2538-2592), FP64 sums over the single-precision
// T matrix exactly as the reference keeps it after reading the T-matrix file.
//
//   ro_prep_kernel   complex(4) copy of T with the symmetric rows filled and
//                    the (beam-free) GB modification applied; per-order traces
//   ro_dm_kernel     one CTA per (w, v) term of the big loop: the am / bm
//                    contractions in shared memory, then dm(u,ku,n,p,n1,p1)
//                    += bm bm* with FP64 atomics (the reference's allreduce)
//   ro_coef_kernel   one CTA per GSF degree w: fm, then aw/bw/cw/dw and the
//                    16 expansion coefficients sm(:,:,w), smcf(:,:,w)
//   ro_calc_kernel   one CTA per polar angle: generalised spherical functions
//                    by the rotcoef recurrence (kmax = 2) and the 16 elements
#include "common.cuh"
#include "ranorient.cuh"
#include "vcoupling.cuh"

namespace {

__device__ __forceinline__ zd ipw(int k)
{
    int e = ((k % 4) + 4) % 4;
    return (e == 0) ? mk(1.0, 0.0) : (e == 1 ? mk(0.0, 1.0) : (e == 2 ? mk(-1.0, 0.0) : mk(0.0, -1.0)));
}
__device__ __forceinline__ void atomic_addz(zd* p, zd v)
{
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
}
__device__ __forceinline__ zd up2(float2 a) { return mk((double)a.x, (double)a.y); }

}  // namespace

// tc(p,mn,q,kl) at ((2(mn-1)+p-1) + nblkt (2(kl-1)+q-1)), as float2
__global__ void ro_prep_kernel(int nodr, const zd* tmat, float2* tc)
{
    const int nblk = nodr * (nodr + 2), nblkt = 2 * nblk;
    // one thread per (p, mn, kl): the q = 1, 2 pair of the GB modification
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)2 * nblk * nblk; e += (size_t)gridDim.x * blockDim.x) {
        int row = (int)(e % nblkt), kl = (int)(e / nblkt) + 1;
        int mn = row / 2 + 1, p = row % 2 + 1;
        int n = 1;
        while (n * (n + 2) < mn) n++;
        int l = 1;
        while (l * (l + 2) < kl) l++;
        float2 v[2];
        for (int q = 1; q <= 2; q++) {
            zd t;
            if (n <= l) {
                t = tmat[(size_t)row + (size_t)nblkt * (2 * (kl - 1) + q - 1)];
            } else {
                int m = mn - n * (n + 1), k = kl - l * (l + 1);
                int srow = 2 * (l * (l + 1) - k - 1) + (q - 1), scol = 2 * (n * (n + 1) - m - 1) + (p - 1);
                zd s = tmat[(size_t)srow + (size_t)nblkt * scol];
                // the file reader copies the single-precision value times (-1)^(m+k)
                float sg = (float)pm1(m + k);
                t = mk((double)((float)s.x * sg), (double)((float)s.y * sg));
            }
            v[q - 1] = make_float2((float)t.x, (float)t.y);
        }
        // GB-modified T matrix without a beam: pp(l,1,1) = -i^(l+1) sqrt(2l+1)/2,
        // pp(l,2,1) = pp(l,1,2) = pp(l,2,2) = -pp(l,1,1); results stored in single precision
        zd pp11 = (-0.5 * sqrt((double)(l + l + 1))) * ipw(l + 1);
        zd pp21 = -pp11, pp12 = -pp11, pp22 = pp21;
        zd a = up2(v[0]);
        zd t1 = a * pp11 + up2(v[1]) * pp12;
        float2 n1 = make_float2((float)t1.x, (float)t1.y);
        zd t2 = a * pp21 + up2(v[1]) * pp22;
        float2 n2 = make_float2((float)t2.x, (float)t2.y);
        tc[(size_t)row + (size_t)nblkt * (2 * (kl - 1))] = n1;
        tc[(size_t)row + (size_t)nblkt * (2 * (kl - 1) + 1)] = n2;
    }
}

// trace(p,k,n) = sum_kt tc(p, n(n+1)+kt, k, n(n+1)+kt) in double (the coherent part)
__global__ void ro_trace_kernel(int nodr, const float2* tc, zd* trace)
{
    const int nblkt = 2 * nodr * (nodr + 2);
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 4 * nodr) return;
    int n = e / 4 + 1, k = (e / 2) % 2 + 1, p = e % 2 + 1;
    int nn1 = n * (n + 1);
    zd s = mk(0.0, 0.0);
    for (int kt = -n; kt <= n; kt++) {
        int mn = nn1 + kt;
        s = s + up2(tc[(size_t)(2 * (mn - 1) + p - 1) + (size_t)nblkt * (2 * (mn - 1) + k - 1)]);
    }
    trace[e] = s;
}

// the big loop of ranorientscatmatrix, one CTA per (w, v)
__global__ void __launch_bounds__(RO_NT) ro_dm_kernel(RoArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const int nodr = a.nodr, nodr2 = 2 * nodr, nodrw = nodr2, nblk = nodr * (nodr + 2), nblkt = 2 * nblk;
    const int tid = threadIdx.x;
    const VCTab vt{a.bcof, a.fnr, a.nbc};
    zd* bm = reinterpret_cast<zd*>(smraw);                 // bm(k,mn,p): 2 x nblk x 2
    zd* bmcf = bm + 4 * nblk;
    zd* am = bmcf + 4 * nblk;                              // am(k,l,p): 2 x (nodr+1) x 2
    zd* amcf = am + 4 * (nodr + 1);
    double* vct = reinterpret_cast<double*>(amcf + 4 * (nodr + 1));   // (2 nodr + 1) rows of vcfunc(v,w,-t,n)
    const int VL = 3 * nodr + 2;
    double* vthr = a.vscr + ((size_t)blockIdx.x * RO_NT + tid) * VL;  // per-thread vcfunc(-u,w,m,n)
    const int nitems = (nodr2 + 1) * (nodr2 + 1);
#define TCG(p, mn, q, kl) up2(a.tc[(size_t)(2 * ((mn) - 1) + (p) - 1) + (size_t)nblkt * (2 * ((kl) - 1) + (q) - 1)])
#define BMX(arr, k, mn, p) arr[((k) - 1) + 2 * (((mn) - 1) + nblk * ((p) - 1))]
#define AMX(arr, k, l, p) arr[((k) - 1) + 2 * (((l) - 1) + (nodr + 1) * ((p) - 1))]
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        int ww = (int)sqrtf((float)item);
        while (ww * ww > item) ww--;
        while ((ww + 1) * (ww + 1) <= item) ww++;
        const int W = ww, v = item - W * W - W;   // items ordered (w, v = -w..w)
        for (int e = tid; e < 8 * nblk; e += RO_NT) bm[e] = mk(0.0, 0.0);
        __syncthreads();
        for (int n = 1; n <= nodr; n++) {
            const int nn1 = n * (n + 1), lmax = min(nodr, W + n);
            for (int e = tid; e < 8 * (nodr + 1); e += RO_NT) am[e] = mk(0.0, 0.0);
            // vcfunc(v, w, -t, n) for t = -n..n
            for (int t = -n + tid; t <= n; t += RO_NT) vc_func(vt, v, W, -t, n, vct + (size_t)(t + n) * VL);
            __syncthreads();
            // am(k,l,p) = sum_t vc(l) tc(p, n(n+1)+t, k, l(l+1)+t-v)
            for (int e = tid; e < 4 * lmax; e += RO_NT) {
                int l = e / 4 + 1, k = (e / 2) % 2 + 1, p = e % 2 + 1;
                zd s = mk(0.0, 0.0), sc = mk(0.0, 0.0);
                for (int t = -n; t <= n; t++) {
                    if (l < max(max(1, abs(v - t)), abs(n - W))) continue;
                    double vcl = vct[(size_t)(t + n) * VL + l];
                    s = s + vcl * TCG(p, nn1 + t, k, l * (l + 1) + t - v);
                    if (l == n && v == 0) {
                        zd tv = vcl * a.trace[4 * (n - 1) + 2 * (k - 1) + (p - 1)];
                        sc = sc + mk(tv.x / (double)(n + n + 1), tv.y / (double)(n + n + 1));
                    }
                }
                AMX(am, k, l, p) = s;
                AMX(amcf, k, l, p) = sc;
            }
            __syncthreads();
            // bm(k, n(n+1)+m, p) += sum_l am(k,l,p) fl(l), fl = -(-1)^l vcfunc(-u,w,m,n)(l)/(2l+1)
            for (int e = tid; e < 2 * (2 * n + 1); e += RO_NT) {
                int m = e / 2 - n, k = e % 2 + 1;
                int u = m - (-3 + 2 * k);
                if (abs(u) > W) continue;
                vc_func(vt, -u, W, m, n, vthr);
                int mn = nn1 + m;
                for (int l = max(1, abs(W - n)); l <= lmax; l++) {
                    double fl = -pm1(l) * vthr[l] / (double)(l + l + 1);
                    for (int p = 1; p <= 2; p++) {
                        BMX(bm, k, mn, p) = BMX(bm, k, mn, p) + AMX(am, k, l, p) * fl;
                        if (v == 0) BMX(bmcf, k, mn, p) = BMX(bmcf, k, mn, p) + AMX(amcf, k, l, p) * fl;
                    }
                }
            }
            __syncthreads();
        }
        // dm(u,ku,n,p,n1,p1) += bm(ik,nu,p) i^(n-n1) fl conj(bm(ik1,nu1,p1))
        const int umax = min(W, nodr + 1), nu_ = 2 * umax + 1;
        const int tot = nu_ * 3 * nodr * nodr;
        for (int e = tid; e < tot; e += RO_NT) {
            int u = e % nu_ - umax;
            int r = e / nu_;
            int ku = r % 3 + 1;
            r /= 3;
            int n = r % nodr + 1, n1 = r / nodr + 1;
            int k = (ku == 1) ? -1 : 1, k1 = (ku == 2) ? 1 : -1;
            int m = u + k, m1 = u + k1;
            if (n < max(1, abs(m)) || n1 < max(max(1, abs(m1)), n - nodrw) || n1 > min(nodr, n + nodrw)) continue;
            int ik = (k + 1) / 2 + 1, ik1 = (k1 + 1) / 2 + 1;
            int nu = n * (n + 1) + m, nu1 = n1 * (n1 + 1) + m1;
            zd cin = ipw(n - n1);
            double fl = -a.fnr[n + n + 1] * a.fnr[n1 + n1 + 1] * (double)(W + W + 1);
            for (int p = 1; p <= 2; p++)
                for (int p1 = 1; p1 <= 2; p1++) {
                    size_t ix = (size_t)(u + nodr + 1) + (size_t)(2 * nodr + 3) * ((ku - 1) + 3 * ((n - 1) + nodr * ((p - 1) + 2 * ((n1 - 1) + nodr * (p1 - 1)))));
                    atomic_addz(&a.dm[ix], BMX(bm, ik, nu, p) * cin * fl * cj(BMX(bm, ik1, nu1, p1)));
                    if (v == 0) atomic_addz(&a.dmcf[ix], BMX(bmcf, ik, nu, p) * cin * fl * cj(BMX(bmcf, ik1, nu1, p1)));
                }
        }
        __syncthreads();
    }
#undef TCG
#undef BMX
#undef AMX
}

// expansion coefficients of degree w (one CTA per w)
__global__ void __launch_bounds__(RO_NT) ro_coef_kernel(RoArgs a)
{
    const int nodr = a.nodr, w = blockIdx.x, tid = threadIdx.x;
    const VCTab vt{a.bcof, a.fnr, a.nbc};
    const int VL = 3 * nodr + 2;
    double* vthr = a.vscr + ((size_t)blockIdx.x * RO_NT + tid) * VL;
    zd* fm = a.fm + (size_t)w * 2 * (3 * nodr * 2 * nodr * 2);
    zd* fmcf = fm + 3 * nodr * 2 * nodr * 2;
#define FMX(arr, k, n, p, n1, p1) arr[((k) - 1) + 3 * (((n) - 1) + nodr * (((p) - 1) + 2 * (((n1) - 1) + nodr * ((p1) - 1))))]
#define DMX(arr, u, ku, n, p, n1, p1) arr[(size_t)((u) + nodr + 1) + (size_t)(2 * nodr + 3) * ((ku) - 1 + 3 * (((n) - 1) + nodr * (((p) - 1) + 2 * (((n1) - 1) + nodr * ((p1) - 1)))))]
    // fm(ik,n,p,n1,p1): one thread per (ik, n, n1), all u, p, p1
    for (int e = tid; e < 3 * nodr * nodr; e += RO_NT) {
        int ik = e % 3 + 1, n = (e / 3) % nodr + 1, n1 = e / (3 * nodr) + 1;
        zd f[4], fc[4];
        for (int j = 0; j < 4; j++) { f[j] = mk(0.0, 0.0); fc[j] = mk(0.0, 0.0); }
        if (!(n + n1 < w || abs(n - n1) > w)) {
            for (int u = -nodr - 1; u <= nodr + 1; u++) {
                int m, mlim;
                if (ik < 3) {
                    int k = (ik == 1) ? -1 : 1;
                    m = u + k;
                    mlim = max(1, abs(m));
                    if (n < mlim || n1 < mlim) continue;
                    vc_func(vt, m, n, 0, w, vthr);
                } else {
                    if (w < 2) break;
                    m = u + 1;
                    int m1 = u - 1;
                    if (n < max(1, abs(m)) || n1 < max(1, abs(m1))) continue;
                    vc_func(vt, m, n, -2, w, vthr);
                }
                double fl = -pm1(n) * vthr[n1] * a.fnr[w + w + 1] / a.fnr[n1 + n1 + 1];
                for (int p = 1; p <= 2; p++)
                    for (int p1 = 1; p1 <= 2; p1++) {
                        f[(p - 1) + 2 * (p1 - 1)] = f[(p - 1) + 2 * (p1 - 1)] + DMX(a.dm, u, ik, n, p, n1, p1) * fl;
                        fc[(p - 1) + 2 * (p1 - 1)] = fc[(p - 1) + 2 * (p1 - 1)] + DMX(a.dmcf, u, ik, n, p, n1, p1) * fl;
                    }
            }
        }
        for (int p = 1; p <= 2; p++)
            for (int p1 = 1; p1 <= 2; p1++) {
                FMX(fm, ik, n, p, n1, p1) = f[(p - 1) + 2 * (p1 - 1)];
                FMX(fmcf, ik, n, p, n1, p1) = fc[(p - 1) + 2 * (p1 - 1)];
            }
    }
    __syncthreads();
    if (tid != 0) return;
    // aw(0:2,-1:1), bw, cw, dw for this w, in the reference's order
    zd aw[2][3][3], bw[2][3][3], cw[2], dw[2];
    for (int c = 0; c < 2; c++) {
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < 3; k++) { aw[c][i][k] = mk(0.0, 0.0); bw[c][i][k] = mk(0.0, 0.0); }
        cw[c] = mk(0.0, 0.0);
        dw[c] = mk(0.0, 0.0);
    }
    for (int n = 1; n <= nodr; n++) {
        int n1s = max(1, abs(n - w)), n1e = min(nodr, n + w);
        double in = pm1(n);
        vc_func(vt, 1, n, 0, w, vthr);
        for (int n1 = n1s; n1 <= n1e; n1++) {
            double fl = 2.0 * in * vthr[n1] * a.fnr[w + w + 1] / a.fnr[n1 + n1 + 1];
            int i = (n + n1 - w) % 2 + 1;
            for (int p = 1; p <= 2; p++) {
                int p1 = (2 - i) * p + (i - 1) * (3 - p);
                for (int c = 0; c < 2; c++) {
                    zd* F = c ? fmcf : fm;
                    for (int k = -1; k <= 1; k += 2) {
                        int ik = (k + 1) / 2 + 1;
                        aw[c][0][k + 1] = aw[c][0][k + 1] + FMX(F, ik, n, p, n1, p1) * fl;
                        bw[c][0][k + 1] = bw[c][0][k + 1] + FMX(F, ik, n, p, n1, 3 - p1) * fl;
                    }
                    bw[c][2][1] = bw[c][2][1] + FMX(F, 3, n, p, n1, 3 - p1) * fl;
                    aw[c][2][1] = aw[c][2][1] + FMX(F, 3, n, p, n1, p1) * fl;
                }
            }
        }
        if (w < 2) continue;
        vc_func(vt, 1, n, -2, w, vthr);
        for (int n1 = n1s; n1 <= n1e; n1++) {
            double fl = 2.0 * in * vthr[n1] * a.fnr[w + w + 1] / a.fnr[n1 + n1 + 1];
            int i = (n + n1 - w) % 2 + 1;
            for (int p = 1; p <= 2; p++) {
                int p1 = (2 - i) * p + (i - 1) * (3 - p);
                for (int c = 0; c < 2; c++) {
                    zd* F = c ? fmcf : fm;
                    for (int k = -1; k <= 1; k += 2) {
                        int ik = (k + 1) / 2 + 1;
                        aw[c][2][k + 1] = aw[c][2][k + 1] + FMX(F, ik, n, p, n1, p1) * (fl * pm1(p1));
                        bw[c][2][k + 1] = bw[c][2][k + 1] + FMX(F, ik, n, p, n1, 3 - p1) * (fl * pm1(3 - p1));
                    }
                }
            }
            double fl2 = 2.0 * pm1(n1 + w) * vthr[n1] * a.fnr[w + w + 1] / a.fnr[n1 + n1 + 1];
            for (int p = 1; p <= 2; p++)
                for (int p1 = 1; p1 <= 2; p1++)
                    for (int c = 0; c < 2; c++) {
                        zd* F = c ? fmcf : fm;
                        cw[c] = cw[c] + FMX(F, 3, n, p, n1, p1) * (fl * pm1(p1));
                        dw[c] = dw[c] + FMX(F, 3, n, p, n1, p1) * (fl2 * pm1(p));
                    }
        }
    }
    for (int c = 0; c < 2; c++) {
        double* o = (c ? a.smcf : a.sm) + 16 * w;
#define SMO(i, j) o[((i) - 1) + 4 * ((j) - 1)]
#define AWX(i, k) aw[c][i][(k) + 1]
#define BWX(i, k) bw[c][i][(k) + 1]
        for (int e = 0; e < 16; e++) o[e] = 0.0;
        SMO(1, 1) = (AWX(0, -1) + AWX(0, 1)).x;
        SMO(1, 2) = (AWX(2, -1) + AWX(2, 1)).x;
        SMO(1, 3) = 2.0 * AWX(2, 0).y;
        SMO(1, 4) = (AWX(0, 1) - AWX(0, -1)).x;
        SMO(2, 2) = dw[c].x;
        SMO(2, 3) = dw[c].y;
        SMO(2, 4) = (AWX(2, 1) - AWX(2, -1)).x;
        SMO(3, 1) = -(BWX(2, -1) + BWX(2, 1)).y;
        SMO(3, 2) = cw[c].y;
        SMO(3, 3) = cw[c].x;
        SMO(3, 4) = (BWX(2, -1) - BWX(2, 1)).y;
        SMO(4, 1) = (BWX(0, -1) + BWX(0, 1)).x;
        SMO(4, 2) = 2.0 * BWX(2, 0).x;
        SMO(4, 4) = (BWX(0, 1) - BWX(0, -1)).x;
        for (int e = 0; e < 16; e++) o[e] = o[e] / a.rimed_re / 2.0;
#undef SMO
#undef AWX
#undef BWX
    }
#undef FMX
#undef DMX
}

// ranorienscatmatrixcalc at theta_i = i pi/(nang-1) (pi as the reference stores it)
__global__ void ro_calc_kernel(int nodrexp, int nang, const double* smc, const double* fnr, const double* bcofd, double* dscr, double* smat)
{
    const int ia = blockIdx.x;
    if (ia >= nang) return;
    const int nmax = nodrexp, kmax = 2, W = 2 * nmax + 1;
    const double ct = cos((double)ia * MSTMG_REF_PI / (double)(nang - 1));
    double* dk0 = dscr + (size_t)ia * (16 * nmax + 40) + (nmax + 1);
    double* dk01 = dk0 + (2 * nmax + 3);
    double* dc = dk01 + (2 * nmax + 3);   // rows m = -2..2 of the current degree, columns k = -nmax..nmax
#define DCR(m, k) dc[((m) + 2) * W + ((k) + nmax)]
#define SC(i, j, n) smc[((i) - 1) + 4 * ((j) - 1) + 16 * (n)]
    __shared__ double so[16];
#define SO(i, j) so[((i) - 1) + 4 * ((j) - 1)]
    if (threadIdx.x < 16) so[threadIdx.x] = 0.0;
    const double sbe = (fabs(ct) >= 1.0) ? 0.0 : sqrt(fabs((1.0 + ct) * (1.0 - ct)));
    const double cbe2 = 0.5 * (1.0 + ct), sbe2 = 0.5 * (1.0 - ct);
    for (int k = threadIdx.x; k < 2 * nmax + 3; k += blockDim.x) { dk0[k - (nmax + 1)] = 0.0; dk01[k - (nmax + 1)] = 0.0; }
    __syncthreads();
    if (threadIdx.x == 0) {
        dk0[0] = 1.0;
        // degree 0: dc(0,0) = 1
        SO(1, 1) = SO(1, 1) + SC(1, 1, 0);
        SO(1, 4) = SO(1, 4) + SC(1, 4, 0);
        SO(4, 1) = SO(4, 1) + SC(4, 1, 0);
        SO(4, 4) = SO(4, 4) + SC(4, 4, 0);
    }
    __syncthreads();
    int sgn = 1;
    double sben = 1.0;
    for (int n = 1; n <= nmax; n++) {
        int kk = min(n, kmax);
        sgn = -sgn;
        sben = sben * sbe / 2.0;
        if (sben < 1.0e-30) sben = 0.0;
        double newv[8];
        int cnt = 0;
        for (int k = -n + 1 + (int)threadIdx.x; k <= n - 1; k += blockDim.x)
            newv[cnt++] = (ct * (double)(n + n - 1) * dk0[k] - fnr[n - k - 1] * fnr[n + k - 1] * dk01[k]) / (fnr[n + k] * fnr[n - k]);
        __syncthreads();
        cnt = 0;
        for (int k = -n + 1 + (int)threadIdx.x; k <= n - 1; k += blockDim.x) {
            dk01[k] = dk0[k];
            dk0[k] = newv[cnt++];
        }
        if (threadIdx.x == 0) {
            dk0[n] = sgn * sben * bcofd[n];
            dk0[-n] = sgn * dk0[n];
            dk01[n] = 0.0;
            dk01[-n] = 0.0;
        }
        __syncthreads();
        for (int k = -n + (int)threadIdx.x; k <= n; k += blockDim.x) DCR(0, k) = dk0[k];
        __syncthreads();
        int im = 1;
        for (int m = 1; m <= kk; m++) {
            im = -im;
            double fmn = 1.0 / fnr[n - m + 1] / fnr[n + m];
            for (int k = -n + (int)threadIdx.x; k <= n; k += blockDim.x) {
                double dkm1 = (k == -n) ? 0.0 : DCR(m - 1, k - 1);
                double dkn1 = (k == n) ? 0.0 : DCR(m - 1, k + 1);
                double v = (fnr[n + k] * fnr[n - k + 1] * cbe2 * dkm1 - fnr[n - k] * fnr[n + k + 1] * sbe2 * dkn1 -
                            (double)k * sbe * DCR(m - 1, k)) * fmn;
                DCR(m, k) = v;
                DCR(-m, -k) = v * pm1(k) * im;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            // dc(k, n(n+1)+m) of rotcoef(ct, 2, nodrexp) is DCR(k, m) here
            double d00 = DCR(0, 0);
            SO(1, 1) = SO(1, 1) + d00 * SC(1, 1, n);
            SO(1, 4) = SO(1, 4) + d00 * SC(1, 4, n);
            SO(4, 1) = SO(4, 1) + d00 * SC(4, 1, n);
            SO(4, 4) = SO(4, 4) + d00 * SC(4, 4, n);
            if (n >= 2) {
                double d20 = DCR(2, 0), d2m = DCR(2, -2), d2p = DCR(2, 2);
                SO(1, 2) = SO(1, 2) + d20 * SC(1, 2, n);
                SO(2, 4) = SO(2, 4) + d20 * SC(2, 4, n);
                SO(3, 4) = SO(3, 4) + d20 * SC(3, 4, n);
                SO(1, 3) = SO(1, 3) + d20 * SC(1, 3, n);
                SO(3, 1) = SO(1, 3) + d20 * SC(3, 1, n);   // as the reference writes it
                SO(4, 2) = SO(4, 2) + d20 * SC(4, 2, n);
                SO(2, 2) = SO(2, 2) + d2m * SC(2, 2, n) + d2p * SC(3, 3, n);
                SO(2, 3) = SO(2, 3) + d2p * SC(2, 3, n) + d2p * SC(3, 2, n);
                SO(3, 3) = SO(3, 3) - d2m * SC(2, 2, n) + d2p * SC(3, 3, n);
                SO(3, 2) = SO(3, 2) + d2p * SC(2, 3, n) - d2p * SC(3, 2, n);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        SO(2, 1) = SO(1, 2);
        SO(4, 3) = -SO(3, 4);
        for (int e = 0; e < 16; e++) smat[16 * (size_t)ia + e] = so[e];
    }
#undef DCR
#undef SC
#undef SO
}

size_t ro_dm_smem(int nodr)
{
    int nblk = nodr * (nodr + 2);
    return sizeof(zd) * (8 * (size_t)nblk + 8 * (size_t)(nodr + 1)) + sizeof(double) * (size_t)(2 * nodr + 1) * (3 * nodr + 2);
}
int ro_dm_grid(int nodr, int nsm) { return std::min((2 * nodr + 1) * (2 * nodr + 1), nsm * 2); }
size_t ro_vscr_doubles(int nodr, int nsm)
{
    size_t g = (size_t)std::max(ro_dm_grid(nodr, nsm), 2 * nodr + 1);
    return g * RO_NT * (size_t)(3 * nodr + 2);
}
size_t ro_dm_elems(int nodr) { return (size_t)(2 * nodr + 3) * 3 * nodr * 2 * nodr * 2; }

int launch_ranorient(const RoArgs& a, const zd* tmat, int nang, const double* bcofd, double* dscr, double* smat, int nsm, cudaStream_t st)
{
    const int nodr = a.nodr;
    size_t nblk = (size_t)nodr * (nodr + 2);
    int g = (int)std::min<size_t>((2 * nblk * nblk + 255) / 256, (size_t)nsm * 16);
    ro_prep_kernel<<<g, 256, 0, st>>>(nodr, tmat, a.tc);
    ro_trace_kernel<<<(4 * nodr + 63) / 64, 64, 0, st>>>(nodr, a.tc, a.trace);
    size_t smem = ro_dm_smem(nodr);
    if (smem > 227 * 1024) return -1;
    cudaFuncSetAttribute(ro_dm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ro_dm_kernel<<<ro_dm_grid(nodr, nsm), RO_NT, smem, st>>>(a);
    ro_coef_kernel<<<2 * nodr + 1, RO_NT, 0, st>>>(a);
    if (nang > 1) ro_calc_kernel<<<nang, 64, 0, st>>>(2 * nodr, nang, a.sm, a.fnr, bcofd, dscr, smat);
    launch_counter() += (nang > 1) ? 5 : 4;
    return 0;
}
