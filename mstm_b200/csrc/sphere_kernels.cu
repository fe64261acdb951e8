// sphere_kernels.cu -- per-sphere device kernels: Mie coefficients, incident
// plane-wave coefficients, the Mie multiply, and the efficiency sums.  All
// coefficient generation and the final cross-section sums run in FP64.
#include "common.cuh"
#include "special.cuh"
#include "kernels.cuh"
#include "sphere_kernels.cuh"

#define MIE_NMAX 48   // largest Mie order a sphere may need (x up to ~30)

// ---------------------------------------------------------------------------
// mieoa for a non-optically-active sphere in a medium (december2023/
// mstm-modules-33.f90:5438-5578).  mode 0: determine the order from qeps
// (qeps>0 convergence test; qeps<0 forces ceiling(-qeps)); mode 1: write the
// 2x2 LR-basis matrices anp(2,2,n) and their inverses for the given order.
// ---------------------------------------------------------------------------
// With dnp (mode 1) also the coefficients of a host sphere: D, U, V of
// (a, f) = [[A, U], [D, V]] (g, b), b the exciting field inside the sphere and
// f the regular field there (mieoa's dnp_mie, unp_mie, vnp_mie,
// modules:5495-5528).
__device__ void mie_one(double x, zd ri, zd rimed, double qeps, int mode, int* nodr_io, zd* anp, zd* anpinv,
                        double* qext_o, double* qabs_o, zd* dnp = nullptr, zd* unp = nullptr, zd* vnp = nullptr)
{
    int nstop;
    if (mode == 0) {
        if (qeps > 0.0) nstop = (int)llround(x + 4.0 * pow(x, (double)(1.0f / 3.0f))) + 5;
        else if (qeps < 0.0) nstop = (int)ceil(-qeps);
        else nstop = *nodr_io;
    } else {
        nstop = *nodr_io;
    }
    if (nstop > MIE_NMAX - 2) nstop = MIE_NMAX - 2;
    const int nb = nstop + 1;
    zd psi[2][MIE_NMAX], xi[2][MIE_NMAX], scr[2 * MIE_NMAX];
    // both helicities share one index: rii(:,i) equal; i=0 medium, i=1 sphere
    zd rii[2] = {rimed, ri};
    zd ribulk[2] = {cdivr(2.0, cdivr(1.0, rii[0]) + cdivr(1.0, rii[0])), cdivr(2.0, cdivr(1.0, rii[1]) + cdivr(1.0, rii[1]))};
    zd xri[2] = {x * rii[0], x * rii[1]};
    for (int i = 0; i < 2; i++) {
        mstm_cricbessel(nb, xri[i], psi[i], scr);
        mstm_crichankel(nb, xri[i], xi[i], scr);
    }
    double qsca = 0.0, qext = 0.0;
    double qext1[MIE_NMAX];
    for (int n = 1; n <= nstop; n++) {
        zd psip[2], xip[2], psipn[2];
        for (int i = 0; i < 2; i++) {
            psip[i] = psi[i][n - 1] - cdiv((double)n * psi[i][n], xri[i]);
            xip[i] = xi[i][n - 1] - cdiv((double)n * xi[i][n], xri[i]);
            psipn[i] = cdiv(psi[i][n - 1], psi[i][n]) - cdivr((double)n, xri[i]);
        }
        zd gmat[4], amat[4];
        for (int s = 1; s <= 2; s++) {
            double ss = pm1(s);
            for (int t = 1; t <= 2; t++) {
                double st = pm1(t);
                zd pre = cdiv(ss * ribulk[0] + st * ribulk[1], rii[1] * rii[0]);
                gmat[(s - 1) + 2 * (t - 1)] = pre * (psipn[1] * xi[0][n] - (ss * st) * xip[0]);
                amat[(s - 1) + 2 * (t - 1)] = pre * (psipn[1] * psi[0][n] - (ss * st) * psip[0]);
            }
        }
        zd ginv[4], am[4];
        mstm_inv22(gmat, ginv);
        for (int r = 1; r <= 2; r++)
            for (int c = 1; c <= 2; c++)
                am[(r - 1) + 2 * (c - 1)] = -(ginv[(r - 1)] * amat[2 * (c - 1)] + ginv[(r - 1) + 2] * amat[1 + 2 * (c - 1)]);
        if (mode == 1) {
            for (int k = 0; k < 4; k++) anp[4 * (n - 1) + k] = am[k];
            mstm_inv22(am, anpinv + 4 * (n - 1));
        }
        if (mode == 1 && dnp) {
            const zd xipn0 = cdiv(xi[0][n - 1], xi[0][n]) - cdivr((double)n, xri[0]);
            zd bm[4], um[4], dm[4], vm[4];
            for (int s = 1; s <= 2; s++) {
                double ss = pm1(s);
                for (int t = 1; t <= 2; t++) {
                    double st = pm1(t);
                    const int k = (s - 1) + 2 * (t - 1);
                    const zd pb = cdiv(ss * ribulk[1] + st * ribulk[0], rii[0] * rii[1]);
                    um[k] = cdiv((ss + st) * ribulk[1], rii[1] * rii[1]) * cdiv(mk(0.0, 1.0), psi[1][n]);
                    dm[k] = -(cdiv((ss + st) * ribulk[0], rii[0] * rii[0]) * cdiv(mk(0.0, 1.0), xi[0][n]));
                    bm[k] = pb * (xipn0 * psi[1][n] - (ss * st) * psip[1]);
                    vm[k] = pb * (xipn0 * xi[1][n] - (ss * st) * xip[1]);
                }
            }
            zd binv[4];
            mstm_inv22(bm, binv);
            for (int r = 0; r < 2; r++)
                for (int c = 0; c < 2; c++) {
                    const int k = r + 2 * c;
                    unp[4 * (n - 1) + k] = -(ginv[r] * um[2 * c] + ginv[r + 2] * um[1 + 2 * c]);
                    dnp[4 * (n - 1) + k] = -(binv[r] * dm[2 * c] + binv[r + 2] * dm[1 + 2 * c]);
                    vnp[4 * (n - 1) + k] = -(binv[r] * vm[2 * c] + binv[r + 2] * vm[1 + 2 * c]);
                }
        }
        qext1[n] = 0.0;
        double fn1 = n + n + 1;
        for (int p = 1; p <= 2; p++) {
            for (int q = 1; q <= 2; q++) {
                double ab = cabsd(am[(p - 1) + 2 * (q - 1)]);
                qsca = qsca + fn1 * ab * ab;
            }
            qext1[n] = qext1[n] - fn1 * am[(p - 1) * 3].x;
        }
        qext = qext + qext1[n];
    }
    if (mode == 0) {
        if (qeps > 0.0) {
            double qextt = qext;
            qext = 0.0;
            int n;
            for (n = 1; n <= nstop; n++) {
                qext = qext + qext1[n];
                if (fabs(1.0 - qext / qextt) < qeps || n == nstop) break;
            }
            *nodr_io = n;
        } else {
            *nodr_io = nstop;
        }
    }
    qsca = 2.0 / x / x * qsca;
    qext = 2.0 / x / x * qext;
    if (qext_o) *qext_o = qext;
    if (qabs_o) *qabs_o = qext - qsca;
}

// rext (per sphere re, im; may be null): the index around each sphere, else
// the medium's
__device__ __forceinline__ zd exterior(const double* rext, int i, double mre, double mim)
{
    return rext ? mk(rext[2 * i], rext[2 * i + 1]) : mk(mre, mim);
}

__global__ void mie_order_kernel(int n, const double* radius, const double* ri, double rimed_re, double rimed_im, const double* rext,
                                 double qeps, int* order)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int nodr = 0;
    mie_one(radius[i], mk(ri[2 * i], ri[2 * i + 1]), exterior(rext, i, rimed_re, rimed_im), qeps, 0, &nodr, nullptr, nullptr, nullptr,
            nullptr);
    order[i] = nodr;
}

// hoff (may be null): spheres with hoff[i] >= 0 hold others and also get D, U, V
__global__ void mie_coef_kernel(int n, const double* radius, const double* ri, double rimed_re, double rimed_im, const double* rext,
                                const int* order, const int* mie_offset, const int* hoff, zd* an, zd* an_inv, float* an32, zd* dn,
                                zd* un, zd* vn, double* qext, double* qabs)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int nodr = order[i];
    const int mo = mie_offset[i];
    const bool h = hoff && hoff[i] >= 0;
    mie_one(radius[i], mk(ri[2 * i], ri[2 * i + 1]), exterior(rext, i, rimed_re, rimed_im), 0.0, 1, &nodr, an + mo, an_inv + mo, &qext[i],
            &qabs[i], h ? dn + mo : nullptr, h ? un + mo : nullptr, h ? vn + mo : nullptr);
    for (int k = 0; k < 4 * order[i]; k++) {
        an32[2 * (mo + k)] = (float)an[mo + k].x;
        an32[2 * (mo + k) + 1] = (float)an[mo + k].y;
    }
}

void launch_mie_orders(int n, const double* radius, const double* ri, double mre, double mim, const double* rext, double qeps, int* order,
                       cudaStream_t st)
{
    mie_order_kernel<<<(n + 63) / 64, 64, 0, st>>>(n, radius, ri, mre, mim, rext, qeps, order);
    launch_counter() += 1;
}
void launch_mie_coefs(int n, const double* radius, const double* ri, double mre, double mim, const double* rext, const int* order,
                      const int* mie_offset, const int* hoff, zd* an, zd* an_inv, float* an32, zd* dn, zd* un, zd* vn, double* qext,
                      double* qabs, cudaStream_t st)
{
    mie_coef_kernel<<<(n + 63) / 64, 64, 0, st>>>(n, radius, ri, mre, mim, rext, order, mie_offset, hoff, an, an_inv, an32, dn, un, vn,
                                                  qext, qabs);
    launch_counter() += 1;
}

// ---------------------------------------------------------------------------
// Plane-wave coefficients: genplanewavecoef (modules:1453-1520) for order
// lmax into pw0(nb(lmax), 2 polarisations), then per sphere the phase of
// layerplanewavecoef without plane boundaries (modules:3901-3965).
// ---------------------------------------------------------------------------
__global__ void planewave_common_kernel(double alpha, zd cb, int nodr, zd* pw0, zd* drot /* 3*(nodr(nodr+2)+1) */)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    // crotcoef(cb, kmax=1, nodr) (modules:1187-1246)
    const int kmax = 1, ld = 3;
    int nd = nodr * (nodr + 2) + 1;
    for (int k = 0; k < ld * nd; k++) drot[k] = mk(0.0, 0.0);
#define DC(m, nk) drot[((m) + kmax) + ld * (nk)]
    zd sbe = csqrtd((mk(1.0, 0.0) + cb) * (mk(1.0, 0.0) - cb));
    zd cbe2 = 0.5 * (mk(1.0, 0.0) + cb), sbe2 = 0.5 * (mk(1.0, 0.0) - cb);
    zd dk0s[2 * MSTMG_LMAX + 3], dk01s[2 * MSTMG_LMAX + 3];
    zd* dk0 = dk0s + (MSTMG_LMAX + 1);
    zd* dk01 = dk01s + (MSTMG_LMAX + 1);
    for (int k = 0; k < 2 * MSTMG_LMAX + 3; k++) { dk0s[k] = mk(0.0, 0.0); dk01s[k] = mk(0.0, 0.0); }
    int in = 1;
    dk0[0] = mk(1.0, 0.0);
    zd sben = mk(1.0, 0.0);
    DC(0, 0) = mk(1.0, 0.0);
    // bcof(n,n) = sqrt((2n)!/(n!)^2), built by the same recurrence as numconstants::init
    double bnn = 1.0;
    for (int n = 1; n <= nodr; n++) {
        bnn = sqrt((double)(n + n)) * sqrt((double)(n + n - 1)) * bnn / sqrt((double)n) / sqrt((double)n);
        int knmax = n < kmax ? n : kmax;
        int nn1 = n * (n + 1);
        in = -in;
        {
            zd tq = sben * sbe;   // sben = sben*sbe/2
            sben = mk(tq.x / 2.0, tq.y / 2.0);
        }
        dk0[n] = ((double)in * sben) * bnn;
        dk0[-n] = (double)in * dk0[n];
        dk01[n] = mk(0.0, 0.0);
        dk01[-n] = mk(0.0, 0.0);
        DC(0, nn1 + n) = dk0[n];
        DC(0, nn1 - n) = dk0[-n];
        for (int k = -n + 1; k <= n - 1; k++) {
            int kn = nn1 + k;
            zd dkt = dk01[k];
            dk01[k] = dk0[k];
            double c1 = (double)(n + n - 1), c2 = sqrt((double)(n - k - 1)) * sqrt((double)(n + k - 1));
            double c3 = sqrt((double)(n + k)) * sqrt((double)(n - k));
            zd num = (cb * c1) * dk01[k] - c2 * dkt;
            dk0[k] = mk(num.x / c3, num.y / c3);
            DC(0, kn) = dk0[k];
        }
        int im = 1;
        for (int m = 1; m <= knmax; m++) {
            im = -im;
            double fmn = 1.0 / sqrt((double)(n - m + 1)) / sqrt((double)(n + m));
            int m1 = m - 1;
            zd dkm0 = mk(0.0, 0.0);
            for (int k = -n; k <= n; k++) {
                int kn = nn1 + k;
                zd dkm1 = dkm0;
                dkm0 = DC(m1, kn);
                zd dkn1 = (k == n) ? mk(0.0, 0.0) : DC(m1, kn + 1);
                zd v = (sqrt((double)(n + k)) * sqrt((double)(n - k + 1))) * cbe2 * dkm1 -
                       (sqrt((double)(n - k)) * sqrt((double)(n + k + 1))) * sbe2 * dkn1 - ((double)k * sbe) * DC(m1, kn);
                DC(m, kn) = v * fmn;
                DC(-m, nn1 - k) = DC(m, kn) * (pm1(k) * im);
            }
        }
    }
    int nb = 2 * nodr * (nodr + 2);
    // tau(0:nodr+1,nodr,2) then the LR combination
    for (int n = 1; n <= nodr; n++) {
        int nn1 = n * (n + 1);
        double fnm = sqrt((double)(n + n + 1) / 2.0) / 4.0;
        zd cin;
        {
            int e = (n + 1) % 4;
            zd ipw = (e == 0) ? mk(1.0, 0.0) : (e == 1 ? mk(0.0, 1.0) : (e == 2 ? mk(-1.0, 0.0) : mk(0.0, -1.0)));
            cin = 4.0 * ipw;
        }
        for (int m = -n; m <= n; m++) {
            int mn = nn1 + m;
            zd tau1 = -fnm * (-DC(-1, mn) + DC(1, mn));
            zd tau2 = -fnm * (DC(-1, mn) + DC(1, mn));
            zd taulr[2] = {(tau1 + tau2) * 0.5, (tau1 - tau2) * 0.5};
            // ealpham(-m): powers of e^{i alpha} as ephicoef builds them
            zd ea;
            zd ep = mk(cos(alpha), sin(alpha));
            zd pw = mk(1.0, 0.0);
            for (int q = 1; q <= (m < 0 ? -m : m); q++) pw = ep * pw;
            ea = (m <= 0) ? pw : cj(pw);
            for (int p = 1; p <= 2; p++) {
                double sp = -pm1(p);
                int ai = aidx(m, n, p - 1, nodr);
                pw0[ai] = -(cin * taulr[p - 1] * ea);
                pw0[nb + ai] = sp * imul(cin * taulr[p - 1] * ea);
            }
        }
    }
#undef DC
}

// outside (may be null): 1 for the spheres outside every other; the others,
// and the blocks of the fields inside host spheres (sphere indices >= nreal),
// get no incident wave (sphereplanewavecoef, scatprops:268)
__global__ void planewave_phase_kernel(int nslots2, const int* slot_sphere, const int* order, const int* offset, const double* pos,
                                       int lmax, const zd* pw0, zd cbinc, zd riinc, double sinc, double alpha, zd* pmnp, int ld,
                                       int nreal, const int* outside)
{
    // nslots2 = neqns: every coefficient of every sphere block (both modes)
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nslots2) return;
    int half = e;  // index in the full vector
    // locate sphere via slot_sphere over the first-mode half of each block
    int i = slot_sphere[e];
    if (outside && (i >= nreal || !outside[i])) {
        for (int k = 0; k < 2; k++) pmnp[(size_t)k * ld + e] = mk(0.0, 0.0);
        return;
    }
    int L = order[i], off = offset[i];
    int loc = half - off;
    int hb = L * (L + 2);
    int p = loc / hb, rem = loc % hb;
    int row = rem % (L + 2), col = rem / (L + 2) + 1;
    int m, n;
    if (row <= col) { m = row; n = col; } else { n = row - 1; m = -col; }
    zd phz = cexpd(imul(riinc * cbinc * mk(pos[3 * i + 2] - 0.0, 0.0)));
    zd phl = cexpd(imul(mk(sinc * (cos(alpha) * pos[3 * i] + sin(alpha) * pos[3 * i + 1]), 0.0)));
    int nbl = 2 * lmax * (lmax + 2);
    int src = aidx(m, n, p, lmax);
    for (int k = 0; k < 2; k++) pmnp[(size_t)k * ld + e] = (pw0[(size_t)k * nbl + src] * phz) * phl;
}

void launch_planewave(double alpha, double sinc, int dir, int lmax, int neqns, const int* slot_full, const int* order,
                      const int* offset, const double* pos, zd* pw0, zd* drot, zd* pmnp, cudaStream_t st, int nreal, const int* outside)
{
    zd riinc = mk(1.0, 0.0);
    zd a = cdiv(mk(sinc, 0.0), riinc);
    zd cbinc = csqrtd((mk(1.0, 0.0) - a) * (mk(1.0, 0.0) + a)) * (double)(3 - 2 * dir);
    planewave_common_kernel<<<1, 32, 0, st>>>(alpha, cbinc, lmax, pw0, drot);
    planewave_phase_kernel<<<(neqns + 255) / 256, 256, 0, st>>>(neqns, slot_full, order, offset, pos, lmax, pw0, cbinc, riinc,
                                                                 sinc, alpha, pmnp, neqns, nreal, outside);
    launch_counter() += 2;
}

// ---------------------------------------------------------------------------
// Mie multiply (multmiecoeffmult, modules:5633-5751, external spheres):
// y(m,n,p) = sum_q A(p,q,n) x(m,n,q)  (idir=1) or A(q,p,n) (idir!=1).
// One thread per (m,n) slot of the first mode half; in-place is allowed.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void mie_kernel(int nslots, const int* slot_sphere, const int* order, const int* offset, const int* mie_offset,
                           const cpx<T>* an, int idir, int conj_in, const cpx<T>* x, cpx<T>* y)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nslots) return;
    int i = slot_sphere[e];
    int L = order[i];
    int hb = L * (L + 2);
    int loc = e - offset[i] / 2;   // slot index inside the sphere's first half
    int row = loc % (L + 2), col = loc / (L + 2) + 1;
    int n = (row <= col) ? col : row - 1;
    int base = offset[i] + loc;
    cpx<T> x0 = x[base], x1 = x[base + hb];
    if (conj_in) { x0 = cj(x0); x1 = cj(x1); }
    const cpx<T>* A = an + mie_offset[i] + 4 * (n - 1);   // A(p,q) at (p-1)+2(q-1)
    cpx<T> y0, y1;
    if (idir == 1) {
        y0 = A[0] * x0 + A[2] * x1;
        y1 = A[1] * x0 + A[3] * x1;
    } else {
        y0 = A[0] * x0 + A[1] * x1;
        y1 = A[2] * x0 + A[3] * x1;
    }
    y[base] = y0;
    y[base + hb] = y1;
}

template <typename T>
void launch_mie(int nslots, const int* slot_sphere, const int* order, const int* offset, const int* mie_offset, const cpx<T>* an,
                int idir, int conj_in, const cpx<T>* x, cpx<T>* y, cudaStream_t st)
{
    mie_kernel<T><<<(nslots + 255) / 256, 256, 0, st>>>(nslots, slot_sphere, order, offset, mie_offset, an, idir, conj_in, x, y);
    launch_counter() += 1;
}
template void launch_mie<double>(int, const int*, const int*, const int*, const int*, const zd*, int, int, const zd*, zd*, cudaStream_t);
template void launch_mie<float>(int, const int*, const int*, const int*, const int*, const zf*, int, int, const zf*, zf*, cudaStream_t);

// ---------------------------------------------------------------------------
// Mie multiply with host spheres (multmiecoeffmult with its host branch,
// modules:5633-5751).  A sphere that holds others has a second block at
// hoff[i], the regular field inside it; with g its exciting field outside
// and b inside:  idir=1  a = A g + U b,  f = D g + V b;
//               idir!=1 a = A^T g + D^T b,  f = U^T g + V^T b.
// One thread per (m,n) slot of a sphere's first mode half; the slots of the
// internal blocks (slot sphere >= nreal) are done by their host's thread.
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ void m22(const cpx<T>* X, bool tr, cpx<T> v0, cpx<T> v1, cpx<T>& o0, cpx<T>& o1)
{
    if (!tr) {
        o0 = o0 + X[0] * v0 + X[2] * v1;
        o1 = o1 + X[1] * v0 + X[3] * v1;
    } else {
        o0 = o0 + X[0] * v0 + X[1] * v1;
        o1 = o1 + X[2] * v0 + X[3] * v1;
    }
}

template <typename T>
__global__ void hmie_kernel(int nslots, int nreal, const int* slot_sphere, const int* order, const int* offset, const int* mie_offset,
                            const int* hoff, const cpx<T>* an, const cpx<T>* dn, const cpx<T>* un, const cpx<T>* vn, int idir, int conj_in,
                            const cpx<T>* x, cpx<T>* y)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nslots) return;
    int i = slot_sphere[e];
    if (i >= nreal) return;
    int L = order[i];
    int hb = L * (L + 2);
    int loc = e - offset[i] / 2;
    int row = loc % (L + 2), col = loc / (L + 2) + 1;
    int n = (row <= col) ? col : row - 1;
    int base = offset[i] + loc;
    cpx<T> g0 = x[base], g1 = x[base + hb];
    if (conj_in) { g0 = cj(g0); g1 = cj(g1); }
    const int q = mie_offset[i] + 4 * (n - 1);
    const bool tr = idir != 1;
    cpx<T> a0 = mk((T)0, (T)0), a1 = mk((T)0, (T)0);
    m22<T>(an + q, tr, g0, g1, a0, a1);
    if (hoff[i] < 0) {
        y[base] = a0;
        y[base + hb] = a1;
        return;
    }
    const int bb = hoff[i] + loc;
    cpx<T> b0 = x[bb], b1 = x[bb + hb];
    if (conj_in) { b0 = cj(b0); b1 = cj(b1); }
    cpx<T> f0 = mk((T)0, (T)0), f1 = mk((T)0, (T)0);
    m22<T>((tr ? dn : un) + q, tr, b0, b1, a0, a1);
    m22<T>((tr ? un : dn) + q, tr, g0, g1, f0, f1);
    m22<T>(vn + q, tr, b0, b1, f0, f1);
    y[base] = a0;
    y[base + hb] = a1;
    y[bb] = f0;
    y[bb + hb] = f1;
}

template <typename T>
void launch_hmie(int nslots, int nreal, const int* slot_sphere, const int* order, const int* offset, const int* mie_offset, const int* hoff,
                 const cpx<T>* an, const cpx<T>* dn, const cpx<T>* un, const cpx<T>* vn, int idir, int conj_in, const cpx<T>* x, cpx<T>* y,
                 cudaStream_t st)
{
    hmie_kernel<T><<<(nslots + 255) / 256, 256, 0, st>>>(nslots, nreal, slot_sphere, order, offset, mie_offset, hoff, an, dn, un, vn, idir,
                                                         conj_in, x, y);
    launch_counter() += 1;
}
template void launch_hmie<double>(int, int, const int*, const int*, const int*, const int*, const int*, const zd*, const zd*, const zd*,
                                  const zd*, int, int, const zd*, zd*, cudaStream_t);
template void launch_hmie<float>(int, int, const int*, const int*, const int*, const int*, const int*, const zf*, const zf*, const zf*,
                                 const zf*, int, int, const zf*, zf*, cudaStream_t);

// ---------------------------------------------------------------------------
// Efficiencies: lrsphereqeff (scatprops:676-776) per sphere, npol=2, with
// g = A^{-1} a (qefficiencyfactors, scatprops:782-870, no host spheres).
// qeff(3,3,N): qeff[q + 3*(pol + 3*i)].
// ---------------------------------------------------------------------------
// With host spheres (gmnp given) the exciting field is the interaction
// without the Mie multiply plus the incident field, and each sphere sits in
// the index rext around it (qefficiencyfactors, scatprops:807-840).
__global__ void qeff_kernel(int nsph, const int* order, const int* offset, const int* mie_offset, const double* radius, zd rimed,
                            const zd* an_inv, const zd* amnp, const zd* pmnp0, int ld, double* qeff, const double* rext, const zd* gmnp)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsph) return;
    int L = order[i], off = offset[i];
    double xsp = radius[i];
    zd ri0 = rext ? mk(rext[2 * i], rext[2 * i + 1]) : rimed;
    zd xri = xsp * ri0;
    zd rib = cdivr(2.0, cdivr(1.0, ri0) + cdivr(1.0, ri0));
    zd psi[MIE_NMAX], xi[MIE_NMAX], scr[2 * MIE_NMAX];
    mstm_cricbessel(L, xri, psi, scr);
    mstm_crichankel(L, xri, xi, scr);
    double qe[3] = {0, 0, 0}, qa[3] = {0, 0, 0}, qi[3] = {0, 0, 0};
    const zd* Ai = an_inv + mie_offset[i];
    int hb = L * (L + 2);
    for (int n = 1; n <= L; n++) {
        zd psip = psi[n - 1] - cdiv((double)n * psi[n], xri);
        zd xip = xi[n - 1] - cdiv((double)n * xi[n], xri);
        zd aam[4], ggm[4], agm[4];
        zd cterm = imul(cdiv(cj(cdivr(1.0, ri0)), ri0));
        for (int s = 1; s <= 2; s++) {
            double ss = pm1(s);
            for (int t = 1; t <= 2; t++) {
                double st = pm1(t);
                int k = (s - 1) + 2 * (t - 1);
                aam[k] = cterm * (xip * cj(xi[n]) - (ss * st) * (xi[n] * cj(xip)));
                ggm[k] = cterm * (psip * cj(psi[n]) - (ss * st) * (psi[n] * cj(psip)));
                agm[k] = cterm * (xip * cj(psi[n]) - (ss * st) * (xi[n] * cj(psip)));
            }
        }
        const zd* Ain = Ai + 4 * (n - 1);
        for (int m = -n; m <= n; m++) {
            int a0 = aidx(m, n, 0, L);
            zd av[2][2], gv[2][2], fv[2][2];   // [pol][mode]
            for (int pol = 0; pol < 2; pol++) {
                zd x0 = amnp[(size_t)pol * ld + off + a0], x1 = amnp[(size_t)pol * ld + off + a0 + hb];
                av[pol][0] = x0;
                av[pol][1] = x1;
                if (gmnp) {
                    gv[pol][0] = gmnp[(size_t)pol * ld + off + a0];
                    gv[pol][1] = gmnp[(size_t)pol * ld + off + a0 + hb];
                } else {
                    // onemiecoeffmult with the inverse: g(p) = sum_q Ainv(p,q) a(q)
                    gv[pol][0] = Ain[0] * x0 + Ain[2] * x1;
                    gv[pol][1] = Ain[1] * x0 + Ain[3] * x1;
                }
                fv[pol][0] = pmnp0[(size_t)pol * ld + off + a0];
                fv[pol][1] = pmnp0[(size_t)pol * ld + off + a0 + hb];
            }
            for (int p1 = 0; p1 < 2; p1++)
                for (int p2 = 0; p2 < 2; p2++) {
                    int k;
                    double cst;
                    if (p1 == 0 && p2 == 0) { k = 0; cst = 1.0; }
                    else if (p1 == 1 && p2 == 1) { k = 1; cst = 1.0; }
                    else { k = 2; cst = 0.5; }
                    for (int s = 0; s < 2; s++)
                        for (int t = 0; t < 2; t++) {
                            int mk_ = s + 2 * t;
                            double sgn = pm1(s + t);
                            zd crib = cj(rib) + sgn * rib;
                            qi[k] = qi[k] + (cst * (ggm[mk_] * fv[p1][s] * cj(rib * fv[p2][t]))).x;
                            qa[k] = qa[k] + (cst * (aam[mk_] * av[p1][s] * cj(rib * av[p2][t]) + ggm[mk_] * gv[p1][s] * cj(rib * gv[p2][t]) +
                                                    agm[mk_] * av[p1][s] * cj(gv[p2][t]) * crib)).x;
                            qe[k] = qe[k] + (cst * (agm[mk_] * av[p1][s] * cj(fv[p2][t]) * crib)).x;
                        }
                }
        }
    }
    double qeffi[3][3];
    for (int k = 0; k < 3; k++) {
        qi[k] = qi[k] * 2.0 / xsp / xsp;
        qe[k] = qe[k] * 2.0 / xsp / xsp;
        qa[k] = qa[k] * 2.0 / xsp / xsp;
        qeffi[0][k] = qe[k];
        qeffi[1][k] = qa[k];
        qeffi[2][k] = qi[k];
    }
    for (int q = 0; q < 3; q++) {
        qeff[q + 3 * (0 + 3 * i)] = 0.5 * (qeffi[q][0] + qeffi[q][1]);
        qeff[q + 3 * (1 + 3 * i)] = qeffi[q][0];
        qeff[q + 3 * (2 + 3 * i)] = qeffi[q][1];
    }
}

// qtotcalc (scatprops:872-912), no host spheres, one block, fixed summation order.
// qtotcalc (scatprops:872-912): one block of QTOT_NT threads, strided partial
// sums of the area-weighted efficiencies reduced in shared memory (the
// reference sums the spheres in order; only the summation order differs)
#define QTOT_NT 256
__global__ void __launch_bounds__(QTOT_NT) qtot_kernel(int nsph, const double* radius, const double* qeff, double xg, double* qtot)
{
    __shared__ double red[9][QTOT_NT];
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < nsph; i += QTOT_NT)
        for (int k = 0; k < 9; k++) s[k] = s[k] + qeff[k + 9 * i] * radius[i] * radius[i] / (xg * xg);
    for (int k = 0; k < 9; k++) red[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int w = QTOT_NT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 9; k++) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double t[9];
        for (int k = 0; k < 9; k++) t[k] = red[k][0];
        for (int pol = 0; pol < 3; pol++) t[2 + 3 * pol] = t[0 + 3 * pol] + t[2 + 3 * pol] - t[1 + 3 * pol];
        for (int k = 0; k < 9; k++) qtot[k] = t[k];
    }
}

// totals over the spheres of each configuration of an ensemble (one thread
// a configuration, the spheres summed in order as qtotcalc does)
__global__ void qtot_configs_kernel(int nc, const int* cfg_start, const double* radius, const double* qeff, const double* xg, double* qtot)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nc) return;
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = cfg_start[k]; i < cfg_start[k + 1]; i++)
        for (int q = 0; q < 9; q++) s[q] = s[q] + qeff[q + 9 * i] * radius[i] * radius[i] / (xg[k] * xg[k]);
    for (int pol = 0; pol < 3; pol++) s[2 + 3 * pol] = s[0 + 3 * pol] + s[2 + 3 * pol] - s[1 + 3 * pol];
    for (int q = 0; q < 9; q++) qtot[q + 9 * k] = s[q];
}

void launch_qtot_configs(int nc, const int* cfg_start, const double* radius, const double* qeff, const double* xg, double* qtot, cudaStream_t st)
{
    qtot_configs_kernel<<<(nc + 63) / 64, 64, 0, st>>>(nc, cfg_start, radius, qeff, xg, qtot);
    launch_counter() += 1;
}

// qtotcalc (scatprops:872-912) with host spheres, one block: each host's
// absorption net of the spheres it holds (qabsvol), then theirs added back,
// both scaled by the area ratio, written into qeff's absorption rows as the
// reference does; the totals over the spheres outside every other.
// qv: scratch of 3 nsph doubles.
// held[hstart[i] .. hstart[i+1]): the spheres sphere i holds, in order
__global__ void __launch_bounds__(QTOT_NT) qtot_hosts_kernel(int nsph, const double* radius, const int* host, const int* hstart,
                                                             const int* held, double* qeff, double* qv, double xg, double* qtot)
{
    __shared__ double red[9][QTOT_NT];
    for (int i = threadIdx.x; i < nsph; i += QTOT_NT)
        for (int p = 0; p < 3; p++) {
            double v = qeff[1 + 3 * (p + 3 * i)];
            for (int q = hstart[i]; q < hstart[i + 1]; q++) {
                const int j = held[q];
                v = v - qeff[1 + 3 * (p + 3 * j)] * radius[j] * radius[j] / (radius[i] * radius[i]);
            }
            qv[p + 3 * i] = v;
        }
    __syncthreads();
    for (int i = threadIdx.x; i < nsph; i += QTOT_NT)
        for (int p = 0; p < 3; p++) {
            double v = qv[p + 3 * i];
            for (int q = hstart[i]; q < hstart[i + 1]; q++) {
                const int j = held[q];
                v = v + qv[p + 3 * j] * radius[j] * radius[j] / (radius[i] * radius[i]);
            }
            qeff[1 + 3 * (p + 3 * i)] = v;
        }
    __syncthreads();
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < nsph; i += QTOT_NT)
        if (host[i] < 0)
            for (int k = 0; k < 9; k++) s[k] = s[k] + qeff[k + 9 * i] * radius[i] * radius[i] / (xg * xg);
    for (int k = 0; k < 9; k++) red[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int w = QTOT_NT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 9; k++) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double t[9];
        for (int k = 0; k < 9; k++) t[k] = red[k][0];
        for (int pol = 0; pol < 3; pol++) t[2 + 3 * pol] = t[0 + 3 * pol] + t[2 + 3 * pol] - t[1 + 3 * pol];
        for (int k = 0; k < 9; k++) qtot[k] = t[k];
    }
}

void launch_qeff(int nsph, const int* order, const int* offset, const int* mie_offset, const double* radius, zd rimed, const zd* an_inv,
                 const zd* amnp, const zd* pmnp0, int ld, double* qeff, double xg, double* qtot, cudaStream_t st, const double* rext,
                 const zd* gmnp, const int* host, double* qv, const int* hstart, const int* held)
{
    qeff_kernel<<<(nsph + 63) / 64, 64, 0, st>>>(nsph, order, offset, mie_offset, radius, rimed, an_inv, amnp, pmnp0, ld, qeff, rext, gmnp);
    if (host) qtot_hosts_kernel<<<1, QTOT_NT, 0, st>>>(nsph, radius, host, hstart, held, qeff, qv, xg, qtot);
    else qtot_kernel<<<1, QTOT_NT, 0, st>>>(nsph, radius, qeff, xg, qtot);
    launch_counter() += 2;
}
