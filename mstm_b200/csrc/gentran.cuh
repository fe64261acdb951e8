// gentran.cuh -- dense VSWF translation matrices on the device
// (gentranmatrix, december2023/mstm-modules-33.f90:1762-1888, with the
// tran_coef constants of gentrancoefconstants, :1724-1760, built on the host).
//
// One translation per CTA: gt_prepare fills the CTA's shared tables (e^{i m phi},
// the normalised Legendre functions ymn(v, w) of normalizedlegendre,
// modules:1063-1085, and the radial functions h_w or j_w of the translation
// distance), then any thread evaluates matrix elements with gt_element.
#pragma once
#include "common.cuh"
#include "special.cuh"
#include <vector>

#define GT_WMAX 40   // largest nodr_s + nodr_t

struct GtConst {
    const double* tc;    // tran_coef(mn, kl, w), nd x nd x (2 nmax + 1), nd = nmax (nmax + 2)
    int nmax, nd;
    const double* fnr;   // sqrt(n)
    const double* bcd;   // bcof(m, m), m <= GT_WMAX
};

struct GtShared {
    zd ephim[2 * GT_WMAX + 1];
    double ymn[(2 * GT_WMAX + 1) * (GT_WMAX + 1)];
    zd hn[GT_WMAX + 2];
    zd scr[2 * (GT_WMAX + 2)];
    int zero;   // r == 0
};

// host: tran_coef for orders up to nmax (gentrancoefconstants)
void gentran_constants(int nmax, std::vector<double>& tc);

// Whole CTA.  vtype 3: outgoing (Hankel), 1: regular (Bessel).  wmax = nodr_s + nodr_t.
__device__ inline void gt_prepare(GtShared& s, const GtConst& g, const double xp[3], int vtype, zd ri, int wmax)
{
    const int tid = threadIdx.x;
    const double rr = xp[0] * xp[0] + xp[1] * xp[1] + xp[2] * xp[2];
    if (tid == 0) s.zero = (rr == 0.0);
    __syncthreads();
    if (s.zero) return;
    const double r = sqrt(rr), ct = xp[2] / r;
    if (tid == 0) {
        zd ephi = (xp[0] == 0.0 && xp[1] == 0.0) ? mk(1.0, 0.0) : mk(xp[0] / sqrt(xp[0] * xp[0] + xp[1] * xp[1]), xp[1] / sqrt(xp[0] * xp[0] + xp[1] * xp[1]));
        zd* e = s.ephim + wmax;
        e[0] = mk(1.0, 0.0);
        for (int m = 1; m <= wmax; m++) {
            e[m] = ephi * e[m - 1];
            e[-m] = cj(e[m]);
        }
        zd rri = r * ri;
        if (vtype == 3) {
            zd ci = mk(0.0, 1.0);
            s.hn[0] = -cdiv(ci * cexpd(ci * rri), rri);
            s.hn[1] = cdiv(cdiv(-(cexpd(ci * rri) * (ci + rri)), rri), rri);
            for (int n = 2; n <= wmax; n++) s.hn[n] = cdiv(mk((double)(n + n - 1), 0.0), rri) * s.hn[n - 1] - s.hn[n - 2];
        } else {
            mstm_cricbessel(wmax, rri, s.hn, s.scr);
            for (int n = 0; n <= wmax; n++) s.hn[n] = cdiv(s.hn[n], rri);
        }
    }
    // normalizedlegendre(ct, wmax, wmax): ymn(m, n), one thread per m >= 0
    const int ld = 2 * wmax + 1;
    for (int e = tid; e < ld * (wmax + 1); e += blockDim.x) s.ymn[e] = 0.0;
    __syncthreads();
    const double sbe = sqrt((1.0 + ct) * (1.0 - ct));
    for (int m = tid; m <= wmax; m += blockDim.x) {
        double* col = s.ymn + (m + wmax);   // ymn(m, n) at col[ld * n]
        double dmm = pm1(m) * pow(0.5 * sbe, (double)m) * g.bcd[m];
        col[ld * m] = dmm;
        if (m < wmax) {
            col[ld * (m + 1)] = g.fnr[m + m + 1] * ct * dmm;
            for (int n = m + 1; n <= wmax - 1; n++)
                col[ld * (n + 1)] = (-g.fnr[n - m] * g.fnr[n + m] * col[ld * (n - 1)] + (double)(n + n + 1) * ct * col[ld * n]) /
                                    (g.fnr[n + 1 - m] * g.fnr[n + 1 + m]);
        }
    }
    __syncthreads();
    for (int e = tid; e < wmax * (wmax + 1); e += blockDim.x) {
        int m = e / (wmax + 1) + 1, n = e % (wmax + 1);
        if (n >= m) s.ymn[(-m + wmax) + ld * n] = pm1(m) * s.ymn[(m + wmax) + ld * n];
    }
    __syncthreads();
}

// (m, n) of slot idx of a(0:L+1, 1:L) (index model 2)
__device__ __forceinline__ void gt_mn(int idx, int L, int& m, int& n)
{
    int row = idx % (L + 2), col = idx / (L + 2) + 1;
    if (row <= col) { m = row; n = col; }
    else { m = -col; n = row - 1; }
}

// Element (kla, mna) of both modes of gentranmatrix(nodr_s, nodr_t): target
// (l, k) of order <= nodr_t, source (n, m) of order <= nodr_s.
__device__ __forceinline__ void gt_element(const GtShared& s, const GtConst& g, int vtype, int wmaxt, int n, int m, int l, int k, zd& e1,
                                           zd& e2)
{
    if (s.zero) {
        zd v = (vtype == 1 && n == l && m == k) ? mk(1.0, 0.0) : mk(0.0, 0.0);
        e1 = v;
        e2 = v;
        return;
    }
    const int ld = 2 * wmaxt + 1;
    const int mn = n * (n + 1) + m, kl = l * (l + 1) + k, v = m - k;
    const int wmax = n + l, wmin = max(abs(v), abs(n - l));
    zd a1 = mk(0.0, 0.0), b1 = mk(0.0, 0.0);
    for (int w = wmax; w >= wmin; w--) {
        double t = g.tc[(size_t)(kl - 1) + (size_t)g.nd * ((size_t)(mn - 1) + (size_t)g.nd * w)];
        zd term = (s.hn[w] * s.ymn[(v + wmaxt) + ld * w]) * t;
        if ((wmax - w) % 2 == 0) a1 = a1 + term;
        else b1 = b1 + term;
    }
    const zd ep = s.ephim[v + wmaxt];
    e1 = ep * (a1 + imul(b1));
    e2 = ep * (a1 - imul(b1));
}
