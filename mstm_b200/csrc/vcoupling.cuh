// vcoupling.cuh -- vector-coupling coefficients, one implementation for the
// host tables (tables.cpp) and the device kernels (postproc.cu, ranorient.cu).
//
// vcfunc / vcfuncuprec (december2023/mstm-modules-33.f90:950-1056): the
// coefficients C_w(m, n, k, l) of the product of two Wigner functions for
// w = |n - l| .. n + l, by the downward recurrence in w from w = n + l, which
// hands over to the upward recurrence (vcfuncuprec) from the lowest w once
// the downward values have fallen below 1 % of their largest.  Tab supplies
// bc(n, l) = ((n+l)! / (n! l!))^(1/2) and fr(n) = sqrt(n).
#pragma once
#include <cmath>
#include <cstdlib>

#ifdef __CUDACC__
#define VC_HD __host__ __device__
#else
#define VC_HD
#endif

// bcof / fnr tables of side nbc + 1 in device or host memory
struct VCTab {
    const double* bcof;  // (nbc+1)^2
    const double* fnr;   // 0..2*nbc
    int nbc;
    VC_HD double bc(int n, int l) const { return bcof[(size_t)n * (nbc + 1) + l]; }
    VC_HD double fr(int n) const { return fnr[n]; }
};

namespace vcc {
VC_HD inline double sgn(int n) { return (n & 1) ? -1.0 : 1.0; }
VC_HD inline int iabs(int a) { return a < 0 ? -a : a; }
VC_HD inline int imin(int a, int b) { return a < b ? a : b; }
VC_HD inline int imax(int a, int b) { return a > b ? a : b; }
}  // namespace vcc

// vcfuncuprec: upward in w from the lowest w up to min(wmax, n + l)
template <typename Tab> VC_HD void vc_uprec(const Tab& t, int m, int n, int k, int l, int wmax, double* vcn)
{
    int mk = vcc::iabs(m + k), nl = vcc::iabs(n - l), w, m1, l1, k1;
    double vc1;
    if (nl >= mk) {
        w = nl;
        if (n >= l) { m1 = m; l1 = l; k1 = k; }
        else { m1 = k; k1 = m; l1 = n; }
        vc1 = vcc::sgn(k1 + l1) * t.bc(l1 + k1, w - m1 - k1) * t.bc(l1 - k1, w + m1 + k1) / t.bc(l1 + l1, w + w + 1);
    } else {
        w = mk;
        if (m + k >= 0) vc1 = vcc::sgn(n + m) * t.bc(n - l + w, l - k) * t.bc(l - n + w, n - m) / t.bc(w + w + 1, n + l - w);
        else vc1 = vcc::sgn(l + k) * t.bc(n - l + w, l + k) * t.bc(l - n + w, n + m) / t.bc(w + w + 1, n + l - w);
    }
    const int w1 = w;
    vcn[w] = vc1;
    w = w1 + 1;
    mk = m + k;
    const int w2 = vcc::imin(wmax, n + l);
    auto t1f = [&](int w_) {
        return 2 * w_ * t.fr(w_ + w_ + 1) * t.fr(w_ + w_ - 1) /
               (t.fr(w_ + mk) * t.fr(w_ - mk) * t.fr(n - l + w_) * t.fr(l - n + w_) * t.fr(n + l - w_ + 1) * t.fr(n + l + w_ + 1));
    };
    auto t2f = [&](int w_) {
        return (double)((m - k) * w_ * (w_ - 1) - mk * n * (n + 1) + mk * l * (l + 1)) / (double)(2 * w_ * (w_ - 1));
    };
    auto t3f = [&](int w_) {
        return t.fr(w_ - mk - 1) * t.fr(w_ + mk - 1) * t.fr(l - n + w_ - 1) * t.fr(n - l + w_ - 1) * t.fr(n + l - w_ + 2) * t.fr(n + l + w_) /
               ((double)(2 * (w_ - 1)) * t.fr(2 * w_ - 3) * t.fr(2 * w_ - 1));
    };
    if (w2 > w1) {
        const double t2 = (w1 == 0) ? 0.5 * (double)(m - k) : t2f(w);
        vcn[w] = t1f(w) * t2 * vcn[w1];
    }
    for (w = w1 + 2; w <= w2; w++) vcn[w] = t1f(w) * (t2f(w) * vcn[w - 1] - t3f(w) * vcn[w - 2]);
}

// vcfunc: vcn[0 .. n + l] (zero below the lowest w)
template <typename Tab> VC_HD void vc_func(const Tab& t, int m, int n, int k, int l, double* vcn)
{
    for (int w = 0; w <= n + l; w++) vcn[w] = 0.0;
    const int wmax = n + l;
    const int wmin = vcc::imax(vcc::iabs(n - l), vcc::iabs(m + k));
    vcn[wmax] = t.bc(n + m, l + k) * t.bc(n - m, l - k) / t.bc(n + n, l + l);
    if (wmin == wmax) return;
    vcn[wmax - 1] = vcn[wmax] * (l * m - k * n) * t.fr(2 * (l + n) - 1) / t.fr(l) / t.fr(n) / t.fr(n + l + m + k) / t.fr(n + l - m - k);
    if (wmin == wmax - 1) return;
    const int mk = m + k;
    double vcmax = fabs(vcn[wmax]) + fabs(vcn[wmax - 1]);
    int w;
    for (w = wmax; w >= wmin + 2; w--) {
        const double t1 = 2 * w * t.fr(w + w + 1) * t.fr(w + w - 1) /
                          (t.fr(w + mk) * t.fr(w - mk) * t.fr(n - l + w) * t.fr(l - n + w) * t.fr(n + l - w + 1) * t.fr(n + l + w + 1));
        const double t2 = (double)((m - k) * w * (w - 1) - mk * n * (n + 1) + mk * l * (l + 1)) / (double)(2 * w * (w - 1));
        const double t3 = t.fr(w - mk - 1) * t.fr(w + mk - 1) * t.fr(l - n + w - 1) * t.fr(n - l + w - 1) * t.fr(n + l - w + 2) * t.fr(n + l + w) /
                          ((double)(2 * (w - 1)) * t.fr(2 * w - 3) * t.fr(2 * w - 1));
        vcn[w - 2] = (t2 * vcn[w - 1] - vcn[w] / t1) / t3;
        if ((wmax - w) % 2 == 1) {
            const double vctest = fabs(vcn[w - 2]) + fabs(vcn[w - 1]);
            vcmax = vcmax > vctest ? vcmax : vctest;
            if (vctest / vcmax < 0.01) break;
        }
    }
    if (w - 2 > wmin) vc_uprec(t, m, n, k, l, w - 3, vcn);
}
