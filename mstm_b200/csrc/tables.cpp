// tables.cpp -- host-side FP64 constant tables uploaded once per context:
// the sqrt table and binomial roots of MSTM's numconstants::init
// (december2023/mstm-modules-33.f90:23-113), the vector-coupling
// coefficients (vcfunc / vcfuncuprec, modules:950-1056) and the axial
// translation constants vcc_const, fnm1_const, fn_const, fnp1_const
// (axialtrancoefinit, modules:1680-1722).
#include "tables.h"
#include <cmath>
#include <cstdlib>

namespace mstmg {

static inline double pm1(int n) { return (n & 1) ? -1.0 : 1.0; }

Tables::Tables(int nbc_) : nbc(nbc_)
{
    fnr.assign(2 * nbc + 1, 0.0);
    for (int n = 1; n <= 2 * nbc; n++) fnr[n] = std::sqrt((double)n);
    bcof.assign((size_t)(nbc + 1) * (nbc + 1), 0.0);
    auto B = [&](int n, int l) -> double& { return bcof[(size_t)n * (nbc + 1) + l]; };
    B(0, 0) = 1.0;
    for (int n = 0; n <= nbc - 1; n++) {
        for (int l = n + 1; l <= nbc; l++) {
            B(n, l) = fnr[n + l] * B(n, l - 1) / fnr[l];
            B(l, n) = B(n, l);
        }
        B(n + 1, n + 1) = fnr[n + n + 2] * fnr[n + n + 1] * B(n, n) / fnr[n + 1] / fnr[n + 1];
    }
}

void Tables::vcfuncuprec(int m, int n, int k, int l, int wmax, double* vcn) const
{
    int mk = std::abs(m + k), nl = std::abs(n - l), w, m1, l1, k1;
    double vc1;
    if (nl >= mk) {
        w = nl;
        if (n >= l) { m1 = m; l1 = l; k1 = k; }
        else { m1 = k; k1 = m; l1 = n; }
        vc1 = pm1(k1 + l1) * bc(l1 + k1, w - m1 - k1) * bc(l1 - k1, w + m1 + k1) / bc(l1 + l1, w + w + 1);
    } else {
        w = mk;
        if (m + k >= 0) vc1 = pm1(n + m) * bc(n - l + w, l - k) * bc(l - n + w, n - m) / bc(w + w + 1, n + l - w);
        else vc1 = pm1(l + k) * bc(n - l + w, l + k) * bc(l - n + w, n + m) / bc(w + w + 1, n + l - w);
    }
    int w1 = w;
    vcn[w] = vc1;
    w = w1 + 1;
    mk = m + k;
    int w2 = wmax < n + l ? wmax : n + l;
    auto t1f = [&](int w) {
        return 2 * w * fnr[w + w + 1] * fnr[w + w - 1] /
               (fnr[w + mk] * fnr[w - mk] * fnr[n - l + w] * fnr[l - n + w] * fnr[n + l - w + 1] * fnr[n + l + w + 1]);
    };
    auto t2f = [&](int w) { return (double)((m - k) * w * (w - 1) - mk * n * (n + 1) + mk * l * (l + 1)) / (double)(2 * w * (w - 1)); };
    auto t3f = [&](int w) {
        return fnr[w - mk - 1] * fnr[w + mk - 1] * fnr[l - n + w - 1] * fnr[n - l + w - 1] * fnr[n + l - w + 2] * fnr[n + l + w] /
               ((double)(2 * (w - 1)) * fnr[2 * w - 3] * fnr[2 * w - 1]);
    };
    if (w2 > w1) {
        double t1 = t1f(w);
        double t2 = (w1 == 0) ? 0.5 * (double)(m - k) : t2f(w);
        vcn[w] = t1 * t2 * vcn[w1];
    }
    for (w = w1 + 2; w <= w2; w++) vcn[w] = t1f(w) * (t2f(w) * vcn[w - 1] - t3f(w) * vcn[w - 2]);
}

void Tables::vcfunc(int m, int n, int k, int l, double* vcn) const
{
    for (int w = 0; w <= n + l; w++) vcn[w] = 0.0;
    int wmax = n + l;
    int wmin = std::max(std::abs(n - l), std::abs(m + k));
    vcn[wmax] = bc(n + m, l + k) * bc(n - m, l - k) / bc(n + n, l + l);
    if (wmin == wmax) return;
    vcn[wmax - 1] = vcn[wmax] * (l * m - k * n) * fnr[2 * (l + n) - 1] / fnr[l] / fnr[n] / fnr[n + l + m + k] / fnr[n + l - m - k];
    if (wmin == wmax - 1) return;
    int mk = m + k;
    double vcmax = std::fabs(vcn[wmax]) + std::fabs(vcn[wmax - 1]);
    int w;
    for (w = wmax; w >= wmin + 2; w--) {
        double t1 = 2 * w * fnr[w + w + 1] * fnr[w + w - 1] /
                    (fnr[w + mk] * fnr[w - mk] * fnr[n - l + w] * fnr[l - n + w] * fnr[n + l - w + 1] * fnr[n + l + w + 1]);
        double t2 = (double)((m - k) * w * (w - 1) - mk * n * (n + 1) + mk * l * (l + 1)) / (double)(2 * w * (w - 1));
        double t3 = fnr[w - mk - 1] * fnr[w + mk - 1] * fnr[l - n + w - 1] * fnr[n - l + w - 1] * fnr[n + l - w + 2] * fnr[n + l + w] /
                    ((double)(2 * (w - 1)) * fnr[2 * w - 3] * fnr[2 * w - 1]);
        vcn[w - 2] = (t2 * vcn[w - 1] - vcn[w] / t1) / t3;
        if ((wmax - w) % 2 == 1) {
            double vctest = std::fabs(vcn[w - 2]) + std::fabs(vcn[w - 1]);
            vcmax = vcmax > vctest ? vcmax : vctest;
            if (vctest / vcmax < 0.01) break;
        }
    }
    if (w - 2 > wmin) vcfuncuprec(m, n, k, l, w - 3, vcn);
}

void Tables::axial_constants(int nmax, std::vector<double>& vcc, std::vector<double>& fnm1, std::vector<double>& fnc,
                             std::vector<double>& fnp1) const
{
    vcc.assign((size_t)nmax * nmax * (nmax + 2) * (2 * nmax + 1), 0.0);
    auto V = [&](int n, int ml, int w) -> double& {
        return vcc[(size_t)(n - 1) + (size_t)nmax * ((size_t)(ml - 1) + (size_t)nmax * (nmax + 2) * w)];
    };
    std::vector<double> vc1(2 * nmax + 2), vc2(2 * nmax + 2);
    for (int n = 1; n <= nmax; n++) {
        for (int l = 1; l <= nmax; l++) {
            double c1 = fnr[n + n + 1] * fnr[l + l + 1];
            vcfunc(-1, n, 1, l, vc2.data());
            int wmin = std::abs(n - l), wmax = n + l, nlmin = std::min(l, n);
            for (int m = -nlmin; m <= nlmin; m++) {
                int ml = l * (l + 1) + m;
                double c2 = -c1 * pm1(m);
                vcfunc(-m, n, m, l, vc1.data());
                for (int w = wmin; w <= wmax; w++) {
                    int e = ((n - l + w) % 4 + 4) % 4;   // i^(n-l+w): real+imag part
                    double ri = (e == 0) ? 1.0 : (e == 1 ? 1.0 : (e == 2 ? -1.0 : -1.0));
                    V(n, ml, w) = c2 * vc1[w] * vc2[w] * ri;
                }
            }
        }
    }
    size_t nf = (size_t)(2 * nmax + 1) * nmax;
    fnm1.assign(nf, 0.0);
    fnc.assign(nf, 0.0);
    fnp1.assign(nf, 0.0);
    for (int m = -nmax; m <= nmax; m++)
        for (int l = std::max(1, std::abs(m)); l <= nmax; l++) {
            size_t ix = (size_t)(m + nmax) + (2 * nmax + 1) * (size_t)(l - 1);
            int lp1 = l + 1, lm1 = l - 1;
            fnm1[ix] = fnr[lm1] * fnr[lp1] * fnr[l - m] * fnr[l + m] / fnr[lm1 + l] / fnr[l + lp1] / (double)l;
            fnc[ix] = (double)m / (double)l / (double)lp1;
            fnp1[ix] = fnr[l] * fnr[l + 2] * fnr[lp1 - m] * fnr[lp1 + m] / fnr[l + lp1] / fnr[l + l + 3] / (double)lp1;
        }
}

}  // namespace mstmg
