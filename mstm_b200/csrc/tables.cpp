// tables.cpp -- host-side FP64 constant tables uploaded once per context:
// the sqrt table and binomial roots of MSTM's numconstants::init
// (december2023/mstm-modules-33.f90:23-113), the vector-coupling
// coefficients (vcfunc / vcfuncuprec, modules:950-1056) and the axial
// translation constants vcc_const, fnm1_const, fn_const, fnp1_const
// (axialtrancoefinit, modules:1680-1722).
#include "tables.h"
#include "vcoupling.cuh"
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
    vc_uprec(VCTab{bcof.data(), fnr.data(), nbc}, m, n, k, l, wmax, vcn);
}

void Tables::vcfunc(int m, int n, int k, int l, double* vcn) const
{
    vc_func(VCTab{bcof.data(), fnr.data(), nbc}, m, n, k, l, vcn);
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
