// tables.h -- host FP64 constant tables (see tables.cpp).
#pragma once
#include <vector>
#include <algorithm>

namespace mstmg {

struct Tables {
    int nbc;
    std::vector<double> fnr;   // sqrt(n), n = 0..2*nbc
    std::vector<double> bcof;  // ((n+l)!/(n! l!))^(1/2), (nbc+1)^2
    explicit Tables(int nbc);
    double bc(int n, int l) const { return bcof[(size_t)n * (nbc + 1) + l]; }
    void vcfunc(int m, int n, int k, int l, double* vcn) const;
    void vcfuncuprec(int m, int n, int k, int l, int wmax, double* vcn) const;
    void axial_constants(int nmax, std::vector<double>& vcc, std::vector<double>& fnm1, std::vector<double>& fnc,
                         std::vector<double>& fnp1) const;
};

}  // namespace mstmg
