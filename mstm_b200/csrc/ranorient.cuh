// ranorient.cuh -- orientation-averaged scattering matrix from the T matrix (ranorient.cu).
#pragma once
#include "common.cuh"
#include <cstddef>
#include <algorithm>

#define RO_NT 128

struct RoArgs {
    int nodr;              // T-matrix order
    float2* tc;            // nblkt x nblkt single-precision GB-modified T matrix
    zd* trace;             // 4 nodr: per-order traces (coherent part)
    zd* dm;                // ro_dm_elems(nodr), zeroed by the caller
    zd* dmcf;
    zd* fm;                // (2 nodr + 1) x 2 x 3 nodr 2 nodr 2
    double* sm;            // 16 x (2 nodr + 1) expansion coefficients
    double* smcf;          // coherent part
    const double* bcof;    // bcof table (nbc + 1)^2
    const double* fnr;     // sqrt table
    int nbc;
    double* vscr;          // ro_vscr_doubles(nodr, nsm)
    double rimed_re;
};

size_t ro_dm_smem(int nodr);
int ro_dm_grid(int nodr, int nsm);
size_t ro_vscr_doubles(int nodr, int nsm);
size_t ro_dm_elems(int nodr);
// returns -1 when the order needs more shared memory than a CTA has
int launch_ranorient(const RoArgs& a, const zd* tmat, int nang, const double* bcofd, double* dscr, double* smat, int nsm, cudaStream_t st);
