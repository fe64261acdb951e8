// postproc.cuh -- device post-processing launchers (see postproc.cu).
#pragma once
#include "common.cuh"
#include <cstddef>

// Regular (J) translation between the cluster origin and every sphere.
// mode 0 (merge_to_common_origin): sphere block (order L_i, LR) -> origin block
//   of order min(T, tord_i), converted to TE/TM and accumulated into amnp0;
// mode 1 (distribute_from_common_origin): origin block of order T (LR, column p
//   of amnp, leading dimension ld) -> sphere block of order L_i written to out.
struct MergeArgs {
    int mode;
    zd* out;                // mode 1: ldo x npol sphere blocks (zeroed by the caller)
    int ldo;
    int nsph;
    const double* pos;
    const int* order;
    const int* offset;
    const int* tord;        // translation order per sphere (already capped)
    int T;                  // t_matrix_order
    double r0[3];
    double rimed_re, rimed_im;
    const zd* amnp;         // ld x npol, LR basis
    int ld, npol;
    zd* amnp0;              // ld0 x npol, TE/TM basis, accumulated (zeroed by the caller)
    int ld0;
    const double* vcc;      // vcc_const slice (n <= vcT, ml <= vcML, w <= vcT + L)
    int vcT, vcML;
    const double* fnm1;     // (-fcN..fcN, 1..fcN)
    const double* fnc;
    const double* fnp1;
    int fcN;
    const double* fnr;
    const double* bcofd;
    zd* scratch;
    size_t scratch_stride;  // zd units per CTA
    const int* active = nullptr;   // with host spheres: 1 for the spheres merged or distributed to (those outside every other)
};

size_t tranorder_scratch(int nsph, int sstride);   // complex values of scratch launch_tranorder needs
void launch_tranorder(int nsph, const double* pos, const int* order, const double* origin, double rire, double eps, int maxt,
                      const double* bcof, const double* fnr, int nbc, zd* scratch, int sstride, int* tord, cudaStream_t st);
#define MERGE_PC 16   // columns a CTA of the merge kernel translates together
// zd units of merge-kernel scratch per CTA; a launch of `grid` CTAs per chunk
// of MERGE_PC columns needs grid * merge_chunks(npol) of them
size_t merge_scratch_per_cta(int T, int L);
int merge_chunks(int npol);
// grid CTAs over the spheres times merge_chunks(npol) column chunks
void launch_merge(const MergeArgs& a, int grid, cudaStream_t st);
int fosm_grid(int ntot);
size_t fosm_scratch_doubles(int ntot);
size_t fosmcalc_scratch_doubles(int ntot, int nang);
void launch_fosm(int ntot, const zd* a0, const double* bcof, const double* fnr, int nbc, double* s00, double* s02, double* sp22,
                 double* sm22, double* vscr, cudaStream_t st);
void launch_fosmcalc(int ntot, int nang, const double* s00, const double* s02, const double* sp22, const double* sm22,
                     const double* fnr, const double* bcofd, double* dscr, double* smat, cudaStream_t st);

// scatteringmatrix at the directions i = ldim..udim of scattering_matrix_calculation
#define PS_TMAX 200
struct PlaneSmArgs {
    int T;                  // order of the origin expansion (<= PS_TMAX)
    const zd* a0;           // 2T(T+2) x 2, TE/TM basis
    int ldim, udim;         // udim > ldim
    double amin, amax;      // degrees
    double alpha;           // incident azimuth (radians)
    int rotate;             // rotate_plane
    double rimed_re;
    const double* fnr;      // sqrt table, indices 0..2T+1
    const double* bcofd;    // bcof(n, n), n = 0..T
    double* smat;           // 16 x (udim - ldim + 1)
};
void launch_planesm(const PlaneSmArgs& a, cudaStream_t st);
