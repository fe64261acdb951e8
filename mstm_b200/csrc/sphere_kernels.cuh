// sphere_kernels.cuh -- launchers for the per-sphere kernels.
#pragma once
#include "common.cuh"

// rext (per sphere re, im; null: the medium for every sphere) is the index
// around each sphere; hoff (null: none) marks the spheres holding others,
// which also get the D, U, V coefficients
void launch_mie_orders(int n, const double* radius, const double* ri, double mre, double mim, const double* rext, double qeps, int* order,
                       cudaStream_t st);
void launch_mie_coefs(int n, const double* radius, const double* ri, double mre, double mim, const double* rext, const int* order,
                      const int* mie_offset, const int* hoff, zd* an, zd* an_inv, float* an32, zd* dn, zd* un, zd* vn, double* qext,
                      double* qabs, cudaStream_t st);
// outside (null: every sphere): 1 for the spheres the incident wave reaches
void launch_planewave(double alpha, double sinc, int dir, int lmax, int neqns, const int* slot_full, const int* order,
                      const int* offset, const double* pos, zd* pw0, zd* drot, zd* pmnp, cudaStream_t st, int nreal = 0,
                      const int* outside = nullptr);
// Mie multiply with host spheres' second blocks at hoff[i] (>= 0)
template <typename T>
void launch_hmie(int nslots, int nreal, const int* slot_sphere, const int* order, const int* offset, const int* mie_offset, const int* hoff,
                 const cpx<T>* an, const cpx<T>* dn, const cpx<T>* un, const cpx<T>* vn, int idir, int conj_in, const cpx<T>* x, cpx<T>* y,
                 cudaStream_t st);
// per-configuration totals of an ensemble: qtot[9 k ..] from the spheres
// cfg_start[k] .. cfg_start[k+1]-1, volume radius xg[k] (device arrays)
void launch_qtot_configs(int nc, const int* cfg_start, const double* radius, const double* qeff, const double* xg, double* qtot, cudaStream_t st);
// with host spheres: rext the index around each sphere, gmnp the exciting
// fields (interaction without the Mie multiply plus incident), host the
// holding sphere (-1 none), held[hstart[i] .. hstart[i+1]) the spheres
// sphere i holds and qv a scratch of 3 nsph doubles
void launch_qeff(int nsph, const int* order, const int* offset, const int* mie_offset, const double* radius, zd rimed,
                 const zd* an_inv, const zd* amnp, const zd* pmnp0, int ld, double* qeff, double xg, double* qtot,
                 cudaStream_t st, const double* rext = nullptr, const zd* gmnp = nullptr, const int* host = nullptr,
                 double* qv = nullptr, const int* hstart = nullptr, const int* held = nullptr);
