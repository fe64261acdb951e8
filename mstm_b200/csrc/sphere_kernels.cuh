// sphere_kernels.cuh -- launchers for the per-sphere kernels.
#pragma once
#include "common.cuh"

void launch_mie_orders(int n, const double* radius, const double* ri, double mre, double mim, double qeps, int* order,
                       cudaStream_t st);
void launch_mie_coefs(int n, const double* radius, const double* ri, double mre, double mim, const int* order,
                      const int* mie_offset, zd* an, zd* an_inv, float* an32, double* qext, double* qabs, cudaStream_t st);
void launch_planewave(double alpha, double sinc, int dir, int lmax, int neqns, const int* slot_full, const int* order,
                      const int* offset, const double* pos, zd* pw0, zd* drot, zd* pmnp, cudaStream_t st);
// per-configuration totals of an ensemble: qtot[9 k ..] from the spheres
// cfg_start[k] .. cfg_start[k+1]-1, volume radius xg[k] (device arrays)
void launch_qtot_configs(int nc, const int* cfg_start, const double* radius, const double* qeff, const double* xg, double* qtot, cudaStream_t st);
void launch_qeff(int nsph, const int* order, const int* offset, const int* mie_offset, const double* radius, zd rimed,
                 const zd* an_inv, const zd* amnp, const zd* pmnp0, int ld, double* qeff, double xg, double* qtot,
                 cudaStream_t st);
