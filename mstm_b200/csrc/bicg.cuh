// bicg.cuh -- BiCG device scalars and vector-kernel launchers.
#pragma once
#include "common.cuh"

struct BicgScalars {
    double csk[2], alpha[2], beta[2];
    double enorm, eerr;
    int stop, breakdown;
    int pad[2];
    double csk_prev[2];   // csk before the last update (residual replacement recomputes beta from it)
};

struct SlotMaps {
    int nslots;              // neqns/2: (m,n) slots of the first mode half of all sphere blocks
    const int* slot;         // slot -> sphere
    const int* order;
    const int* offset;
    const int* mie_offset;
};

int reduce_grid(int n, int nsm);
template <typename T>
void launch_post(const SlotMaps& sm, const cpx<T>* an, const cpx<T>* p, const cpx<T>* w, const cpx<T>* y0, const cpx<T>* y1,
                 cpx<T>* cap, cpx<T>* caw, double* part, BicgScalars* sc, int nsm, cudaStream_t st);
template <typename T>
void launch_init(const SlotMaps& sm, const cpx<T>* an, const cpx<T>* b, const cpx<T>* x, const cpx<T>* y0, int have_y, cpx<T>* r,
                 cpx<T>* p, cpx<T>* w, cpx<T>* q, double* part, BicgScalars* sc, int normalize, int nsm, cudaStream_t st);
template <typename T>
void launch_upd(int n, cpx<T>* x, cpx<T>* r, cpx<T>* q, cpx<T>* p, cpx<T>* w, const cpx<T>* cap, const cpx<T>* caw, double* part,
                BicgScalars* sc, double eps, int nsm, cudaStream_t st);
template <typename T, typename TB>
void launch_resid(const SlotMaps& sm, const cpx<T>* an, const cpx<T>* b, const cpx<T>* x, const cpx<T>* y, cpx<TB>* rout, double* part,
                  double* out2, int nsm, cudaStream_t st);
void launch_add_correction_f(int n, zd* x, const zf* d, cudaStream_t st);
void launch_add_correction_d(int n, zd* x, const zd* d, cudaStream_t st);
void launch_rr_dot_norm(int n, const zd* v, double* part, double* out, int nsm, cudaStream_t st);   // out[0] = sum |v|^2
template <typename T> void launch_conj_copy(int n, const cpx<T>* a, cpx<T>* b, cudaStream_t st);
void launch_d2f(int n, const zd* a, zf* b, cudaStream_t st);
