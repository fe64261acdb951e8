// kernels.cuh -- argument blocks and launchers shared by the .cu files.
#pragma once
#include "common.cuh"

struct OpGenArgs {
    int npairs;
    const int2* pairs;       // (i, j), i < j
    const double* pos;       // 3N
    const int* order;        // N
    const long long* opoff;  // per pair, in storage units
    double* op64;            // may be null
    float* op32;             // may be null
    int row32;               // > 0: op32 holds row records (translate_rows.cuh) of one order, row32 floats each
    const double* vcc;       // vcc_const(vn, vn(vn+2), 0:2vn)
    int vnmax;
    const double* fnr;       // fnr[k] = sqrt(k)
    const double* rfnr;      // 1 / sqrt(k) (k >= 1)
    const double* bcofd;     // bcof(n,n)
    double rimed_re, rimed_im;
    const double* pmed = nullptr;   // per pair re, im: the index the pair sits in (null: rimed)
    int regular = 0;         // 1: regular translations (vswf_type 1, Bessel j) instead of outgoing
    int* err;
    zd* xi;                  // scratch, opgen_xi_scratch(npairs) complex: Hankel (or Bessel) functions per pair
};

#include "oplayout.cuh"
size_t opgen_xi_scratch(int npairs);
void launch_opgen(const OpGenArgs& a, int nsm, cudaStream_t st);

template <typename T> struct TransArgs {
    int npairs;
    const int2* pairs;
    const int* order;
    const int* offset;       // sphere_offset (complex units)
    const T* ops;
    const long long* opoff;  // storage units
    const cpx<T>* x;         // ld x nrhs
    cpx<T>* y;               // ld x nrhs, accumulated
    int ld;
    int nrhs;
    unsigned contran;        // bit r set: rhs r is a conjugate-transpose product
    int lmax;                // largest order (smem strides)
    int maxrec;              // largest operator record, storage units
    int* err;
    int uniform = 0;         // 1: every pair has both orders lmax
};
template <typename T> void launch_translate(const TransArgs<T>& a, int nsm, cudaStream_t st);
template <typename T> size_t translate_smem_bytes(int lmax, int nrhs, int maxrec);
// y(:, r) += the order-truncated copies between the blocks of each pair
// (i, j) and back: coincident centres of a host and a sphere it holds
template <typename T>
void launch_mtransfer(int npairs, const int2* pairs, const int* order, const int* offset, const cpx<T>* x, cpx<T>* y, int ld, int nrhs,
                      cudaStream_t st);

// Mie multiply over all spheres: y(:,r) = A x(:,r) (idir=1) or A^T x(:,r);
// optional conjugation of the input.  slot_sphere maps each (row, column)
// slot of the first mode half of every sphere block to its sphere.
template <typename T> void launch_mie(int nslots, const int* slot_sphere, const int* order, const int* offset,
                                      const int* mie_offset, const cpx<T>* an, int idir, int conj_in,
                                      const cpx<T>* x, cpx<T>* y, cudaStream_t st);
