// densepair.cuh -- dense pair translation (densepair.cu).
#pragma once
#include "common.cuh"
#include "gentran.cuh"

struct DenseArgs {
    int npairs;
    const int2* pairs;       // (i, j), i < j
    const int* order;
    const int* offset;
    const double* pos;
    const long long* off;    // record offset per pair (complex units); record = nblk_i x nblk_j x 2
    zd* rec64;               // generation targets (either may be null)
    zf* rec32;
    double rimed_re, rimed_im;
    const double* pmed = nullptr;   // per pair re, im: the index the pair sits in (null: rimed)
    GtConst g;
};

void launch_dense_gen(const DenseArgs& a, cudaStream_t st);
template <typename T> void launch_dense_apply(const DenseArgs& a, const T* rec, const cpx<T>* x, cpx<T>* y, int ld, int nrhs, unsigned contran,
                                              cudaStream_t st);
