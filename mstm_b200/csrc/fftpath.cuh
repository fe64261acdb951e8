// fftpath.cuh -- the FFT translation path (fftpath.cu).
#pragma once
#include "common.cuh"
#include "gentran.cuh"

#define FFT_NT 128
#define FFT_NBN_MAX 440   // node order <= 20

struct FftJArgs {
    int nsph, No;
    const int* order;
    const double* pos;
    const int* snode;        // 3N, 1-based cell of each sphere
    double dcell, cb[3];
    const long long* joff;   // per sphere offset of its J blocks (complex units)
    zd* Jsn;                 // node <- sphere: nbN x nb x 2
    zd* Jns;                 // sphere <- node: nb x nbN x 2
    double rimed_re, rimed_im;
    GtConst g;
};

struct FftHArgs {
    int cd[3], No, nnb;
    int nbv[27 * 3];
    double dcell;
    double rimed_re, rimed_im;
    zd* hr;                  // 2 nbN nbN x (8 cd^3): real-space kernels, single-precision values
    GtConst g;
};

struct FftMArgs {
    int nsph, No, nbmax;
    size_t N8;
    const int* order;
    const int* offset;
    const long long* joff;
    const int* slot;         // padded-grid slot of each sphere's cell
};

void launch_fft_j(const FftJArgs& a, cudaStream_t st);
void launch_fft_hbuild(const FftHArgs& a, int nsm, cudaStream_t st);
void launch_fft_round(size_t n, const zd* in, float2* out, cudaStream_t st);
template <typename T>
void launch_fft_s2n(const FftMArgs& a, const cpx<T>* J, const cpx<T>* x, int ld, int ncol, unsigned contran, cpx<T>* A, cudaStream_t st);
template <typename T> void launch_fft_mul(int nbN, size_t N8, int ncol, const float2* H, const cpx<T>* A, cpx<T>* G, int nsm, cudaStream_t st);
template <typename T>
void launch_fft_n2s(const FftMArgs& a, const cpx<T>* J, const cpx<T>* G, int ncol, unsigned contran, cpx<T>* y, int ld, cudaStream_t st);
