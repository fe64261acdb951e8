// common.cuh -- shared device helpers for the MSTM B200 kernels.
//
// Complex values are stored interleaved (re, im) exactly like Fortran
// complex(8) / C double _Complex, so vectors cross the C ABI without copies.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>

// Count of kernels launched by this library (all contexts, all threads).
inline std::atomic<long long>& launch_counter()
{
    static std::atomic<long long> n{0};
    return n;
}

#define MSTMG_LMAX 16          // largest sphere truncation order the kernels accept

// pi as MSTM stores it: a default-real literal assigned to real(8)
// (december2023/mstm-modules-33.f90:18).  Used wherever the reference uses pi.
#define MSTMG_REF_PI 3.1415927410125732

template <typename T> struct cpx { T x, y; };
typedef cpx<double> zd;
typedef cpx<float> zf;

template <typename T> __host__ __device__ __forceinline__ cpx<T> mk(T a, T b) { cpx<T> r; r.x = a; r.y = b; return r; }
template <typename T> __host__ __device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) { return mk(a.x + b.x, a.y + b.y); }
template <typename T> __host__ __device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) { return mk(a.x - b.x, a.y - b.y); }
template <typename T> __host__ __device__ __forceinline__ cpx<T> operator-(cpx<T> a) { return mk(-a.x, -a.y); }
template <typename T> __host__ __device__ __forceinline__ cpx<T> operator*(cpx<T> a, cpx<T> b) { return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename T> __host__ __device__ __forceinline__ cpx<T> operator*(T s, cpx<T> a) { return mk(s * a.x, s * a.y); }
template <typename T> __host__ __device__ __forceinline__ cpx<T> operator*(cpx<T> a, T s) { return mk(s * a.x, s * a.y); }
template <typename T> __host__ __device__ __forceinline__ cpx<T> cj(cpx<T> a) { return mk(a.x, -a.y); }
template <typename T> __host__ __device__ __forceinline__ T cabs2(cpx<T> a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ double cabsd(zd a) { return hypot(a.x, a.y); }
// i * a
template <typename T> __host__ __device__ __forceinline__ cpx<T> imul(cpx<T> a) { return mk(-a.y, a.x); }
// a / b with scaling (Smith's method), full FP64 range
__host__ __device__ inline zd cdiv(zd a, zd b)
{
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return mk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.x * r + b.y;
        return mk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}
__host__ __device__ inline zd cdivr(double a, zd b) { return cdiv(mk(a, 0.0), b); }
__host__ __device__ inline zd cexpd(zd z) { double e = exp(z.x); return mk(e * cos(z.y), e * sin(z.y)); }
__host__ __device__ inline zd csind(zd z) { return mk(sin(z.x) * cosh(z.y), cos(z.x) * sinh(z.y)); }
__host__ __device__ inline zd ccosd(zd z) { return mk(cos(z.x) * cosh(z.y), -sin(z.x) * sinh(z.y)); }
__host__ __device__ inline zd csqrtd(zd z)
{
    double m = hypot(z.x, z.y);
    if (m == 0.0) return mk(0.0, 0.0);
    if (z.x >= 0.0) { double t = sqrt(0.5 * (m + z.x)); return mk(t, z.y / (2.0 * t)); }
    double t = sqrt(0.5 * (m - z.x));
    return mk(fabs(z.y) / (2.0 * t), z.y >= 0.0 ? t : -t);
}

__host__ __device__ __forceinline__ double pm1(int n) { return (n & 1) ? -1.0 : 1.0; }

// Index of a(m,n,p) inside a sphere block of order L (Fortran a(0:L+1,1:L,1:2),
// m>=0 at row m of column n, m<0 at row n+1 of column -m; p in {0,1}).
__host__ __device__ __forceinline__ int aidx(int m, int n, int p, int L)
{
    return (m >= 0) ? (m + (L + 2) * (n - 1) + (L + 2) * L * p) : ((n + 1) + (L + 2) * (-m - 1) + (L + 2) * L * p);
}

// Status codes shared by the C ABI.
#define MSTMG_OK 0
#define MSTMG_NOT_CONVERGED 1
#define MSTMG_ERR_ARG (-1)
#define MSTMG_ERR_CUDA (-2)
#define MSTMG_ERR_UNSUPPORTED (-3)
#define MSTMG_ERR_BREAKDOWN (-4)
