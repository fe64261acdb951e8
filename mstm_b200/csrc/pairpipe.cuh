// pairpipe.cuh -- device helpers shared by the pair translation kernels:
// mbarrier waits and bulk copies (cp.async.bulk), vector atomics into y,
// complex multiply-accumulates on the packed FP32x2 FMA, and the index of
// a(m, n) inside one mode of a sphere block.
#pragma once
#include "common.cuh"

namespace pairpipe {

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mb_init(uint64_t* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mb_expect(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(su32(dst)),
                 "l"(src), "r"(bytes), "r"(su32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mb_try(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(su32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// bounded wait: gives up after `limit` polls (the kernels then record
// MSTMG_ERR_CUDA and return instead of hanging)
__device__ __forceinline__ bool mb_wait(uint64_t* bar, uint32_t parity, int limit = 1 << 22)
{
    for (int it = 0; it < limit; ++it)
        if (mb_try(bar, parity)) return true;
    return false;
}

template <typename T> __device__ __forceinline__ void red_add(cpx<T>* p, cpx<T> v);
template <> __device__ __forceinline__ void red_add<float>(cpx<float>* p, cpx<float> v)
{
    atomicAdd(reinterpret_cast<float2*>(p), make_float2(v.x, v.y));
}
template <> __device__ __forceinline__ void red_add<double>(cpx<double>* p, cpx<double> v)
{
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
}

// Multiply-accumulates of the passes: acc + r v (real r) and acc + z v
// (complex z).  FP32 values go through the packed two-lane FMA of sm_100
// (one instruction for both halves of a complex number); FP64 through
// scalar FMAs.
template <typename T> __device__ __forceinline__ cpx<T> mac_r(cpx<T> acc, T r, cpx<T> v)
{
    return mk(fma(r, v.x, acc.x), fma(r, v.y, acc.y));
}
template <> __device__ __forceinline__ cpx<float> mac_r<float>(cpx<float> acc, float r, cpx<float> v)
{
    const float2 o = __ffma2_rn(make_float2(r, r), make_float2(v.x, v.y), make_float2(acc.x, acc.y));
    return mk(o.x, o.y);
}
template <typename T> __device__ __forceinline__ cpx<T> mac_c(cpx<T> acc, cpx<T> z, cpx<T> v)
{
    return mk(fma(z.x, v.x, fma(-z.y, v.y, acc.x)), fma(z.x, v.y, fma(z.y, v.x, acc.y)));
}
template <> __device__ __forceinline__ cpx<float> mac_c<float>(cpx<float> acc, cpx<float> z, cpx<float> v)
{
    float2 o = __ffma2_rn(make_float2(-z.y, z.y), make_float2(v.y, v.x), make_float2(acc.x, acc.y));
    o = __ffma2_rn(make_float2(z.x, z.x), make_float2(v.x, v.y), o);
    return mk(o.x, o.y);
}

// half-block (one mode) slot of degree m, order n: MSTM's a(0:L+1,1:L) index
template <int L> __host__ __device__ constexpr int hidx(int m, int n) { return m >= 0 ? m + (L + 2) * (n - 1) : (n + 1) + (L + 2) * (-m - 1); }

}  // namespace pairpipe
