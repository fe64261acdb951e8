// warmstart.cu -- kernels of the learned warm start: a message-passing network
// over each sphere's k nearest neighbours that predicts the sphere's
// interaction correction to its isolated-sphere (Mie) solution, which becomes
// the BiCG initial guess in place of MSTM's Mie-solution start
// (fixedorsoln, mstm-solver-8.f90:482-483).  MSTM has no counterpart.
//
// Forward and backward passes are composed on the host from these primitives:
//   nn_gemm        C (+)= op(A) op(B), FP32 activations, weights in BF16 (or
//                  FP32 for the gradient check), FP32 accumulation: the
//                  activation products with BF16 weights on the tensor cores
//                  (tcgen05 kind::f16, activations as BF16 hi + lo), the
//                  rest (weight gradients, FP32 weights) in 64x64 CUDA-core
//                  tiles, split-K with FP32 atomics for the weight gradients
//   nn_bias_act    Y = act(Z + b) (identity or SiLU), keeps Z for backward
//   nn_act_back    dZ = dY * act'(Z)
//   nn_colsum      db = column sums of dZ
//   nn_edge_concat / nn_edge_concat_back   [h_dst, h_src, e] rows per edge
//   nn_scatter_add / nn_gather             message sum per node and its backward
//   nn_mse         masked mean-square loss and its gradient
//   nn_adam        Adam step on FP32 master weights + BF16 copy
//   nn_knn         k nearest neighbours per sphere (brute force per configuration)
#include "common.cuh"
#include <cuda_bf16.h>

#define NN_TM 64
#define NN_TN 64
#define NN_TK 16

namespace {
__device__ __forceinline__ float wload(const float* p) { return *p; }
__device__ __forceinline__ float wload(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_d(float z)
{
    float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}
}  // namespace

// C[M x N] (+)= op(A)[M x K] op(B)[K x N]; op(A)(i,k) = TA ? A[k lda + i] : A[i lda + k],
// op(B)(k,j) = TB ? B[j ldb + k] : B[k ldb + j].  Grid (N/64, M/64, splits of K).
template <bool TA, bool TB, typename TW>
__global__ void __launch_bounds__(256) nn_gemm_kernel(int M, int N, int K, const float* A, int lda, const TW* B, int ldb, float* C, int ldc,
                                                      int kchunk, int atomic)
{
    __shared__ float As[NN_TK][NN_TM + 4];
    __shared__ float Bs[NN_TK][NN_TN + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int i0 = blockIdx.y * NN_TM, j0 = blockIdx.x * NN_TN;
    const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0f;
    for (int k0 = kb; k0 < ke; k0 += NN_TK) {
        for (int e = threadIdx.x; e < NN_TK * NN_TM; e += 256) {
            int kk = e / NN_TM, ii = e % NN_TM;
            int i = i0 + ii, k = k0 + kk;
            float v = 0.0f;
            if (i < M && k < ke) v = TA ? A[(size_t)k * lda + i] : A[(size_t)i * lda + k];
            As[kk][ii] = v;
        }
        for (int e = threadIdx.x; e < NN_TK * NN_TN; e += 256) {
            int kk = e / NN_TN, jj = e % NN_TN;
            int j = j0 + jj, k = k0 + kk;
            float v = 0.0f;
            if (j < N && k < ke) v = TB ? wload(&B[(size_t)j * ldb + k]) : wload(&B[(size_t)k * ldb + j]);
            Bs[kk][jj] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < NN_TK; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                a[q] = As[kk][ty + 16 * q];
                b[q] = Bs[kk][tx + 16 * q];
            }
#pragma unroll
            for (int p = 0; p < 4; p++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[p][q] = fmaf(a[p], b[q], acc[p][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < 4; p++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int i = i0 + ty + 16 * p, j = j0 + tx + 16 * q;
            if (i < M && j < N) {
                float* c = &C[(size_t)i * ldc + j];
                if (atomic) atomicAdd(c, acc[p][q]);
                else *c = acc[p][q];
            }
        }
}

// ---------------------------------------------------------------------------
// The network's activation products on the tensor cores: C[M x N] (+)= A op(B)
// with A FP32 activations (row-major) split into BF16 hi + lo parts, B the
// BF16 weights, FP32 accumulation in tensor memory (tcgen05.mma kind::f16).
// One CTA per 128-row tile and up to 256 output columns (one accumulator in
// 256 tensor-memory columns); K in chunks of 16 staged by the CTA's threads into shared
// memory in the MMA's K-major layout (core matrices of 8 rows x 16 bytes),
// double-buffered: the next chunk is written while the MMAs of the current
// one run.  Every wait is bounded.
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ uint32_t nn_su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool nn_mb_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool nn_mb_wait(uint32_t bar, uint32_t parity)
{
    for (int it = 0; it < (1 << 22); ++it)
        if (nn_mb_try(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ uint64_t nn_sdesc(uint32_t saddr)
{
    // K-major, no swizzle: LBO 128 bytes (the two core matrices of a K step), SBO 256 bytes (8-row groups)
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) | (1ull << 46);
}
// kind::f16 with BF16 A and B, FP32 D, both K-major, M = 128
__device__ __forceinline__ uint32_t nn_idesc(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ int nn_off(int r, int k) { return (r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2; }
}  // namespace

#define NN_TC_MAXN 256
template <bool TB>
__global__ void __launch_bounds__(128) nn_gemm_tc_kernel(int M, int N, int K, const float* A, int lda, const __nv_bfloat16* B, int ldb,
                                                         float* C, int ldc, int accumulate, int* err)
{
    // per buffer: A hi, A lo (128 x 16 BF16 = 4 KB each), B (up to 256 x 16 BF16 = 8 KB)
    __shared__ __align__(1024) unsigned char sbuf[2][8192 + 8192];
    __shared__ __align__(8) uint64_t bars[3];
    __shared__ uint32_t tmem_holder;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * NN_TC_MAXN;
    const int ncols = min(NN_TC_MAXN, N - n0);
    const int npad = (ncols + 15) / 16 * 16;
    const int nseg = (npad + 255) / 256;
    if (tid == 0) {
        for (int b = 0; b < 3; b++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(nn_su32(&bars[b])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(nn_su32(&tmem_holder)), "r"(256));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = tmem_holder;
    const int nk = (K + 15) / 16;
    bool ok = true;
    for (int kc = 0; kc < nk; kc++) {
        const int b = kc & 1;
        // the MMAs that read this buffer two chunks ago are done
        if (kc >= 2 && !nn_mb_wait(nn_su32(&bars[b]), (uint32_t)(((kc - 2) >> 1) & 1))) ok = false;
        unsigned char* ah = sbuf[b];
        unsigned char* al = sbuf[b] + 4096;
        unsigned char* bs = sbuf[b] + 8192;
        const int k0 = kc * 16;
        for (int e = tid; e < 128 * 16; e += 128) {
            const int r = e >> 4, k = e & 15;
            float v = 0.0f;
            if (m0 + r < M && k0 + k < K) v = A[(size_t)(m0 + r) * lda + k0 + k];
            const __nv_bfloat16 hi = __float2bfloat16_rn(v);
            const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
            *reinterpret_cast<__nv_bfloat16*>(ah + nn_off(r, k)) = hi;
            *reinterpret_cast<__nv_bfloat16*>(al + nn_off(r, k)) = lo;
        }
        for (int e = tid; e < npad * 16; e += 128) {
            const int nn = e >> 4, k = e & 15;
            __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
            const int j = n0 + nn, kk = k0 + k;
            if (nn < ncols && kk < K) v = TB ? B[(size_t)j * ldb + kk] : B[(size_t)kk * ldb + j];
            *reinterpret_cast<__nv_bfloat16*>(bs + nn_off(nn, k)) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic writes -> the tensor cores' reads
        __syncthreads();
        if (tid == 0 && ok) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int sg = 0; sg < nseg; sg++) {
                const int nw = min(256, npad - sg * 256);
                const uint32_t d = tbase + (uint32_t)(sg * 256);
                const uint64_t bd = nn_sdesc(nn_su32(bs) + (uint32_t)(sg * 256 / 8) * 256u);
                const uint32_t idesc = nn_idesc(nw), acc0 = kc > 0 ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d),
                    "l"(nn_sdesc(nn_su32(ah))), "l"(bd), "r"(idesc), "r"(acc0), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d),
                    "l"(nn_sdesc(nn_su32(al))), "l"(bd), "r"(idesc), "r"(1u), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(nn_su32(&bars[b])) : "memory");
        }
    }
    // all MMAs done: the last commit covers every earlier one of this thread
    if (tid == 0 && ok) asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(nn_su32(&bars[2])) : "memory");
    if (!(ok && nn_mb_wait(nn_su32(&bars[2]), 0u))) ok = false;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        const int r = warp * 32 + lane;
        for (int c0 = 0; c0 < npad; c0 += 16) {
            uint32_t v[16];
            const uint32_t ta = tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)((c0 / 256) * 256 + c0 % 256);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]),
                  "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(ta));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m0 + r < M) {
                float* c = C + (size_t)(m0 + r) * ldc + n0;
#pragma unroll
                for (int q = 0; q < 16; q++)
                    if (c0 + q < ncols) c[c0 + q] = (accumulate ? c[c0 + q] : 0.0f) + __uint_as_float(v[q]);
            }
        }
    } else if (tid == 0) {
        atomicExch(err, MSTMG_ERR_CUDA);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(256));
}

__global__ void nn_bias_act_kernel(int M, int N, const float* Z, const float* b, float* Y, int act)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)M * N; e += (size_t)gridDim.x * blockDim.x) {
        float z = Z[e] + (b ? b[e % N] : 0.0f);
        Y[e] = act ? silu(z) : z;
    }
}
// dZ = dY * act'(Z + b)
__global__ void nn_act_back_kernel(int M, int N, const float* Z, const float* b, const float* dY, float* dZ, int act)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)M * N; e += (size_t)gridDim.x * blockDim.x) {
        float z = Z[e] + (b ? b[e % N] : 0.0f);
        dZ[e] = act ? dY[e] * silu_d(z) : dY[e];
    }
}
// db[j] = sum_i dZ[i, j] (fixed order per column)
__global__ void nn_colsum_kernel(int M, int N, const float* dZ, float* db)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    float s = 0.0f;
    for (int i = 0; i < M; i++) s += dZ[(size_t)i * N + j];
    db[j] = s;
}
// Z[e] = [h[dst[e]], h[src[e]], ef[e]]  (H hidden, F edge features)
__global__ void nn_edge_concat_kernel(int E, int H, int F, const int* dst, const int* src, const float* h, const float* ef, float* Z)
{
    const int W = 2 * H + F;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)E * W; t += (size_t)gridDim.x * blockDim.x) {
        int e = (int)(t / W), c = (int)(t % W);
        float v;
        if (c < H) v = h[(size_t)dst[e] * H + c];
        else if (c < 2 * H) v = h[(size_t)src[e] * H + c - H];
        else v = ef[(size_t)e * F + c - 2 * H];
        Z[t] = v;
    }
}
__global__ void nn_edge_concat_back_kernel(int E, int H, int F, const int* dst, const int* src, const float* dZ, float* dh)
{
    const int W = 2 * H + F;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)E * 2 * H; t += (size_t)gridDim.x * blockDim.x) {
        int e = (int)(t / (2 * H)), c = (int)(t % (2 * H));
        float g = dZ[(size_t)e * W + c];
        if (c < H) atomicAdd(&dh[(size_t)dst[e] * H + c], g);
        else atomicAdd(&dh[(size_t)src[e] * H + c - H], g);
    }
}
// out[dst[e]] += in[e]  (rows of width H)
__global__ void nn_scatter_add_kernel(int E, int H, const int* dst, const float* in, float* out)
{
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)E * H; t += (size_t)gridDim.x * blockDim.x) {
        int e = (int)(t / H), c = (int)(t % H);
        atomicAdd(&out[(size_t)dst[e] * H + c], in[t]);
    }
}
// out[e] = in[idx[e]]  (rows of width H), optionally accumulated
__global__ void nn_gather_kernel(int E, int H, const int* idx, const float* in, float* out, int accumulate)
{
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)E * H; t += (size_t)gridDim.x * blockDim.x) {
        int e = (int)(t / H), c = (int)(t % H);
        float v = in[(size_t)idx[e] * H + c];
        out[t] = accumulate ? out[t] + v : v;
    }
}
// loss = sum mask (y - t)^2 / sum mask ; dy = 2 mask (y - t) / sum mask
__global__ void nn_mse_kernel(size_t n, const float* y, const float* t, const float* mask, float msum, float* dy, double* loss)
{
    double s = 0.0;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        float d = (y[e] - t[e]) * mask[e];
        dy[e] = 2.0f * d / msum;
        s += (double)d * d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s / msum);
}
__global__ void nn_adam_kernel(size_t n, float* p, const float* g, float* m, float* v, __nv_bfloat16* pb, float lr, float b1, float b2, float eps,
                               float c1, float c2)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        float gg = g[e];
        float mm = b1 * m[e] + (1.0f - b1) * gg;
        float vv = b2 * v[e] + (1.0f - b2) * gg * gg;
        m[e] = mm;
        v[e] = vv;
        float upd = lr * (mm / c1) / (sqrtf(vv / c2) + eps);
        float np = p[e] - upd;
        p[e] = np;
        if (pb) pb[e] = __float2bfloat16(np);
    }
}
__global__ void nn_axpy_kernel(size_t n, float a, const float* x, float* y)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) y[e] = y[e] + a * x[e];
}
__global__ void nn_to_bf16_kernel(size_t n, const float* p, __nv_bfloat16* pb)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) pb[e] = __float2bfloat16(p[e]);
}
// k nearest neighbours of every sphere within its configuration (brute force;
// ties broken by index).  cfg_start[c]..cfg_start[c+1]: spheres of config c;
// sphere_cfg[i]: its configuration.  nbr[i k + q], q < k (fewer spheres: -1).
__global__ void nn_knn_kernel(int n, int k, const int* cfg_start, const int* sphere_cfg, const double* pos, int* nbr)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = sphere_cfg[i], s0 = cfg_start[c], s1 = cfg_start[c + 1];
    double bd[32];
    int bi[32];
    int cnt = 0;
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    for (int j = s0; j < s1; j++) {
        if (j == i) continue;
        double dx = pos[3 * j] - xi, dy = pos[3 * j + 1] - yi, dz = pos[3 * j + 2] - zi;
        double d = dx * dx + dy * dy + dz * dz;
        if (cnt < k) {
            int q = cnt++;
            while (q > 0 && (bd[q - 1] > d)) { bd[q] = bd[q - 1]; bi[q] = bi[q - 1]; q--; }
            bd[q] = d;
            bi[q] = j;
        } else if (d < bd[k - 1]) {
            int q = k - 1;
            while (q > 0 && (bd[q - 1] > d)) { bd[q] = bd[q - 1]; bi[q] = bi[q - 1]; q--; }
            bd[q] = d;
            bi[q] = j;
        }
    }
    for (int q = 0; q < k; q++) nbr[(size_t)i * k + q] = q < cnt ? bi[q] : -1;
}

// ---------------------------------------------------------------------------
// C ABI (device pointers, the caller's stream)
// ---------------------------------------------------------------------------
static int grid1(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 32); }

static int* nn_err_flag()
{
    static int* p = nullptr;   // device status word of the tensor-core products (set on a wait that gave up)
    if (!p && cudaMalloc((void**)&p, sizeof(int)) == cudaSuccess) cudaMemset(p, 0, sizeof(int));
    return p;
}

extern "C" int mstmg_nn_gemm(int M, int N, int K, const float* A, int lda, int transA, const void* B, int ldb, int transB, int b_bf16,
                             float* C, int ldc, int accumulate, void* stream)
{
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return MSTMG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    // activation products with BF16 weights: the tensor cores
    if (b_bf16 && !transA && nn_err_flag()) {
        dim3 grid((M + 127) / 128, (N + NN_TC_MAXN - 1) / NN_TC_MAXN);
        const __nv_bfloat16* Bw = (const __nv_bfloat16*)B;
        if (transB) nn_gemm_tc_kernel<true><<<grid, 128, 0, st>>>(M, N, K, A, lda, Bw, ldb, C, ldc, accumulate, nn_err_flag());
        else nn_gemm_tc_kernel<false><<<grid, 128, 0, st>>>(M, N, K, A, lda, Bw, ldb, C, ldc, accumulate, nn_err_flag());
        launch_counter() += 1;
        return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
    }
    dim3 grid((N + NN_TN - 1) / NN_TN, (M + NN_TM - 1) / NN_TM, 1);
    int tiles = grid.x * grid.y;
    int splits = 1;
    // long reductions (weight gradients) split K across CTAs, summed with atomics
    if (tiles < 148 && K > 1024) splits = std::min((K + 511) / 512, (148 * 2 + tiles - 1) / tiles);
    int kchunk = ((K + splits - 1) / splits + NN_TK - 1) / NN_TK * NN_TK;
    splits = (K + kchunk - 1) / kchunk;
    grid.z = splits;
    int atomic = (splits > 1 || accumulate) ? 1 : 0;
    if (atomic && !accumulate) cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * ldc, st);
#define NN_LAUNCH(TA, TB, TW) nn_gemm_kernel<TA, TB, TW><<<grid, 256, 0, st>>>(M, N, K, A, lda, (const TW*)B, ldb, C, ldc, kchunk, atomic)
    if (b_bf16) {
        if (!transA && !transB) NN_LAUNCH(false, false, __nv_bfloat16);
        else if (!transA && transB) NN_LAUNCH(false, true, __nv_bfloat16);
        else if (transA && !transB) NN_LAUNCH(true, false, __nv_bfloat16);
        else NN_LAUNCH(true, true, __nv_bfloat16);
    } else {
        if (!transA && !transB) NN_LAUNCH(false, false, float);
        else if (!transA && transB) NN_LAUNCH(false, true, float);
        else if (transA && !transB) NN_LAUNCH(true, false, float);
        else NN_LAUNCH(true, true, float);
    }
#undef NN_LAUNCH
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}

extern "C" int mstmg_nn_bias_act(int M, int N, const float* Z, const float* b, float* Y, int act, void* stream)
{
    nn_bias_act_kernel<<<grid1((size_t)M * N), 256, 0, (cudaStream_t)stream>>>(M, N, Z, b, Y, act);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_act_back(int M, int N, const float* Z, const float* b, const float* dY, float* dZ, int act, void* stream)
{
    nn_act_back_kernel<<<grid1((size_t)M * N), 256, 0, (cudaStream_t)stream>>>(M, N, Z, b, dY, dZ, act);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_colsum(int M, int N, const float* dZ, float* db, void* stream)
{
    nn_colsum_kernel<<<(N + 127) / 128, 128, 0, (cudaStream_t)stream>>>(M, N, dZ, db);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_edge_concat(int E, int H, int F, const int* dst, const int* src, const float* h, const float* ef, float* Z, void* stream)
{
    nn_edge_concat_kernel<<<grid1((size_t)E * (2 * H + F)), 256, 0, (cudaStream_t)stream>>>(E, H, F, dst, src, h, ef, Z);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_edge_concat_back(int E, int H, int F, const int* dst, const int* src, const float* dZ, float* dh, void* stream)
{
    nn_edge_concat_back_kernel<<<grid1((size_t)E * 2 * H), 256, 0, (cudaStream_t)stream>>>(E, H, F, dst, src, dZ, dh);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_scatter_add(int E, int H, const int* dst, const float* in, float* out, void* stream)
{
    nn_scatter_add_kernel<<<grid1((size_t)E * H), 256, 0, (cudaStream_t)stream>>>(E, H, dst, in, out);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_gather(int E, int H, const int* idx, const float* in, float* out, int accumulate, void* stream)
{
    nn_gather_kernel<<<grid1((size_t)E * H), 256, 0, (cudaStream_t)stream>>>(E, H, idx, in, out, accumulate);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_mse(long long n, const float* y, const float* t, const float* mask, float msum, float* dy, double* loss, void* stream)
{
    cudaMemsetAsync(loss, 0, sizeof(double), (cudaStream_t)stream);
    nn_mse_kernel<<<grid1((size_t)n), 256, 0, (cudaStream_t)stream>>>((size_t)n, y, t, mask, msum, dy, loss);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_adam(long long n, float* p, const float* g, float* m, float* v, void* pb, float lr, float b1, float b2, float eps, int step,
                             void* stream)
{
    float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    nn_adam_kernel<<<grid1((size_t)n), 256, 0, (cudaStream_t)stream>>>((size_t)n, p, g, m, v, (__nv_bfloat16*)pb, lr, b1, b2, eps, c1, c2);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_to_bf16(long long n, const float* p, void* pb, void* stream)
{
    nn_to_bf16_kernel<<<grid1((size_t)n), 256, 0, (cudaStream_t)stream>>>((size_t)n, p, (__nv_bfloat16*)pb);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_axpy(long long n, float a, const float* x, float* y, void* stream)
{
    nn_axpy_kernel<<<grid1((size_t)n), 256, 0, (cudaStream_t)stream>>>((size_t)n, a, x, y);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
extern "C" int mstmg_nn_knn(int n, int k, const int* cfg_start, const int* sphere_cfg, const double* pos, int* nbr, void* stream)
{
    if (k < 1 || k > 32) return MSTMG_ERR_ARG;
    nn_knn_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(n, k, cfg_start, sphere_cfg, pos, nbr);
    launch_counter() += 1;
    return cudaGetLastError() == cudaSuccess ? MSTMG_OK : MSTMG_ERR_CUDA;
}
