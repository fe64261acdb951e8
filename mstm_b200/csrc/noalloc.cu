// noalloc.cu -- incident plane-wave coefficients without any device allocation.
//
// Some callers cannot call cudaMalloc: a Fortran code that hands this library
// memory it manages itself and forbids allocations behind its back, a host
// application that runs under a fixed device-memory budget, or code that must
// not allocate in the middle of its own stream work.  For them
// mstmg_planewave_noalloc computes the same coefficients as mstmg_planewave
// (no context, no cudaMalloc): the caller passes device input and output
// buffers, and the two small intermediate tables live in the file-scope
// device array below.
//
// The array is a fixed, modest size (enough for sphere order MSTMG_LMAX = 16,
// about 32 KB) and every GPU that loads the library holds it until the
// process exits.  Its device address is looked up with cudaGetSymbolAddress
// on every call made outside stream capture, with the calling thread's
// current device and context (a context that was destroyed and made again
// may load the module at another address); a call made while its stream is
// being captured reuses the address the last uncaptured call on that device
// found, so the first call on each device must come before any stream
// capture.  All calls share the array: each call rewrites every entry it
// reads, but calls that overlap on the GPU (different streams, or host
// threads on one device) race on it and must be serialised by the caller.
// The incident field is the free-space one (medium refractive index 1).
#include <mutex>
#include <string>
#include "../../include/mstm_b200.h"
#include "common.cuh"
#include "sphere_kernels.cuh"

#define NOALLOC_PW0 (2 * 2 * MSTMG_LMAX * (MSTMG_LMAX + 2))       // pw0: nb(L) x 2 polarisations
#define NOALLOC_DROT (3 * (MSTMG_LMAX * (MSTMG_LMAX + 2) + 1))    // Wigner-d table with |m| <= 1

static __device__ __align__(256) zd g_pw_scratch[NOALLOC_PW0 + NOALLOC_DROT];

namespace {
std::mutex g_mu;
zd* g_scratch_ptr[64] = {nullptr};
}
void mstmg_internal_set_error(const std::string& msg);   // message for mstmg_last_error (capi.cu)

__global__ void planewave_common_kernel(double alpha, zd cb, int nodr, zd* pw0, zd* drot);

// Per-sphere phase for spheres that all have order L (layerplanewavecoef without
// plane boundaries, december2023/mstm-modules-33.f90:3901-3965).
__global__ void planewave_phase_uniform_kernel(int nsph, int L, const double* pos, const zd* pw0, zd cbinc, zd riinc, double sinc,
                                               double alpha, zd* pmnp)
{
    const int nb = 2 * L * (L + 2), hb = L * (L + 2);
    const long long ne = (long long)nsph * nb;
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int i = (int)(e / nb), loc = (int)(e - (long long)i * nb);
    int p = loc / hb, rem = loc - p * hb;
    int row = rem % (L + 2), col = rem / (L + 2) + 1;
    int m, n;
    if (row <= col) { m = row; n = col; } else { n = row - 1; m = -col; }
    zd phz = cexpd(imul(riinc * cbinc * mk(pos[3 * i + 2] - 0.0, 0.0)));
    zd phl = cexpd(imul(mk(sinc * (cos(alpha) * pos[3 * i] + sin(alpha) * pos[3 * i + 1]), 0.0)));
    int src = aidx(m, n, p, L);
    for (int k = 0; k < 2; k++) pmnp[(size_t)k * ne + e] = (pw0[(size_t)k * nb + src] * phz) * phl;
}

// Memory the kernels on device `dev` can use directly: device memory of
// that device, or managed memory.
static bool dev_ptr(const void* p, int dev)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

extern "C" int mstmg_planewave_noalloc(int nsphere, int order, const double* pos, double alpha, double sinc, int dir,
                                       double* pmnp, void* stream)
{
    if (nsphere < 1 || order < 1 || !pos || !pmnp || (dir != 1 && dir != 2)) {
        mstmg_internal_set_error("mstmg_planewave_noalloc: bad arguments");
        return MSTMG_ERR_ARG;
    }
    if (order > MSTMG_LMAX) {
        mstmg_internal_set_error("mstmg_planewave_noalloc: sphere order " + std::to_string(order) + " exceeds the built-in scratch limit " +
                        std::to_string(MSTMG_LMAX));
        return MSTMG_ERR_UNSUPPORTED;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        mstmg_internal_set_error("mstmg_planewave_noalloc: no usable CUDA device");
        return MSTMG_ERR_CUDA;
    }
    if (!dev_ptr(pos, dev) || !dev_ptr(pmnp, dev)) {
        mstmg_internal_set_error("mstmg_planewave_noalloc: pos and pmnp must be device memory of the current device");
        return MSTMG_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) {
        mstmg_internal_set_error(std::string("mstmg_planewave_noalloc: cudaStreamIsCapturing: ") + cudaGetErrorString(e));
        return MSTMG_ERR_CUDA;
    }
    zd* scratch;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (cap == cudaStreamCaptureStatusNone) {
            // the address in the current context (looked up every time: the
            // context may have been destroyed and created again since)
            zd* ptr = nullptr;
            e = cudaGetSymbolAddress((void**)&ptr, g_pw_scratch);
            if (e != cudaSuccess || !ptr) {
                mstmg_internal_set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return MSTMG_ERR_CUDA;
            }
            g_scratch_ptr[dev] = ptr;
        } else if (!g_scratch_ptr[dev]) {
            mstmg_internal_set_error("mstmg_planewave_noalloc: the first call on a device must come before stream capture");
            return MSTMG_ERR_ARG;
        }
        scratch = g_scratch_ptr[dev];
    }
    zd riinc = mk(1.0, 0.0);
    zd a = cdiv(mk(sinc, 0.0), riinc);
    zd cbinc = csqrtd((mk(1.0, 0.0) - a) * (mk(1.0, 0.0) + a)) * (double)(3 - 2 * dir);
    zd* pw0 = scratch;
    zd* drot = scratch + NOALLOC_PW0;
    planewave_common_kernel<<<1, 32, 0, st>>>(alpha, cbinc, order, pw0, drot);
    long long ne = (long long)nsphere * 2 * order * (order + 2);
    planewave_phase_uniform_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(nsphere, order, pos, pw0, cbinc, riinc, sinc, alpha,
                                                                                  (zd*)pmnp);
    launch_counter() += 2;
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        mstmg_internal_set_error(std::string("mstmg_planewave_noalloc launch: ") + cudaGetErrorString(e));
        return MSTMG_ERR_CUDA;
    }
    return MSTMG_OK;
}
