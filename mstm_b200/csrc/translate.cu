// translate.cu -- the sphere-pair translation matvec (the hot loop of MSTM's
// external_to_external_expansion, december2023/mstm-modules-33.f90:6390-6525,
// applying coefficient_translation, modules:6610-6787, in both directions).
//
// One CTA streams one pair operator record at a time into shared memory with a
// 1-D bulk TMA copy (cp.async.bulk, mbarrier completion), double buffered, and
// applies it to every right-hand side in both directions:
//   j -> i  (shift_op = F): y_i += T_ij x_j
//   i -> j  (shift_op = T): y_j += T_ji x_i, from the same record
// Each application is phase(e^{+-i m phi}) -> rotate (Wigner-d, folded E/O form)
// -> axial translate per degree m -> rotate back -> phase back, with the
// (-1)^m / m<->-m shift of shiftcoefficient (modules:6789-6820) for
// reverse and conjugate-transpose products.  Outputs are accumulated with
// atomics into y (kept L2 resident).
#include "common.cuh"
#include "kernels.cuh"

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after a fixed number of polls (each poll already
// suspends for a hardware-chosen time) and reports failure.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

template <typename T> __device__ __forceinline__ void atomic_add_c(cpx<T>* p, cpx<T> v)
{
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
}

template <typename T> __device__ __forceinline__ cpx<T> ldc(const cpx<T>* p) { return *p; }

// LM: the largest order among the launch's pairs, a compile-time constant so
// that the index decodes of every phase are multiplications, not divisions;
// UNI: every pair has both orders LM (the order tests fold away)
template <typename T, int NT, int LM, bool UNI> __global__ void __launch_bounds__(NT) translate_kernel(TransArgs<T> a)
{
    extern __shared__ __align__(128) unsigned char sm[];
    const int tid = threadIdx.x;
    constexpr int lm = LM;
    const int nrhs = a.nrhs;
    const int NI = 2 * nrhs;
    uint64_t* bar = (uint64_t*)sm;                              // 2 barriers
    int* roff = (int*)(sm + 16);                                // lm+2 ints
    int* zoff = roff + (MSTMG_LMAX + 2);                        // lm+2 ints
    int* flag = zoff + (MSTMG_LMAX + 2);                        // 1 int
    cpx<T>* ephm = (cpx<T>*)(sm + 256);                         // 2*LMAX+1 entries, index q+LMAX
    T* opb = (T*)(sm + 256 + 2 * sizeof(cpx<T>) * (2 * MSTMG_LMAX + 1) + 64);
    opb = (T*)(((uintptr_t)opb + 127) & ~(uintptr_t)127);
    cpx<T>* bufA = (cpx<T>*)(opb + 2 * (size_t)a.maxrec);       // s/t, later g
    const int szA = lm * 2 * (lm + 1);                          // per (inst, p)
    cpx<T>* bufB = bufA + (size_t)NI * 2 * szA;                 // a'
    const int szB = lm * (2 * lm + 1);

    const int G = gridDim.x;
    int q0 = blockIdx.x;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *flag = 0;
    }
    __syncthreads();
    if (tid == 0) {
        for (int b = 0; b < 2; b++) {
            int q = q0 + b * G;
            if (q < a.npairs) {
                int i = a.pairs[q].x, j = a.pairs[q].y;
                uint32_t bytes = (uint32_t)(op_record_units(a.order[i], a.order[j]) * sizeof(T));
                mbar_arrive_expect_tx(&bar[b], bytes);
                bulk_g2s(opb + (size_t)b * a.maxrec, a.ops + a.opoff[q], bytes, &bar[b]);
            }
        }
    }
    int prev_noi = -1, prev_noj = -1;
    int t = 0;
    for (int q = q0; q < a.npairs; q += G, ++t) {
        const int b = t & 1;
        const uint32_t parity = (t >> 1) & 1;
        if (!mbar_wait_bounded(&bar[b], parity)) {
            if (tid == 0) atomicExch(a.err, MSTMG_ERR_CUDA);
            // wait (bounded) for the other buffer's copy in flight, then leave
            mbar_wait_bounded(&bar[b ^ 1], ((t + 1) >> 1) & 1);
            return;
        }
        const T* rec = opb + (size_t)b * a.maxrec;
        const int i = a.pairs[q].x, j = a.pairs[q].y;
        const int noi = UNI ? LM : a.order[i], noj = UNI ? LM : a.order[j];
        const int nmin = noi < noj ? noi : noj, nmax = noi > noj ? noi : noj;
        if (noi != prev_noi || noj != prev_noj) {
            if (tid <= lm + 1) {
                roff[tid] = (tid >= 1 && tid <= nmax) ? 2 + op_rot_offset(tid, nmin) : 0;
                zoff[tid] = (tid <= nmin) ? 2 + op_rot_size(nmax, nmin) + 2 * op_z_offset(tid, noi, noj) : 0;
            }
            prev_noi = noi;
            prev_noj = noj;
        }
        if (tid == 0) {
            cpx<T> ep = mk(rec[0], rec[1]);
            cpx<T>* e = ephm + MSTMG_LMAX;
            e[0] = mk((T)1, (T)0);
            for (int m = 1; m <= nmax; m++) {
                e[m] = ep * e[m - 1];
                e[-m] = cj(e[m]);
            }
        }
        __syncthreads();
        const cpx<T>* e = ephm + MSTMG_LMAX;

        // ---- phase 1: shift, phase, even/odd split of each source block ----
        for (int idx = tid; idx < NI * 2 * lm * (lm + 1); idx += NT) {
            int m = idx % (lm + 1);
            int rest = idx / (lm + 1);
            int n = rest % lm + 1;
            rest /= lm;
            int p = rest & 1, inst = rest >> 1;
            int dir = inst / nrhs, r = inst % nrhs;
            int src = dir ? i : j, nsrc = dir ? noi : noj;
            if (n > nsrc || m > n) continue;
            int sop = dir, top = (a.contran >> r) & 1;
            int im = sop ? -1 : 1;
            const cpx<T>* xs = a.x + (size_t)r * a.ld + a.offset[src];
            cpx<T> u = xs[aidx(m, n, p, nsrc)];
            cpx<T> v = (m == 0) ? u : xs[aidx(-m, n, p, nsrc)];
            T sg = (m & 1) ? (T)-1 : (T)1;
            if (sop != top && m > 0) { cpx<T> tt = u; u = sg * v; v = sg * tt; }
            cpx<T>* st = bufA + (size_t)(inst * 2 + p) * szA + (n - 1) * 2 * (lm + 1);
            if (m == 0) {
                st[0] = (T)2 * u;
                st[lm + 1] = mk((T)0, (T)0);
            } else {
                cpx<T> uu = u * e[im * m], vv = v * e[-im * m];
                st[m] = uu + sg * vv;
                st[lm + 1 + m] = uu - sg * vv;
            }
        }
        __syncthreads();

        // ---- phase 2: forward rotation per degree n (folded Wigner-d) ----
        for (int idx = tid; idx < NI * 2 * lm * (lm + 1); idx += NT) {
            int k = idx % (lm + 1);
            int rest = idx / (lm + 1);
            int n = rest % lm + 1;
            rest /= lm;
            int p = rest & 1, inst = rest >> 1;
            int dir = inst / nrhs;
            int nsrc = dir ? noi : noj;
            int kk = n < nmin ? n : nmin;
            if (n > nsrc || k > kk) continue;
            const T* E = rec + roff[n];
            const T* O = E + (kk + 1) * (n + 1);
            const cpx<T>* st = bufA + (size_t)(inst * 2 + p) * szA + (n - 1) * 2 * (lm + 1);
            cpx<T> P = mk((T)0, (T)0), Q = mk((T)0, (T)0);
            const T* Er = E + k * (n + 1);
            for (int m = 0; m <= n; m++) P = P + Er[m] * st[m];
            if (k > 0) {
                const T* Or = O + (k - 1) * n;
                for (int m = 1; m <= n; m++) Q = Q + Or[m - 1] * st[lm + 1 + m];
            }
            cpx<T>* ap = bufB + (size_t)(inst * 2 + p) * szB + (n - 1) * (2 * lm + 1) + lm;
            ap[k] = P + Q;
            if (k > 0) ap[-k] = ((k & 1) ? (T)-1 : (T)1) * (P - Q);
        }
        __syncthreads();

        // ---- phase 3: axial translation per degree m ----
        for (int idx = tid; idx < NI * 2 * lm * (2 * lm + 1); idx += NT) {
            int m = idx % (2 * lm + 1) - lm;
            int rest = idx / (2 * lm + 1);
            int row = rest % lm + 1;
            rest /= lm;
            int p = rest & 1, inst = rest >> 1;
            int dir = inst / nrhs;
            int am = m < 0 ? -m : m;
            int m1 = am < 1 ? 1 : am;
            if (am > nmin || row < m1) continue;
            int ntg = dir ? noj : noi;
            if (row > ntg) continue;
            int rows = noi - m1 + 1, cols = noj - m1 + 1;
            int pz = (am == 0) ? 0 : (m > 0 ? p : 1 - p);
            const T* zb = rec + zoff[am] + 2 * pz * rows * cols;
            const cpx<T>* ap = bufB + (size_t)(inst * 2 + p) * szB + lm + m;   // ap[(n-1)*(2lm+1)]
            cpx<T> g = mk((T)0, (T)0);
            if (dir == 0) {
                const T* zr = zb + 2 * (row - m1) * cols;
                for (int l = m1; l <= noj; l++) {
                    cpx<T> z = mk(zr[2 * (l - m1)], zr[2 * (l - m1) + 1]);
                    g = g + z * ap[(l - 1) * (2 * lm + 1)];
                }
            } else {
                for (int n = m1; n <= noi; n++) {
                    const T* zz = zb + 2 * ((n - m1) * cols + (row - m1));
                    cpx<T> z = mk(zz[0], zz[1]);
                    g = g + ap[(n - 1) * (2 * lm + 1)] * z;
                }
            }
            bufA[(size_t)(inst * 2 + p) * szA + (row - 1) * (2 * lm + 1) + lm + m] = g;
        }
        __syncthreads();

        // ---- phase 4: back rotation, phase, shift, accumulate ----
        for (int idx = tid; idx < NI * 2 * lm * (lm + 1); idx += NT) {
            int k = idx % (lm + 1);
            int rest = idx / (lm + 1);
            int n = rest % lm + 1;
            rest /= lm;
            int p = rest & 1, inst = rest >> 1;
            int dir = inst / nrhs, r = inst % nrhs;
            int tgt = dir ? j : i, ntg = dir ? noj : noi;
            if (n > ntg || k > n) continue;
            int kk = n < nmin ? n : nmin;
            int sop = dir, top = (a.contran >> r) & 1;
            int im = sop ? -1 : 1;
            const T* E = rec + roff[n];
            const T* O = E + (kk + 1) * (n + 1);
            const cpx<T>* g = bufA + (size_t)(inst * 2 + p) * szA + (n - 1) * (2 * lm + 1) + lm;
            // g'(k) = sum_m g(m) d(m,k): the m=0 term enters once, the +-m
            // pairs through s(m)=g(m)+(-1)^m g(-m) and t(m)=g(m)-(-1)^m g(-m).
            cpx<T> P = g[0] * E[k];
            cpx<T> Q = mk((T)0, (T)0);
            for (int m = 1; m <= kk; m++) {
                T sg = (m & 1) ? (T)-1 : (T)1;
                cpx<T> gp = g[m], gm = sg * g[-m];
                P = P + E[m * (n + 1) + k] * (gp + gm);
                if (k > 0) Q = Q + O[(m - 1) * n + (k - 1)] * (gp - gm);
            }
            cpx<T>* ys = a.y + (size_t)r * a.ld + a.offset[tgt];
            if (k == 0) {
                atomic_add_c(&ys[aidx(0, n, p, ntg)], (T)2 * P);   // E(m,0) holds d(m,0)/2
            } else {
                T sk = (k & 1) ? (T)-1 : (T)1;
                cpx<T> gk = P + Q, gmk = sk * (P - Q);
                cpx<T> outk = gk * e[-im * k];
                cpx<T> outmk = gmk * e[im * k];
                if (sop != top) { cpx<T> tt = outk; outk = sk * outmk; outmk = sk * tt; }
                atomic_add_c(&ys[aidx(k, n, p, ntg)], outk);
                atomic_add_c(&ys[aidx(-k, n, p, ntg)], outmk);
            }
        }
        __syncthreads();
        if (tid == 0) {
            int qn = q + 2 * G;
            if (qn < a.npairs) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                int in = a.pairs[qn].x, jn = a.pairs[qn].y;
                uint32_t bytes = (uint32_t)(op_record_units(a.order[in], a.order[jn]) * sizeof(T));
                mbar_arrive_expect_tx(&bar[b], bytes);
                bulk_g2s(opb + (size_t)b * a.maxrec, a.ops + a.opoff[qn], bytes, &bar[b]);
            }
        }
    }
}

template <typename T> size_t translate_smem_bytes(int lmax, int nrhs, int maxrec)
{
    size_t head = 256 + 2 * sizeof(cpx<T>) * (2 * MSTMG_LMAX + 1) + 64 + 128;
    size_t ops = 2 * (size_t)maxrec * sizeof(T);
    int NI = 2 * nrhs;
    size_t bufs = (size_t)NI * 2 * (lmax * 2 * (lmax + 1) + lmax * (2 * lmax + 1)) * sizeof(cpx<T>);
    return head + ops + bufs;
}

template <typename T, int NT, int LM, bool UNI = false> static void launch_translate_lm(const TransArgs<T>& a, int nsm, cudaStream_t st)
{
    size_t smem = translate_smem_bytes<T>(LM, a.nrhs, a.maxrec);
    auto kern = translate_kernel<T, NT, LM, UNI>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // as many CTAs per SM as registers and shared memory allow
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 1;
    }
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 32) per_sm = 32;
    int blocks = nsm * per_sm;
    if (blocks > a.npairs) blocks = a.npairs;
    if (blocks < 1) return;
    kern<<<blocks, NT, smem, st>>>(a);
    launch_counter() += 1;
}

// Pairs of small orders leave most of a 256-thread CTA idle in every phase:
// two-warp CTAs up to order 6.  a.lmax (1 .. MSTMG_LMAX) picks the instance.
template <typename T> void launch_translate(const TransArgs<T>& a, int nsm, cudaStream_t st)
{
    static_assert(MSTMG_LMAX == 16, "one instance per order up to MSTMG_LMAX");
    if (a.uniform) {
        switch (a.lmax) {
        case 3: launch_translate_lm<T, 64, 3, true>(a, nsm, st); return;
        case 4: launch_translate_lm<T, 64, 4, true>(a, nsm, st); return;
        case 5: launch_translate_lm<T, 64, 5, true>(a, nsm, st); return;
        case 6: launch_translate_lm<T, 64, 6, true>(a, nsm, st); return;
        default: break;
        }
    }
    switch (a.lmax) {
    case 1: launch_translate_lm<T, 64, 1>(a, nsm, st); break;
    case 2: launch_translate_lm<T, 64, 2>(a, nsm, st); break;
    case 3: launch_translate_lm<T, 64, 3>(a, nsm, st); break;
    case 4: launch_translate_lm<T, 64, 4>(a, nsm, st); break;
    case 5: launch_translate_lm<T, 64, 5>(a, nsm, st); break;
    case 6: launch_translate_lm<T, 64, 6>(a, nsm, st); break;
    case 7: launch_translate_lm<T, 256, 7>(a, nsm, st); break;
    case 8: launch_translate_lm<T, 256, 8>(a, nsm, st); break;
    case 9: launch_translate_lm<T, 256, 9>(a, nsm, st); break;
    case 10: launch_translate_lm<T, 256, 10>(a, nsm, st); break;
    case 11: launch_translate_lm<T, 256, 11>(a, nsm, st); break;
    case 12: launch_translate_lm<T, 256, 12>(a, nsm, st); break;
    case 13: launch_translate_lm<T, 256, 13>(a, nsm, st); break;
    case 14: launch_translate_lm<T, 256, 14>(a, nsm, st); break;
    case 15: launch_translate_lm<T, 256, 15>(a, nsm, st); break;
    default: launch_translate_lm<T, 256, 16>(a, nsm, st); break;
    }
}

// Coincident centres of a host and a sphere it holds (coefficient_translation's
// zero_translation with vswf_type 1, mtransfer, modules:2334-2344): the
// regular translation is the identity on the common orders, in both
// directions and whatever the shift.  One CTA per (pair, column).
template <typename T>
__global__ void mtransfer_kernel(int npairs, const int2* pairs, const int* order, const int* offset, const cpx<T>* x, cpx<T>* y, int ld)
{
    const int q = blockIdx.x, r = blockIdx.y;
    if (q >= npairs) return;
    const int i = pairs[q].x, j = pairs[q].y;
    const int Li = order[i], Lj = order[j], L = Li < Lj ? Li : Lj;
    const int nb = L * (L + 2);
    const cpx<T>* xr = x + (size_t)r * ld;
    cpx<T>* yr = y + (size_t)r * ld;
    for (int e = threadIdx.x; e < 2 * nb; e += blockDim.x) {
        const int p = e / nb, k = e - p * nb;
        const int n = (int)sqrt((double)(k + 1) + 0.5), m = k + 1 - n * n - n;   // k + 1 = n(n+1) + m
        const int ai = offset[i] + aidx(m, n, p, Li), aj = offset[j] + aidx(m, n, p, Lj);
        atomicAdd(&yr[ai].x, xr[aj].x);
        atomicAdd(&yr[ai].y, xr[aj].y);
        atomicAdd(&yr[aj].x, xr[ai].x);
        atomicAdd(&yr[aj].y, xr[ai].y);
    }
}

template <typename T>
void launch_mtransfer(int npairs, const int2* pairs, const int* order, const int* offset, const cpx<T>* x, cpx<T>* y, int ld, int nrhs,
                      cudaStream_t st)
{
    if (npairs <= 0) return;
    mtransfer_kernel<T><<<dim3(npairs, nrhs), 128, 0, st>>>(npairs, pairs, order, offset, x, y, ld);
    launch_counter() += 1;
}
template void launch_mtransfer<double>(int, const int2*, const int*, const int*, const zd*, zd*, int, int, cudaStream_t);
template void launch_mtransfer<float>(int, const int2*, const int*, const int*, const zf*, zf*, int, int, cudaStream_t);

template void launch_translate<double>(const TransArgs<double>&, int, cudaStream_t);
template void launch_translate<float>(const TransArgs<float>&, int, cudaStream_t);
template size_t translate_smem_bytes<double>(int, int, int);
template size_t translate_smem_bytes<float>(int, int, int);
