// densepair.cu -- MSTM's dense pair translation for pairs whose smaller order
// is below translation_switch_order (coefficient_translation with rot_op
// false, december2023/mstm-modules-33.f90:6669-6674 and 6751-6780): the
// outgoing-to-regular matrix H(r_i - r_j) of gentranmatrix (vswf_type 3,
// source order L_j, target order L_i, both modes) is stored per pair and
// applied in both directions,
//   j -> i (shift_op = F):  y_i += S^t H S^t x_j
//   i -> j (shift_op = T):  y_j += S^u H^T S^u x_i
// where S = shiftcoefficient(-1, -1) and t = tran_op, u = not tran_op (the
// reference shifts when shift_op differs from tran_op).
#include "common.cuh"
#include "gentran.cuh"
#include "densepair.cuh"

// One CTA per dense pair: H (nblk_i x nblk_j x 2 modes) into the record.
__global__ void __launch_bounds__(128) dense_gen_kernel(DenseArgs a)
{
    __shared__ GtShared gs;
    const int q = blockIdx.x;
    if (q >= a.npairs) return;
    const int i = a.pairs[q].x, j = a.pairs[q].y;
    const int Li = a.order[i], Lj = a.order[j];
    const int nbi = Li * (Li + 2), nbj = Lj * (Lj + 2);
    double xp[3] = {a.pos[3 * i] - a.pos[3 * j], a.pos[3 * i + 1] - a.pos[3 * j + 1], a.pos[3 * i + 2] - a.pos[3 * j + 2]};
    gt_prepare(gs, a.g, xp, 3, a.pmed ? mk(a.pmed[2 * q], a.pmed[2 * q + 1]) : mk(a.rimed_re, a.rimed_im), Li + Lj);
    zd* rec64 = a.rec64 ? a.rec64 + a.off[q] : nullptr;
    zf* rec32 = a.rec32 ? a.rec32 + a.off[q] : nullptr;
    for (int e = threadIdx.x; e < nbi * nbj; e += blockDim.x) {
        int t = e % nbi, s = e / nbi;
        int m, n, k, l;
        gt_mn(s, Lj, m, n);
        gt_mn(t, Li, k, l);
        zd e1, e2;
        gt_element(gs, a.g, 3, Li + Lj, n, m, l, k, e1, e2);
        if (rec64) {
            rec64[e] = e1;
            rec64[e + (size_t)nbi * nbj] = e2;
        }
        if (rec32) {
            rec32[e] = mk((float)e1.x, (float)e1.y);
            rec32[e + (size_t)nbi * nbj] = mk((float)e2.x, (float)e2.y);
        }
    }
}

// shiftcoefficient(-1,-1) of one mode-half slot: the source slot and sign
__device__ __forceinline__ int dp_shift_src(int idx, int L, float& sg)
{
    int m, n;
    gt_mn(idx, L, m, n);
    sg = (m & 1) ? -1.0f : 1.0f;
    return m == 0 ? idx : aidx(-m, n, 0, L);
}

// One CTA per (dense pair, column); both directions, atomics into y.
template <typename T>
__global__ void __launch_bounds__(128) dense_apply_kernel(DenseArgs a, const T* rec, const cpx<T>* x, cpx<T>* y, int ld, unsigned contran)
{
    const int q = blockIdx.x, r = blockIdx.y;
    const int i = a.pairs[q].x, j = a.pairs[q].y;
    const int Li = a.order[i], Lj = a.order[j];
    const int nbi = Li * (Li + 2), nbj = Lj * (Lj + 2);
    const cpx<T>* H = reinterpret_cast<const cpx<T>*>(rec) + a.off[q];
    const bool top = (contran >> r) & 1u;
    const cpx<T>* xi = x + (size_t)r * ld + a.offset[i];
    const cpx<T>* xj = x + (size_t)r * ld + a.offset[j];
    cpx<T>* yi = y + (size_t)r * ld + a.offset[i];
    cpx<T>* yj = y + (size_t)r * ld + a.offset[j];
    // j -> i: row t of H times (S^top x_j), result shifted by S^top
    for (int e = threadIdx.x; e < 2 * nbi; e += blockDim.x) {
        const int p = e / nbi, t0 = e % nbi;
        float so = 1.0f;
        const int t = top ? dp_shift_src(t0, Li, so) : t0;   // output slot t0 takes row t (times its sign)
        const cpx<T>* Hp = H + (size_t)p * nbi * nbj;
        cpx<T> acc = mk((T)0, (T)0);
        for (int s = 0; s < nbj; s++) {
            float si = 1.0f;
            const int ss = top ? dp_shift_src(s, Lj, si) : s;
            cpx<T> v = xj[p * nbj + ss];
            acc = acc + Hp[t + (size_t)nbi * s] * ((T)si * v);
        }
        acc = (T)so * acc;
        atomicAdd(&yi[p * nbi + t0].x, acc.x);
        atomicAdd(&yi[p * nbi + t0].y, acc.y);
    }
    // i -> j: column s of H (H^T) times (S^{!top} x_i), result shifted by S^{!top}
    for (int e = threadIdx.x; e < 2 * nbj; e += blockDim.x) {
        const int p = e / nbj, s0 = e % nbj;
        float so = 1.0f;
        const int s = !top ? dp_shift_src(s0, Lj, so) : s0;
        const cpx<T>* Hp = H + (size_t)p * nbi * nbj;
        cpx<T> acc = mk((T)0, (T)0);
        for (int t = 0; t < nbi; t++) {
            float si = 1.0f;
            const int tt = !top ? dp_shift_src(t, Li, si) : t;
            cpx<T> v = xi[p * nbi + tt];
            acc = acc + Hp[t + (size_t)nbi * s] * ((T)si * v);
        }
        acc = (T)so * acc;
        atomicAdd(&yj[p * nbj + s0].x, acc.x);
        atomicAdd(&yj[p * nbj + s0].y, acc.y);
    }
}

void launch_dense_gen(const DenseArgs& a, cudaStream_t st)
{
    if (a.npairs == 0) return;
    dense_gen_kernel<<<a.npairs, 128, 0, st>>>(a);
    launch_counter() += 1;
}
template <typename T> void launch_dense_apply(const DenseArgs& a, const T* rec, const cpx<T>* x, cpx<T>* y, int ld, int nrhs, unsigned contran,
                                              cudaStream_t st)
{
    if (a.npairs == 0) return;
    dense_apply_kernel<T><<<dim3(a.npairs, nrhs), 128, 0, st>>>(a, rec, x, y, ld, contran);
    launch_counter() += 1;
}
template void launch_dense_apply<double>(const DenseArgs&, const double*, const zd*, zd*, int, int, unsigned, cudaStream_t);
template void launch_dense_apply<float>(const DenseArgs&, const float*, const zf*, zf*, int, int, unsigned, cudaStream_t);
