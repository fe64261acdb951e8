// mrhs.cu -- MSTM's BiCG iteration (cbicg, december2023/mstm-solver-8.f90:654-949)
// for many independent systems at once, and the T-matrix helpers of
// tmatrix_solution (solver:22-332).
//
// Each system keeps exactly the reference's recurrence; systems only share
// launches.  A launch covers the a active systems act[0..a) in grid rows, so
// one iteration of any number of systems is a fixed handful of launches (pack,
// translation, post, upd1, upd2 and three scalar finishes) instead of a handful
// per system.  Dot products accumulate in FP64 per CTA and are summed per
// system in a fixed order, so results do not depend on the other systems.
#include "mrhs.cuh"
#include "special.cuh"

#define MB 256

namespace {

__device__ __forceinline__ double mwarp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
template <int K> __device__ __forceinline__ void mblock_store(double (&v)[K], double* out)
{
    __shared__ double sh[K][MB / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        double s = mwarp_sum(v[k]);
        if (lane == 0) sh[k][w] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            double s = 0.0;
            for (int q = 0; q < MB / 32; q++) s += sh[k][q];
            out[k] = s;
        }
    }
}
template <typename T> __device__ __forceinline__ cpx<double> upd_(cpx<T> a) { return mk((double)a.x, (double)a.y); }

// slot e of the first mode half -> (element of mode 1, element of mode 2, Mie row n, sphere)
struct SlotPos { int b0, b1, n, i; };
__device__ __forceinline__ SlotPos slot_pos(const SlotMaps& sm, int e)
{
    SlotPos r;
    r.i = sm.slot[e];
    int L = sm.order[r.i], hb = L * (L + 2);
    int loc = e - sm.offset[r.i] / 2;
    int row = loc % (L + 2), col = loc / (L + 2) + 1;
    r.n = (row <= col) ? col : row - 1;
    r.b0 = sm.offset[r.i] + loc;
    r.b1 = r.b0 + hb;
    return r;
}

}  // namespace

// ---------------------------------------------------------------------------
// Restarted GMRES for many systems: Arnoldi with classical Gram-Schmidt
// applied twice, FP32 vectors with FP64 sums.  Basis vector i of system s is
// V + (s m1 + i) ld; a launch works on the a systems act[0..a) (packed work
// columns W, XP, Y by position k, basis and norms by system s = act[k]).
// ---------------------------------------------------------------------------
// XP[:, k] = V_{act[k], j} for k < a, zero for a <= k < apad; with jp, j =
// *jp and systems whose alive flag is 0 give zero columns
__global__ void __launch_bounds__(MB) gm_gather_kernel(int ld, int m1, int j, int a, const int* act, const zf* V, zf* XP, const int* jp,
                                                      const int* alive)
{
    const int k = blockIdx.y;
    if (jp) j = *jp;
    const zf* v = (k < a && (!alive || alive[act[k]])) ? V + ((size_t)act[k] * m1 + j) * ld : nullptr;
    zf* o = XP + (size_t)k * ld;
    for (int e = blockIdx.x * MB + threadIdx.x; e < ld; e += gridDim.x * MB) o[e] = v ? v[e] : mk(0.0f, 0.0f);
}

// W[:, k] = XP[:, k] - M Y[:, k]   (A v = v - M H v with Y = H v); an == null:
// Y already holds M H v (the host-sphere Mie multiply runs apart)
__global__ void __launch_bounds__(MB) gm_apply_kernel(SlotMaps sm, const zf* an, int ld, const zf* XP, const zf* Y, zf* W)
{
    const size_t o = (size_t)blockIdx.y * ld;
    for (int e = blockIdx.x * MB + threadIdx.x; e < sm.nslots; e += gridDim.x * MB) {
        SlotPos q = slot_pos(sm, e);
        const zf u0 = Y[o + q.b0], u1 = Y[o + q.b1];
        if (!an) {
            W[o + q.b0] = XP[o + q.b0] - u0;
            W[o + q.b1] = XP[o + q.b1] - u1;
            continue;
        }
        const zf* A = an + sm.mie_offset[q.i] + 4 * (q.n - 1);
        W[o + q.b0] = XP[o + q.b0] - (A[0] * u0 + A[2] * u1);
        W[o + q.b1] = XP[o + q.b1] - (A[1] * u0 + A[3] * u1);
    }
}

// h[i S + s] += V_{s,i}^H W[:, k] (and hacc likewise when given), i = blockIdx.y
__global__ void __launch_bounds__(MB) gm_dots_kernel(int ld, int S, int m1, const int* act, const zf* V, const zf* W, double* h, double* hacc,
                                                     const int* len)
{
    const int i = blockIdx.y, k = blockIdx.z, s = act[k];
    const zf* v = V + ((size_t)s * m1 + i) * ld;
    const zf* w = W + (size_t)k * ld;
    const int ne = len ? len[s] : ld;
    double acc[2] = {0.0, 0.0};
    for (int e = blockIdx.x * MB + threadIdx.x; e < ne; e += gridDim.x * MB) {
        const cpx<double> x = upd_(v[e]), y = upd_(w[e]);
        acc[0] += x.x * y.x + x.y * y.y;
        acc[1] += x.x * y.y - x.y * y.x;
    }
    double out[2];
    mblock_store<2>(acc, out);
    if (threadIdx.x == 0) {
        const size_t o = 2 * ((size_t)i * S + s);
        atomicAdd(&h[o], out[0]);
        atomicAdd(&h[o + 1], out[1]);
        if (hacc) {
            atomicAdd(&hacc[o], out[0]);
            atomicAdd(&hacc[o + 1], out[1]);
        }
    }
}

// W[:, k] -= sum_{i < kp1} V_{s,i} h[i S + s] (FP64 accumulation per
// element); nrm[s] += |W[:, k]|^2 of the result when nrm is given; with
// jp, kp1 = *jp + 1
__global__ void __launch_bounds__(MB) gm_update_kernel(int ld, int S, int m1, int kp1, const int* act, const zf* V, const double* h, zf* W,
                                                      double* nrm, const int* len, const int* jp)
{
    const int k = blockIdx.y, s = act[k];
    if (jp) kp1 = *jp + 1;
    const zf* vs = V + (size_t)s * m1 * ld;
    zf* w = W + (size_t)k * ld;
    const int ne = len ? len[s] : ld;
    double n2[1] = {0.0};
    for (int e = blockIdx.x * MB + threadIdx.x; e < ne; e += gridDim.x * MB) {
        cpx<double> x = upd_(w[e]);
        for (int i = 0; i < kp1; i++) {
            const cpx<double> t = upd_(vs[(size_t)i * ld + e]) * mk(h[2 * ((size_t)i * S + s)], h[2 * ((size_t)i * S + s) + 1]);
            x.x -= t.x;
            x.y -= t.y;
        }
        const zf r = mk((float)x.x, (float)x.y);
        w[e] = r;
        n2[0] += (double)r.x * r.x + (double)r.y * r.y;
    }
    if (nrm) {
        double out[1];
        mblock_store<1>(n2, out);
        if (threadIdx.x == 0) atomicAdd(&nrm[s], out[0]);
    }
}

// V_{s,jd} = src / sqrt(nrm[s stride]) with src = Wsrc[:, s] (by_sys) or
// Wsrc[:, k]; zero where the norm is below tiny
__global__ void __launch_bounds__(MB) gm_scale_kernel(int ld, int m1, int jd, const int* act, int by_sys, const zf* Wsrc, const double* nrm,
                                                     int stride, double tiny, zf* V, const int* len, const int* jp)
{
    const int k = blockIdx.y, s = act[k];
    if (jp) jd = *jp + 1;
    const double n2 = nrm[(size_t)s * stride];
    const float f = (n2 > tiny * tiny) ? (float)(1.0 / sqrt(n2)) : 0.0f;
    const zf* w = Wsrc + (size_t)(by_sys ? s : k) * ld;
    zf* d = V + ((size_t)s * m1 + jd) * ld;
    const int ne = len ? len[s] : ld;
    for (int e = blockIdx.x * MB + threadIdx.x; e < ne; e += gridDim.x * MB) d[e] = f * w[e];
}

// X[:, s] += sum_{i < kp1} y[i S + s] V_{s,i} (FP64); with kp1p, kp1 = *kp1p
__global__ void __launch_bounds__(MB) gm_combine_kernel(int ld, int S, int m1, int kp1, const int* act, const zf* V, const double* y, zd* X,
                                                       const int* kp1p)
{
    const int k = blockIdx.y, s = act[k];
    if (kp1p) kp1 = *kp1p;
    const zf* vs = V + (size_t)s * m1 * ld;
    zd* x = X + (size_t)s * ld;
    for (int e = blockIdx.x * MB + threadIdx.x; e < ld; e += gridDim.x * MB) {
        cpx<double> a = x[e];
        for (int i = 0; i < kp1; i++)
            a = a + upd_(vs[(size_t)i * ld + e]) * mk(y[2 * ((size_t)i * S + s)], y[2 * ((size_t)i * S + s) + 1]);
        x[e] = a;
    }
}

// ---------------------------------------------------------------------------
// Ensembles: independent configurations in one index space (no pairs between
// them).  System s = 2 c + p is polarisation p of configuration c: column p
// of the ne x 2 blocks, elements [off[s], off[s] + len[s]) (slots
// [off[s]/2, (off[s] + len[s])/2)).  Basis vector i of system s at
// V + (s m1 + i) ldv, work column k at W + k ldv.
// ---------------------------------------------------------------------------
// R[p] = B - X + M YP over the segment of system act[k] (rounded to FP32);
// rr[2 s] += |r|^2, rr[2 s + 1] += |b|^2 over it (zeroed by the caller)
__global__ void __launch_bounds__(MB) eg_resid_kernel(SlotMaps sm, const zd* an, int ne, const int* act, const int* off, const int* len,
                                                     const zd* B, const zd* X, const zd* YP, zf* R, double* rr)
{
    const int s = act[blockIdx.y], p = s & 1;
    const size_t o = (size_t)p * ne;
    const int e0 = off[s] / 2, e1 = (off[s] + len[s]) / 2;
    double acc[2] = {0.0, 0.0};
    for (int e = e0 + blockIdx.x * MB + threadIdx.x; e < e1; e += gridDim.x * MB) {
        SlotPos q = slot_pos(sm, e);
        const zd* A = an + sm.mie_offset[q.i] + 4 * (q.n - 1);
        const zd u0 = YP[o + q.b0], u1 = YP[o + q.b1];
        const zd m[2] = {A[0] * u0 + A[2] * u1, A[1] * u0 + A[3] * u1};
        const int bb[2] = {q.b0, q.b1};
        for (int h = 0; h < 2; h++) {
            const zd bv = B[o + bb[h]];
            const zd rv = (bv - X[o + bb[h]]) + m[h];
            R[o + bb[h]] = mk((float)rv.x, (float)rv.y);
            acc[0] += rv.x * rv.x + rv.y * rv.y;
            acc[1] += bv.x * bv.x + bv.y * bv.y;
        }
    }
    double out[2];
    mblock_store<2>(acc, out);
    if (threadIdx.x == 0) {
        atomicAdd(&rr[2 * s], out[0]);
        atomicAdd(&rr[2 * s + 1], out[1]);
    }
}

// V_{s,0} = R[p, segment] / sqrt(rr[2 s]) (zero where the norm is below tiny)
__global__ void __launch_bounds__(MB) eg_start_kernel(int ne, int ldv, int m1, const int* act, const int* off, const int* len, const zf* R,
                                                     const double* rr, double tiny, zf* V)
{
    const int s = act[blockIdx.y], p = s & 1;
    const double n2 = rr[2 * s];
    const float f = (n2 > tiny * tiny) ? (float)(1.0 / sqrt(n2)) : 0.0f;
    const zf* r = R + (size_t)p * ne + off[s];
    zf* v = V + (size_t)s * m1 * ldv;
    for (int e = blockIdx.x * MB + threadIdx.x; e < len[s]; e += gridDim.x * MB) v[e] = f * r[e];
}

// XP[p, segment of s] = V_{s,j} (XP zeroed by the caller); with jp, j = *jp
// and systems whose alive flag is 0 are left out
__global__ void __launch_bounds__(MB) eg_gather_kernel(int ne, int ldv, int m1, int j, const int* act, const int* off, const int* len,
                                                      const zf* V, zf* XP, const int* jp, const int* alive)
{
    const int s = act[blockIdx.y], p = s & 1;
    if (jp) j = *jp;
    if (alive && !alive[s]) return;
    const zf* v = V + ((size_t)s * m1 + j) * ldv;
    zf* x = XP + (size_t)p * ne + off[s];
    for (int e = blockIdx.x * MB + threadIdx.x; e < len[s]; e += gridDim.x * MB) x[e] = v[e];
}

// W[:, k] = (XP - M Y)[p, segment of s], local indices
__global__ void __launch_bounds__(MB) eg_apply_kernel(SlotMaps sm, const zf* an, int ne, int ldv, const int* act, const int* off, const int* len,
                                                     const zf* XP, const zf* Y, zf* W)
{
    const int k = blockIdx.y, s = act[k], p = s & 1;
    const size_t o = (size_t)p * ne;
    const int e0 = off[s] / 2, e1 = (off[s] + len[s]) / 2;
    zf* w = W + (size_t)k * ldv - off[s];
    for (int e = e0 + blockIdx.x * MB + threadIdx.x; e < e1; e += gridDim.x * MB) {
        SlotPos q = slot_pos(sm, e);
        const zf* A = an + sm.mie_offset[q.i] + 4 * (q.n - 1);
        const zf u0 = Y[o + q.b0], u1 = Y[o + q.b1];
        w[q.b0] = XP[o + q.b0] - (A[0] * u0 + A[2] * u1);
        w[q.b1] = XP[o + q.b1] - (A[1] * u0 + A[3] * u1);
    }
}

// X[p, segment of s] += sum_{i < kp1} y[i S + s] V_{s,i} (FP64)
__global__ void __launch_bounds__(MB) eg_combine_kernel(int ne, int ldv, int S, int m1, int kp1, const int* act, const int* off, const int* len,
                                                       const zf* V, const double* y, zd* X, const int* kp1p)
{
    const int s = act[blockIdx.y], p = s & 1;
    if (kp1p) kp1 = *kp1p;
    const zf* vs = V + (size_t)s * m1 * ldv;
    zd* x = X + (size_t)p * ne + off[s];
    for (int e = blockIdx.x * MB + threadIdx.x; e < len[s]; e += gridDim.x * MB) {
        cpx<double> a = x[e];
        for (int i = 0; i < kp1; i++)
            a = a + upd_(vs[(size_t)i * ldv + e]) * mk(y[2 * ((size_t)i * S + s)], y[2 * ((size_t)i * S + s) + 1]);
        x[e] = a;
    }
}

int multi_grid(int nslots, int a, int nsm)
{
    int want = (4 * nsm + a - 1) / (a > 0 ? a : 1);
    int most = (nslots + MB - 1) / MB;
    int g = want < most ? want : most;
    return g < 1 ? 1 : g;
}

template <typename T>
__global__ void __launch_bounds__(MB) m_gather_kernel(int ld, int a, const int* act, const cpx<T>* X, cpx<T>* XP)
{
    const int k = blockIdx.y;
    cpx<T>* dst = XP + (size_t)k * ld;
    if (k >= a) {
        for (int e = blockIdx.x * MB + threadIdx.x; e < ld; e += gridDim.x * MB) dst[e] = mk((T)0, (T)0);
        return;
    }
    const cpx<T>* src = X + (size_t)act[k] * ld;
    for (int e = blockIdx.x * MB + threadIdx.x; e < ld; e += gridDim.x * MB) dst[e] = src[e];
}

template <typename T>
__global__ void __launch_bounds__(MB) m_pack_kernel(SlotMaps sm, const cpx<T>* an, int ld, int a, const int* act, const cpx<T>* P,
                                                    const cpx<T>* W, cpx<T>* XP)
{
    const int k = blockIdx.y;
    cpx<T>* xp = XP + (size_t)(2 * k) * ld;
    cpx<T>* xw = xp + ld;
    if (k >= a) {
        for (int e = blockIdx.x * MB + threadIdx.x; e < ld; e += gridDim.x * MB) {
            xp[e] = mk((T)0, (T)0);
            xw[e] = mk((T)0, (T)0);
        }
        return;
    }
    const int s = act[k];
    const cpx<T>* p = P + (size_t)s * ld;
    const cpx<T>* w = W + (size_t)s * ld;
    for (int e = blockIdx.x * MB + threadIdx.x; e < sm.nslots; e += gridDim.x * MB) {
        SlotPos q = slot_pos(sm, e);
        xp[q.b0] = p[q.b0];
        xp[q.b1] = p[q.b1];
        // A^T conj(w)  (multmiecoeffmult with idir /= 1 on the conjugated
        // vector); an == null: conj(w) alone (the host-sphere multiply follows)
        cpx<T> x0 = cj(w[q.b0]), x1 = cj(w[q.b1]);
        if (!an) {
            xw[q.b0] = x0;
            xw[q.b1] = x1;
            continue;
        }
        const cpx<T>* A = an + sm.mie_offset[q.i] + 4 * (q.n - 1);
        xw[q.b0] = A[0] * x0 + A[1] * x1;
        xw[q.b1] = A[2] * x0 + A[3] * x1;
    }
}

// cr = b - x + M y ; cp = cr ; cq = cw = conj(cr); partials sum cr*cr, sum |b|^2
template <typename T>
__global__ void __launch_bounds__(MB) m_init_kernel(SlotMaps sm, const cpx<T>* an, int ld, const int* act, const cpx<T>* B,
                                                    MultiVecs<T> v, const cpx<T>* YP, int have_y, double* part)
{
    const int k = blockIdx.y, s = act[k];
    const size_t o = (size_t)s * ld;
    const cpx<T>* y = YP + (size_t)k * ld;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int e = blockIdx.x * MB + threadIdx.x; e < sm.nslots; e += gridDim.x * MB) {
        SlotPos q = slot_pos(sm, e);
        cpx<T> m[2] = {mk((T)0, (T)0), mk((T)0, (T)0)};
        if (have_y) {
            cpx<T> u0 = y[q.b0], u1 = y[q.b1];
            m[0] = u0;   // an == null: y already holds M H x
            m[1] = u1;
            if (an) {
                const cpx<T>* A = an + sm.mie_offset[q.i] + 4 * (q.n - 1);
                m[0] = A[0] * u0 + A[2] * u1;
                m[1] = A[1] * u0 + A[3] * u1;
            }
        }
        const int bb[2] = {q.b0, q.b1};
        for (int h = 0; h < 2; h++) {
            size_t g = o + bb[h];
            cpx<T> bv = B[g];
            cpx<T> rv = have_y ? (bv - v.X[g]) + m[h] : bv;
            v.R[g] = rv;
            v.P[g] = rv;
            v.Q[g] = cj(rv);
            v.W[g] = cj(rv);
            cpx<double> rd = upd_(rv), bd = upd_(bv);
            acc[0] += rd.x * rd.x - rd.y * rd.y;
            acc[1] += 2.0 * rd.x * rd.y;
            acc[2] += bd.x * bd.x + bd.y * bd.y;
        }
    }
    mblock_store<3>(acc, part + 3 * ((size_t)k * gridDim.x + blockIdx.x));
}

// The scalar steps of one system after a reduction (same logic as cbicg's):
// mode 0 after init, 1 after post, 2 after upd1.  pk: its G per-CTA partials
// of K values, summed in CTA order; read through L2 (__ldcg), since the
// partials of other CTAs may have been written after this SM cached them.
__device__ void m_fin_one(int mode, int G, const double* pk, BicgScalars* sc, double eps)
{
    const int K = (mode == 1) ? 2 : 3;
    double s[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < G; b++)
        for (int j = 0; j < K; j++) s[j] += __ldcg(pk + K * b + j);
    if (mode == 0) {
        sc->csk[0] = s[0];
        sc->csk[1] = s[1];
        sc->enorm = s[2];
        sc->stop = (s[0] == 0.0 && s[1] == 0.0) ? 1 : 0;
        sc->breakdown = 0;
        sc->eerr = 0.0;
    } else if (mode == 1) {
        zd cak = mk(s[0], s[1]);
        if (cabsd(cak) != 0.0) {
            zd al = cdiv(mk(sc->csk[0], sc->csk[1]), cak);
            sc->alpha[0] = al.x;
            sc->alpha[1] = al.y;
        } else {
            sc->breakdown = 1;
        }
    } else {
        if (sc->breakdown) return;
        double eerr = s[2] / sc->enorm;
        sc->eerr = eerr;
        zd csk = mk(sc->csk[0], sc->csk[1]);
        if (eerr < eps || cabsd(csk) == 0.0) {
            sc->stop = 1;
        } else {
            zd csk2 = mk(s[0], s[1]);
            zd b = cdiv(csk2, csk);
            sc->beta[0] = b.x;
            sc->beta[1] = b.y;
            sc->csk_prev[0] = csk.x;
            sc->csk_prev[1] = csk.y;
            sc->csk[0] = csk2.x;
            sc->csk[1] = csk2.y;
        }
    }
}

// Per-system finish, one thread per active system.
__global__ void m_fin_kernel(int mode, int a, int G, const int* act, const double* part, BicgScalars* scs, const double* epsv)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a) return;
    const int K = (mode == 1) ? 2 : 3;
    m_fin_one(mode, G, part + (size_t)K * G * k, scs + act[k], epsv ? epsv[act[k]] : 0.0);
}

// After a CTA stored its partials: the last CTA of system k to finish (a
// counter per system, reset here for the next launch) does the system's
// finish, so no separate finish launch is needed.
__device__ __forceinline__ void m_last_cta_fin(int mode, int k, int s, const double* part, BicgScalars* scs, const double* epsv,
                                               unsigned* cnt)
{
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&cnt[k], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const int K = (mode == 1) ? 2 : 3;
        m_fin_one(mode, (int)gridDim.x, part + (size_t)K * gridDim.x * k, scs + s, epsv ? epsv[s] : 0.0);
        cnt[k] = 0u;
    }
}

// cap = p - M y0 ; caw = w - conj(y1) ; partial sum conj(w) cap
template <typename T>
__global__ void __launch_bounds__(MB) m_post_kernel(SlotMaps sm, const cpx<T>* an, int ld, const int* act, MultiVecs<T> v,
                                                    const cpx<T>* YP, double* part, BicgScalars* scs, unsigned* cnt)
{
    const int k = blockIdx.y, s = act[k];
    const size_t o = (size_t)s * ld;
    const cpx<T>* y0 = YP + (size_t)(2 * k) * ld;
    const cpx<T>* y1 = y0 + ld;
    double acc[2] = {0.0, 0.0};
    for (int e = blockIdx.x * MB + threadIdx.x; e < sm.nslots; e += gridDim.x * MB) {
        SlotPos q = slot_pos(sm, e);
        cpx<T> u0 = y0[q.b0], u1 = y0[q.b1];
        cpx<T> m0 = u0, m1 = u1;   // an == null: y0 already holds M H p
        if (an) {
            const cpx<T>* A = an + sm.mie_offset[q.i] + 4 * (q.n - 1);
            m0 = A[0] * u0 + A[2] * u1;
            m1 = A[1] * u0 + A[3] * u1;
        }
        cpx<T> c0 = v.P[o + q.b0] - m0, c1 = v.P[o + q.b1] - m1;
        v.CAP[o + q.b0] = c0;
        v.CAP[o + q.b1] = c1;
        cpx<T> w0 = v.W[o + q.b0], w1 = v.W[o + q.b1];
        v.CAW[o + q.b0] = w0 - cj(y1[q.b0]);
        v.CAW[o + q.b1] = w1 - cj(y1[q.b1]);
        cpx<double> wd0 = upd_(w0), wd1 = upd_(w1), d0 = upd_(c0), d1 = upd_(c1);
        acc[0] += wd0.x * d0.x + wd0.y * d0.y + wd1.x * d1.x + wd1.y * d1.y;
        acc[1] += wd0.x * d0.y - wd0.y * d0.x + wd1.x * d1.y - wd1.y * d1.x;
    }
    mblock_store<2>(acc, part + 2 * ((size_t)k * gridDim.x + blockIdx.x));
    if (cnt) m_last_cta_fin(1, k, s, part, scs, nullptr, cnt);
}

// x += a p ; r -= a cap ; q -= conj(a) caw ; partials sum conj(q) r, sum |r|^2
template <typename T>
__global__ void __launch_bounds__(MB) m_upd1_kernel(int ld, const int* act, BicgScalars* sc, MultiVecs<T> v, double* part, unsigned* cnt,
                                                    const double* epsv)
{
    const int k = blockIdx.y, s = act[k];
    const size_t o = (size_t)s * ld;
    double acc[3] = {0.0, 0.0, 0.0};
    if (!sc[s].breakdown) {
        cpx<T> al = mk((T)sc[s].alpha[0], (T)sc[s].alpha[1]);
        cpx<T> ac = cj(al);
        for (int e = blockIdx.x * MB + threadIdx.x; e < ld; e += gridDim.x * MB) {
            size_t g = o + e;
            v.X[g] = v.X[g] + al * v.P[g];
            cpx<T> rv = v.R[g] - al * v.CAP[g];
            cpx<T> qv = v.Q[g] - ac * v.CAW[g];
            v.R[g] = rv;
            v.Q[g] = qv;
            cpx<double> rd = upd_(rv), qd = upd_(qv);
            acc[0] += qd.x * rd.x + qd.y * rd.y;
            acc[1] += qd.x * rd.y - qd.y * rd.x;
            acc[2] += rd.x * rd.x + rd.y * rd.y;
        }
    }
    mblock_store<3>(acc, part + 3 * ((size_t)k * gridDim.x + blockIdx.x));
    if (cnt) m_last_cta_fin(2, k, s, part, sc, epsv, cnt);
}

// p = r + b p ; w = q + conj(b) w  (skipped once the system stopped)
template <typename T>
__global__ void __launch_bounds__(MB) m_upd2_kernel(int ld, const int* act, const BicgScalars* sc, MultiVecs<T> v)
{
    const int k = blockIdx.y, s = act[k];
    if (sc[s].stop || sc[s].breakdown) return;
    const size_t o = (size_t)s * ld;
    cpx<T> b = mk((T)sc[s].beta[0], (T)sc[s].beta[1]);
    cpx<T> bc = cj(b);
    for (int e = blockIdx.x * MB + threadIdx.x; e < ld; e += gridDim.x * MB) {
        size_t g = o + e;
        v.P[g] = v.R[g] + b * v.P[g];
        v.W[g] = v.Q[g] + bc * v.W[g];
    }
}

// Per-system finish, one thread per active system (same logic as cbicg's
// scalar steps): mode 0 after init, 1 after post, 2 after upd1.

// Residual replacement of the systems in act: r was replaced by the true
// residual; csk = sum conj(q) r, beta = csk / csk_prev, enorm = sum |r|^2
// (the new base of eerr).  part: 3 partials per CTA per system.
__global__ void m_rrfin_kernel(int a, int G, const int* act, const double* part, BicgScalars* scs)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a) return;
    BicgScalars* sc = scs + act[k];
    double s[3] = {0.0, 0.0, 0.0};
    const double* pk = part + (size_t)3 * G * k;
    for (int b = 0; b < G; b++)
        for (int j = 0; j < 3; j++) s[j] += pk[3 * b + j];
    zd csk2 = mk(s[0], s[1]), prev = mk(sc->csk_prev[0], sc->csk_prev[1]);
    if (cabsd(prev) == 0.0) {
        sc->breakdown = 1;
        return;
    }
    zd b = cdiv(csk2, prev);
    sc->beta[0] = b.x;
    sc->beta[1] = b.y;
    sc->csk[0] = csk2.x;
    sc->csk[1] = csk2.y;
    sc->enorm = s[2];
    sc->eerr = 1.0;
    sc->stop = (s[0] == 0.0 && s[1] == 0.0) ? 1 : 0;
}

// partials sum conj(q) r, sum |r|^2 of the systems in act
template <typename T>
__global__ void __launch_bounds__(MB) m_rrdot_kernel(int ld, const int* act, MultiVecs<T> v, double* part)
{
    const int k = blockIdx.y, s = act[k];
    const size_t o = (size_t)s * ld;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int e = blockIdx.x * MB + threadIdx.x; e < ld; e += gridDim.x * MB) {
        cpx<double> rd = upd_(v.R[o + e]), qd = upd_(v.Q[o + e]);
        acc[0] += qd.x * rd.x + qd.y * rd.y;
        acc[1] += qd.x * rd.y - qd.y * rd.x;
        acc[2] += rd.x * rd.x + rd.y * rd.y;
    }
    mblock_store<3>(acc, part + 3 * ((size_t)k * gridDim.x + blockIdx.x));
}

template <typename TB>
__global__ void __launch_bounds__(MB) m_resid_kernel(SlotMaps sm, const zd* an, int ld, const int* act, const zd* B, const zd* X,
                                                     const zd* YP, cpx<TB>* Rout, int by_sys, double* part)
{
    const int k = blockIdx.y, s = act[k];
    const size_t o = (size_t)s * ld;
    const zd* y = YP + (size_t)k * ld;
    cpx<TB>* ro = Rout + (size_t)(by_sys ? s : k) * ld;
    double acc[2] = {0.0, 0.0};
    for (int e = blockIdx.x * MB + threadIdx.x; e < sm.nslots; e += gridDim.x * MB) {
        SlotPos q = slot_pos(sm, e);
        zd u0 = y[q.b0], u1 = y[q.b1];
        zd m[2] = {u0, u1};   // an == null: y already holds M H x
        if (an) {
            const zd* A = an + sm.mie_offset[q.i] + 4 * (q.n - 1);
            m[0] = A[0] * u0 + A[2] * u1;
            m[1] = A[1] * u0 + A[3] * u1;
        }
        const int bb[2] = {q.b0, q.b1};
        for (int h = 0; h < 2; h++) {
            zd bv = B[o + bb[h]];
            zd rv = (bv - X[o + bb[h]]) + m[h];
            ro[bb[h]] = mk((TB)rv.x, (TB)rv.y);
            acc[0] += rv.x * rv.x + rv.y * rv.y;
            acc[1] += bv.x * bv.x + bv.y * bv.y;
        }
    }
    mblock_store<2>(acc, part + 2 * ((size_t)k * gridDim.x + blockIdx.x));
}

__global__ void m_sum2_kernel(int a, int G, const int* act, const double* part, double* out2)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a) return;
    double s0 = 0.0, s1 = 0.0;
    const double* pk = part + (size_t)2 * G * k;
    for (int b = 0; b < G; b++) {
        s0 += pk[2 * b];
        s1 += pk[2 * b + 1];
    }
    out2[2 * act[k]] = s0;
    out2[2 * act[k] + 1] = s1;
}

template <typename TL>
__global__ void m_addcorr_kernel(int ld, const int* dst, const int* src, zd* X, const cpx<TL>* D)
{
    const int k = blockIdx.y;
    zd* x = X + (size_t)dst[k] * ld;
    const cpx<TL>* d = D + (size_t)src[k] * ld;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ld; e += gridDim.x * blockDim.x)
        x[e] = x[e] + mk((double)d[e].x, (double)d[e].y);
}

__global__ void m_mie_kernel(SlotMaps sm, const zd* an, int ld, const zd* X, zd* Y)
{
    const int k = blockIdx.y;
    const zd* x = X + (size_t)k * ld;
    zd* y = Y + (size_t)k * ld;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < sm.nslots; e += gridDim.x * blockDim.x) {
        SlotPos q = slot_pos(sm, e);
        const zd* A = an + sm.mie_offset[q.i] + 4 * (q.n - 1);
        zd x0 = x[q.b0], x1 = x[q.b1];
        y[q.b0] = A[0] * x0 + A[2] * x1;
        y[q.b1] = A[1] * x0 + A[3] * x1;
    }
}

// ---------------------------------------------------------------------------
// T matrix helpers
// ---------------------------------------------------------------------------

// Column kq-1 (kq = 1..2(2l+1)) of the order-l right-hand sides: degree
// k = -l + (kq-1)/2, mode q = mod(kq-1,2)+1; a(k,l,1) = 1/2, a(k,l,2) = -(-1)^q/2
// (solver:166-178; the T matrix is TE-TM based).
__global__ void tm_rhs_kernel(int l, zd* P0)
{
    const int nb = 2 * l * (l + 2), ncol = 2 * (2 * l + 1);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nb * ncol; e += gridDim.x * blockDim.x) {
        int col = e / nb, el = e - col * nb;
        int k = -l + col / 2, q = col % 2 + 1;
        zd v = mk(0.0, 0.0);
        if (el == aidx(k, l, 0, l)) v = mk(0.5, 0.0);
        if (el == aidx(k, l, 1, l)) v = mk(-0.5 * pm1(q), 0.0);
        P0[e] = v;
    }
}

// lrsphereqeff (scatprops:676-776) with npol = 1 for one (sphere, column);
// g = A^{-1} a as in qefficiencyfactors (scatprops:782-870, no host spheres).
// G (may be null): the exciting fields of the columns (host spheres: the
// interaction without the Mie multiply plus the incident field), else
// A^{-1} a; rext (may be null): the index around each sphere, else rimed
__global__ void tm_qeff_kernel(int nsph, int ncols, const int* order, const int* offset, const int* mie_offset, const double* radius,
                               zd rimed, const zd* an_inv, const zd* A, const zd* P, int ld, double* qcol, const zd* G, const double* rext)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsph * ncols) return;
    const int c = t / nsph, i = t - c * nsph;
    const int L = order[i], off = offset[i], hb = L * (L + 2);
    const double xsp = radius[i];
    const zd ri0 = rext ? mk(rext[2 * i], rext[2 * i + 1]) : rimed;
    const zd xri = xsp * ri0;
    const zd rib = cdivr(2.0, cdivr(1.0, ri0) + cdivr(1.0, ri0));
    zd psi[MSTMG_LMAX + 2], xi[MSTMG_LMAX + 2], scr[2 * (MSTMG_LMAX + 2)];   // sphere orders are at most MSTMG_LMAX
    mstm_cricbessel(L, xri, psi, scr);
    mstm_crichankel(L, xri, xi, scr);
    const zd* a = A + (size_t)c * ld + off;
    const zd* f = P + (size_t)c * ld + off;
    const zd* Ai = an_inv + mie_offset[i];
    double qe = 0.0, qa = 0.0, qi = 0.0;
    const zd cterm = imul(cdiv(cj(cdivr(1.0, ri0)), ri0));
    for (int n = 1; n <= L; n++) {
        zd psip = psi[n - 1] - cdiv((double)n * psi[n], xri);
        zd xip = xi[n - 1] - cdiv((double)n * xi[n], xri);
        zd aam[4], ggm[4], agm[4];
        for (int s = 1; s <= 2; s++)
            for (int u = 1; u <= 2; u++) {
                double sg = pm1(s) * pm1(u);
                int kk = (s - 1) + 2 * (u - 1);
                aam[kk] = cterm * (xip * cj(xi[n]) - sg * (xi[n] * cj(xip)));
                ggm[kk] = cterm * (psip * cj(psi[n]) - sg * (psi[n] * cj(psip)));
                agm[kk] = cterm * (xip * cj(psi[n]) - sg * (xi[n] * cj(psip)));
            }
        const zd* Ain = Ai + 4 * (n - 1);
        for (int m = -n; m <= n; m++) {
            int a0 = aidx(m, n, 0, L);
            zd av[2] = {a[a0], a[a0 + hb]};
            zd gv[2] = {Ain[0] * av[0] + Ain[2] * av[1], Ain[1] * av[0] + Ain[3] * av[1]};
            if (G) {
                const zd* gc = G + (size_t)c * ld + off;
                gv[0] = gc[a0];
                gv[1] = gc[a0 + hb];
            }
            zd fv[2] = {f[a0], f[a0 + hb]};
            for (int s = 0; s < 2; s++)
                for (int u = 0; u < 2; u++) {
                    int kk = s + 2 * u;
                    zd crib = cj(rib) + pm1(s + u) * rib;
                    qi += (ggm[kk] * fv[s] * cj(rib * fv[u])).x;
                    qa += (aam[kk] * av[s] * cj(rib * av[u]) + ggm[kk] * gv[s] * cj(rib * gv[u]) + agm[kk] * av[s] * cj(gv[u]) * crib).x;
                    qe += (agm[kk] * av[s] * cj(fv[u]) * crib).x;
                }
        }
    }
    double* q = qcol + 3 * ((size_t)i + (size_t)nsph * c);
    q[0] = qe * 2.0 / xsp / xsp;
    q[1] = qa * 2.0 / xsp / xsp;
    q[2] = qi * 2.0 / xsp / xsp;   // qs = qi (the reference's 10-22 patch)
}

// One block: per sphere add the columns in order, then the weighted total in sphere order.
__global__ void tm_qsum_kernel(int nsph, int ncols, const double* qcol, const double* radius, double xv, double* sq, double* qsum)
{
    for (int i = threadIdx.x; i < nsph; i += blockDim.x)
        for (int c = 0; c < ncols; c++)
            for (int j = 0; j < 3; j++) sq[3 * i + j] += qcol[3 * ((size_t)i + (size_t)nsph * c) + j];
    __syncthreads();
    if (threadIdx.x == 0) {
        double s[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < nsph; i++)
            for (int j = 0; j < 3; j++) s[j] = s[j] + sq[3 * i + j] * radius[i] * radius[i] / (xv * xv);
        for (int j = 0; j < 3; j++) qsum[j] = s[j];
    }
}

__global__ void tm_store_kernel(int l, int tmo, const zd* A0, zd* tmat)
{
    const int nb = 2 * l * (l + 2), ncol = 2 * (2 * l + 1), nblkt = 2 * tmo * (tmo + 2);
    const int nrow = l * (l + 2);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 2 * nrow * ncol; e += gridDim.x * blockDim.x) {
        int cc = e / (2 * nrow), rr = e - cc * 2 * nrow;
        int mn = rr / 2 + 1, p = rr % 2;
        int n = 1;
        while (n * (n + 2) < mn) n++;
        int m = mn - n * (n + 1);
        int k = -l + cc / 2, q = cc % 2;
        size_t col = (size_t)(2 * (l * (l + 1) + k - 1) + q);
        tmat[(size_t)(2 * (mn - 1) + p) + (size_t)nblkt * col] = A0[(size_t)cc * nb + aidx(m, n, p, l)];
    }
}

// ranorientscatmatrix's reader (scatprops:2031-2075): complex(4) copy with the
// entries of rows n > l filled from tc(q,l(l+1)-k,p,n(n+1)-m) = (-1)^(m+k) tc(p,n(n+1)+m,q,l(l+1)+k).
__global__ void tm_symm_kernel(int tmo, const zd* tmat, float* tc)
{
    const int nblk = tmo * (tmo + 2), nblkt = 2 * nblk;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)nblkt * nblkt; e += (size_t)gridDim.x * blockDim.x) {
        int row = (int)(e % nblkt), col = (int)(e / nblkt);
        int mn = row / 2 + 1, p = row % 2 + 1, kl = col / 2 + 1, q = col % 2 + 1;
        int n = 1;
        while (n * (n + 2) < mn) n++;
        int l = 1;
        while (l * (l + 2) < kl) l++;
        float re, im;
        if (n <= l) {
            zd t = tmat[e];
            re = (float)t.x;
            im = (float)t.y;
        } else {
            // entry (p, mn, q, kl) with n > l is the image of (q, l(l+1)-k, p, n(n+1)-m) of column order n
            int m = mn - n * (n + 1), k = kl - l * (l + 1);
            int srow = 2 * (l * (l + 1) - k - 1) + (q - 1), scol = 2 * (n * (n + 1) - m - 1) + (p - 1);
            zd t = tmat[(size_t)srow + (size_t)nblkt * scol];
            float s = (float)pm1(m + k);
            re = (float)t.x * s;
            im = (float)t.y * s;
        }
        tc[2 * e] = re;
        tc[2 * e + 1] = im;
    }
}

// qextt = -sum Re tc(q,kl,q,kl), qscatt = sum |tc|^2 (single-precision terms,
// double sums in the reader's order), both times 2/xv^2 (scatprops:2103-2122).
__global__ void tm_qextsca_kernel(int tmo, const float* tc, double xv, double* out2)
{
    const int nblkt = 2 * tmo * (tmo + 2);
    __shared__ double colsum[256];
    double qe = 0.0, qs = 0.0;
    for (int c0 = 0; c0 < nblkt; c0 += blockDim.x) {
        int col = c0 + threadIdx.x;
        double s = 0.0;
        if (col < nblkt)
            for (int row = 0; row < nblkt; row++) {
                float re = tc[2 * ((size_t)row + (size_t)nblkt * col)], im = tc[2 * ((size_t)row + (size_t)nblkt * col) + 1];
                // cabs of a complex(4) value: the modulus formed in double, rounded once to single
                float a = (float)sqrt((double)re * re + (double)im * im);
                s = s + (double)(a * a);
            }
        colsum[threadIdx.x] = s;
        __syncthreads();
        if (threadIdx.x == 0)
            for (int j = 0; j < (int)blockDim.x && c0 + j < nblkt; j++) {
                qs = qs + colsum[j];
                int cj_ = c0 + j;
                qe = qe - (double)tc[2 * ((size_t)cj_ + (size_t)nblkt * cj_)];
            }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out2[0] = qe * 2.0 / (xv * xv);
        out2[1] = qs * 2.0 / (xv * xv);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename T> void launch_m_gather(int ld, int a, int apad, const int* act, const cpx<T>* X, cpx<T>* XP, int nsm, cudaStream_t st)
{
    dim3 g(multi_grid(ld, apad, nsm), apad);
    m_gather_kernel<T><<<g, MB, 0, st>>>(ld, a, act, X, XP);
    launch_counter() += 1;
}
template <typename T>
void launch_m_pack(const SlotMaps& sm, const cpx<T>* an, int ld, int a, int apad, const int* act, const cpx<T>* P, const cpx<T>* W,
                   cpx<T>* XP, int nsm, cudaStream_t st)
{
    dim3 g(multi_grid(sm.nslots, apad, nsm), apad);
    m_pack_kernel<T><<<g, MB, 0, st>>>(sm, an, ld, a, act, P, W, XP);
    launch_counter() += 1;
}
template <typename T>
void launch_m_init(const SlotMaps& sm, const cpx<T>* an, int ld, int a, const int* act, const cpx<T>* B, const MultiVecs<T>& v,
                   const cpx<T>* YP, int have_y, double* part, BicgScalars* sc, int nsm, cudaStream_t st)
{
    int G = multi_grid(sm.nslots, a, nsm);
    m_init_kernel<T><<<dim3(G, a), MB, 0, st>>>(sm, an, ld, act, B, v, YP, have_y, part);
    m_fin_kernel<<<(a + 63) / 64, 64, 0, st>>>(0, a, G, act, part, sc, nullptr);
    launch_counter() += 2;
}
template <typename T>
void launch_m_post(const SlotMaps& sm, const cpx<T>* an, int ld, int a, const int* act, const MultiVecs<T>& v, const cpx<T>* YP,
                   double* part, BicgScalars* sc, int nsm, cudaStream_t st, unsigned* cnt)
{
    int G = multi_grid(sm.nslots, a, nsm);
    m_post_kernel<T><<<dim3(G, a), MB, 0, st>>>(sm, an, ld, act, v, YP, part, sc, cnt);
    launch_counter() += 1;
    if (!cnt) {
        m_fin_kernel<<<(a + 63) / 64, 64, 0, st>>>(1, a, G, act, part, sc, nullptr);
        launch_counter() += 1;
    }
}
template <typename T>
void launch_m_upd(int ld, int a, const int* act, const MultiVecs<T>& v, double* part, BicgScalars* sc, const double* epsv, int nsm,
                  cudaStream_t st, unsigned* cnt)
{
    int G = multi_grid(ld, a, nsm);
    m_upd1_kernel<T><<<dim3(G, a), MB, 0, st>>>(ld, act, sc, v, part, cnt, epsv);
    launch_counter() += 1;
    if (!cnt) {
        m_fin_kernel<<<(a + 63) / 64, 64, 0, st>>>(2, a, G, act, part, sc, epsv);
        launch_counter() += 1;
    }
    m_upd2_kernel<T><<<dim3(G, a), MB, 0, st>>>(ld, act, sc, v);
    launch_counter() += 1;
}
template <typename T>
void launch_m_upd1(int ld, int a, const int* act, const MultiVecs<T>& v, double* part, BicgScalars* sc, int nsm, cudaStream_t st,
                   unsigned* cnt)
{
    int G = multi_grid(ld, a, nsm);
    m_upd1_kernel<T><<<dim3(G, a), MB, 0, st>>>(ld, act, sc, v, part, cnt, nullptr);
    launch_counter() += 1;
    if (!cnt) {
        m_fin_kernel<<<(a + 63) / 64, 64, 0, st>>>(2, a, G, act, part, sc, nullptr);
        launch_counter() += 1;
    }
}
template <typename T> void launch_m_upd2(int ld, int a, const int* act, const MultiVecs<T>& v, const BicgScalars* sc, int nsm, cudaStream_t st)
{
    int G = multi_grid(ld, a, nsm);
    m_upd2_kernel<T><<<dim3(G, a), MB, 0, st>>>(ld, act, sc, v);
    launch_counter() += 1;
}
template <typename T> void launch_m_rrfix(int ld, int a, const int* act, const MultiVecs<T>& v, double* part, BicgScalars* sc, int nsm,
                                          cudaStream_t st)
{
    int G = multi_grid(ld, a, nsm);
    m_rrdot_kernel<T><<<dim3(G, a), MB, 0, st>>>(ld, act, v, part);
    m_rrfin_kernel<<<(a + 63) / 64, 64, 0, st>>>(a, G, act, part, sc);
    launch_counter() += 2;
}
template <typename TB>
void launch_m_resid(const SlotMaps& sm, const zd* an, int ld, int a, const int* act, const zd* B, const zd* X, const zd* YP, cpx<TB>* Rout,
                    double* part, double* out2, int nsm, cudaStream_t st, int by_sys)
{
    int G = multi_grid(sm.nslots, a, nsm);
    m_resid_kernel<TB><<<dim3(G, a), MB, 0, st>>>(sm, an, ld, act, B, X, YP, Rout, by_sys, part);
    m_sum2_kernel<<<(a + 63) / 64, 64, 0, st>>>(a, G, act, part, out2);
    launch_counter() += 2;
}
template <typename TL> void launch_m_addcorr(int ld, int a, const int* dst, const int* src, zd* X, const cpx<TL>* D, cudaStream_t st)
{
    dim3 g(multi_grid(ld, a, 148), a);
    m_addcorr_kernel<TL><<<g, MB, 0, st>>>(ld, dst, src, X, D);
    launch_counter() += 1;
}
void launch_m_mie(const SlotMaps& sm, const zd* an, int ld, int ncols, const zd* X, zd* Y, cudaStream_t st)
{
    dim3 g(multi_grid(sm.nslots, ncols, 148), ncols);
    m_mie_kernel<<<g, MB, 0, st>>>(sm, an, ld, X, Y);
    launch_counter() += 1;
}

void launch_tm_rhs(int l, zd* P0, cudaStream_t st)
{
    int tot = 2 * l * (l + 2) * 2 * (2 * l + 1);
    tm_rhs_kernel<<<(tot + 255) / 256, 256, 0, st>>>(l, P0);
    launch_counter() += 1;
}
void launch_tm_qeff(int nsph, int ncols, const int* order, const int* offset, const int* mie_offset, const double* radius, zd rimed,
                    const zd* an_inv, const zd* A, const zd* P, int ld, double* qcol, cudaStream_t st, const zd* G, const double* rext)
{
    int tot = nsph * ncols;
    tm_qeff_kernel<<<(tot + 63) / 64, 64, 0, st>>>(nsph, ncols, order, offset, mie_offset, radius, rimed, an_inv, A, P, ld, qcol, G, rext);
    launch_counter() += 1;
}
void launch_tm_qsum(int nsph, int ncols, const double* qcol, const double* radius, double xv, double* sq, double* qsum, cudaStream_t st)
{
    tm_qsum_kernel<<<1, 256, 0, st>>>(nsph, ncols, qcol, radius, xv, sq, qsum);
    launch_counter() += 1;
}
void launch_tm_store(int l, int tmo, const zd* A0, zd* tmat, cudaStream_t st)
{
    int tot = 2 * l * (l + 2) * 2 * (2 * l + 1);
    tm_store_kernel<<<(tot + 255) / 256, 256, 0, st>>>(l, tmo, A0, tmat);
    launch_counter() += 1;
}
void launch_tm_qext_qsca(int tmo, const zd* tmat, double xv, float* tc, double* out2, cudaStream_t st)
{
    size_t nblkt = 2 * (size_t)tmo * (tmo + 2);
    int g = (int)std::min<size_t>((nblkt * nblkt + 255) / 256, 148 * 16);
    tm_symm_kernel<<<g, 256, 0, st>>>(tmo, tmat, tc);
    tm_qextsca_kernel<<<1, 256, 0, st>>>(tmo, tc, xv, out2);
    launch_counter() += 2;
}

#define INST(T)                                                                                                                     \
    template void launch_m_gather<T>(int, int, int, const int*, const cpx<T>*, cpx<T>*, int, cudaStream_t);                             \
    template void launch_m_pack<T>(const SlotMaps&, const cpx<T>*, int, int, int, const int*, const cpx<T>*, const cpx<T>*, cpx<T>*, \
                                   int, cudaStream_t);                                                                              \
    template void launch_m_init<T>(const SlotMaps&, const cpx<T>*, int, int, const int*, const cpx<T>*, const MultiVecs<T>&,         \
                                   const cpx<T>*, int, double*, BicgScalars*, int, cudaStream_t);                                   \
    template void launch_m_post<T>(const SlotMaps&, const cpx<T>*, int, int, const int*, const MultiVecs<T>&, const cpx<T>*, double*, \
                                   BicgScalars*, int, cudaStream_t, unsigned*);                                                     \
    template void launch_m_upd<T>(int, int, const int*, const MultiVecs<T>&, double*, BicgScalars*, const double*, int, cudaStream_t,  \
                                  unsigned*);                                                                                       \
    template void launch_m_upd1<T>(int, int, const int*, const MultiVecs<T>&, double*, BicgScalars*, int, cudaStream_t, unsigned*); \
    template void launch_m_upd2<T>(int, int, const int*, const MultiVecs<T>&, const BicgScalars*, int, cudaStream_t);               \
    template void launch_m_rrfix<T>(int, int, const int*, const MultiVecs<T>&, double*, BicgScalars*, int, cudaStream_t);
INST(double)
INST(float)
#undef INST
template void launch_m_resid<double>(const SlotMaps&, const zd*, int, int, const int*, const zd*, const zd*, const zd*, zd*, double*, double*,
                                     int, cudaStream_t, int);
template void launch_m_resid<float>(const SlotMaps&, const zd*, int, int, const int*, const zd*, const zd*, const zd*, zf*, double*, double*,
                                    int, cudaStream_t, int);
template void launch_m_addcorr<float>(int, int, const int*, const int*, zd*, const zf*, cudaStream_t);
template void launch_m_addcorr<double>(int, int, const int*, const int*, zd*, const zd*, cudaStream_t);

// ---- GMRES launchers ----
void launch_gm_gather(int ld, int m1, int j, int a, int apad, const int* act, const zf* V, zf* XP, int nsm, cudaStream_t st)
{
    gm_gather_kernel<<<dim3(multi_grid(ld, apad, nsm), apad), MB, 0, st>>>(ld, m1, j, a, act, V, XP, nullptr, nullptr);
    launch_counter() += 1;
}
void launch_gm_apply(const SlotMaps& sm, const zf* an, int ld, int a, const zf* XP, const zf* Y, zf* W, int nsm, cudaStream_t st)
{
    gm_apply_kernel<<<dim3(multi_grid(sm.nslots, a, nsm), a), MB, 0, st>>>(sm, an, ld, XP, Y, W);
    launch_counter() += 1;
}
void launch_gm_dots(int ld, int S, int m1, int kp1, int a, const int* act, const zf* V, const zf* W, double* h, double* hacc, int nsm,
                    cudaStream_t st, const int* len)
{
    gm_dots_kernel<<<dim3(multi_grid(ld, kp1 * a, nsm), kp1, a), MB, 0, st>>>(ld, S, m1, act, V, W, h, hacc, len);
    launch_counter() += 1;
}
void launch_gm_update(int ld, int S, int m1, int kp1, int a, const int* act, const zf* V, const double* h, zf* W, double* nrm, int nsm,
                      cudaStream_t st, const int* len)
{
    gm_update_kernel<<<dim3(multi_grid(ld, a, nsm), a), MB, 0, st>>>(ld, S, m1, kp1, act, V, h, W, nrm, len, nullptr);
    launch_counter() += 1;
}
void launch_gm_scale(int ld, int m1, int jd, int a, const int* act, int by_sys, const zf* Wsrc, const double* nrm, int stride, double tiny,
                     zf* V, int nsm, cudaStream_t st, const int* len)
{
    gm_scale_kernel<<<dim3(multi_grid(ld, a, nsm), a), MB, 0, st>>>(ld, m1, jd, act, by_sys, Wsrc, nrm, stride, tiny, V, len, nullptr);
    launch_counter() += 1;
}
void launch_gm_combine(int ld, int S, int m1, int kp1, int a, const int* act, const zf* V, const double* y, zd* X, int nsm, cudaStream_t st)
{
    gm_combine_kernel<<<dim3(multi_grid(ld, a, nsm), a), MB, 0, st>>>(ld, S, m1, kp1, act, V, y, X, nullptr);
    launch_counter() += 1;
}
// ---- ensemble launchers (grid rows = active systems) ----
void launch_eg_resid(const SlotMaps& sm, const zd* an, int ne, int ldv, int a, const int* act, const int* off, const int* len, const zd* B,
                     const zd* X, const zd* YP, zf* R, double* rr, int nsm, cudaStream_t st)
{
    eg_resid_kernel<<<dim3(multi_grid(ldv / 2, a, nsm), a), MB, 0, st>>>(sm, an, ne, act, off, len, B, X, YP, R, rr);
    launch_counter() += 1;
}
void launch_eg_start(int ne, int ldv, int m1, int a, const int* act, const int* off, const int* len, const zf* R, const double* rr, double tiny,
                     zf* V, int nsm, cudaStream_t st)
{
    eg_start_kernel<<<dim3(multi_grid(ldv, a, nsm), a), MB, 0, st>>>(ne, ldv, m1, act, off, len, R, rr, tiny, V);
    launch_counter() += 1;
}
void launch_eg_gather(int ne, int ldv, int m1, int j, int a, const int* act, const int* off, const int* len, const zf* V, zf* XP, int nsm,
                      cudaStream_t st)
{
    eg_gather_kernel<<<dim3(multi_grid(ldv, a, nsm), a), MB, 0, st>>>(ne, ldv, m1, j, act, off, len, V, XP, nullptr, nullptr);
    launch_counter() += 1;
}
void launch_eg_apply(const SlotMaps& sm, const zf* an, int ne, int ldv, int a, const int* act, const int* off, const int* len, const zf* XP,
                     const zf* Y, zf* W, int nsm, cudaStream_t st)
{
    eg_apply_kernel<<<dim3(multi_grid(ldv / 2, a, nsm), a), MB, 0, st>>>(sm, an, ne, ldv, act, off, len, XP, Y, W);
    launch_counter() += 1;
}
void launch_eg_combine(int ne, int ldv, int S, int m1, int kp1, int a, const int* act, const int* off, const int* len, const zf* V,
                       const double* y, zd* X, int nsm, cudaStream_t st)
{
    eg_combine_kernel<<<dim3(multi_grid(ldv, a, nsm), a), MB, 0, st>>>(ne, ldv, S, m1, kp1, act, off, len, V, y, X, nullptr);
    launch_counter() += 1;
}

// ---------------------------------------------------------------------------
// Arnoldi cycles driven on the device (the two-column solves: a fixed
// orientation, an ensemble).  The step index j, the systems still iterating
// (alive), the Givens rotations, the rotated Hessenberg columns and the
// least-squares right-hand sides live in device memory, so a whole cycle runs
// as one CUDA graph whose body (one Arnoldi step) repeats under a conditional
// WHILE node that the Givens kernel clears; the host synchronises once per
// cycle.  Same arithmetic as the host's rotations (FP64).
// ---------------------------------------------------------------------------
// h[i S + s] (+ hacc) += V_{s,i}^H W[:, k] for i <= *jp: items (i, k, chunk)
// over a fixed grid, partial dots over chunks of `chunk` elements
__global__ void __launch_bounds__(MB) gm_dots_dev_kernel(int ld, int S, int m1, int a, const int* act, const int* jp, const zf* V, const zf* W,
                                                        double* h, double* hacc, const int* len, int chunk)
{
    const int kp1 = *jp + 1;
    const int nch = (ld + chunk - 1) / chunk;
    const long long nitem = (long long)kp1 * a * nch;
    for (long long it = blockIdx.x; it < nitem; it += gridDim.x) {
        const int ch = (int)(it % nch);
        const int k = (int)((it / nch) % a);
        const int i = (int)(it / ((long long)nch * a));
        const int s = act[k];
        const int ne = len ? len[s] : ld;
        const zf* v = V + ((size_t)s * m1 + i) * ld;
        const zf* w = W + (size_t)k * ld;
        double acc[2] = {0.0, 0.0};
        const int e1 = min(ne, (ch + 1) * chunk);
        for (int e = ch * chunk + threadIdx.x; e < e1; e += MB) {
            const cpx<double> x = upd_(v[e]), y = upd_(w[e]);
            acc[0] += x.x * y.x + x.y * y.y;
            acc[1] += x.x * y.y - x.y * y.x;
        }
        double out[2];
        mblock_store<2>(acc, out);
        if (threadIdx.x == 0) {
            const size_t o = 2 * ((size_t)i * S + s);
            atomicAdd(&h[o], out[0]);
            atomicAdd(&h[o + 1], out[1]);
            if (hacc) {
                atomicAdd(&hacc[o], out[0]);
                atomicAdd(&hacc[o + 1], out[1]);
            }
        }
        __syncthreads();   // mblock_store's shared slots are reused by the next item
    }
}

// One block: the Givens step of every alive system (thread k for system
// act[k]), as the host does it: the Hessenberg column of step j (h1) and
// the norm of the new vector (h0[s]), the earlier rotations, the new one,
// the least-squares right-hand side g; a system stops when its residual
// estimate |g_{j+1}|^2 falls below target[s] or its Krylov space is
// invariant (status 2 when the column is zero).  Thread 0 then advances j and
// sets the cycle's WHILE condition: some system alive and j < jmax.
__global__ void __launch_bounds__(256) gm_givens_kernel(int S, int m, int a, const int* act, const double* h0, const double* h1, GmDevState d,
                                                       cudaGraphConditionalHandle cond)
{
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    const int j = *d.j, m1 = m + 1;
    for (int k = threadIdx.x; k < a; k += blockDim.x) {
        const int s = act[k];
        if (!d.alive[s]) continue;
        double2* col = d.Rm + ((size_t)s * m + j) * m1;
        double cn = 0.0;
        for (int i = 0; i <= j; i++) {
            const size_t o = 2 * ((size_t)i * S + s);
            col[i] = make_double2(h1[o], h1[o + 1]);
            cn += h1[o] * h1[o] + h1[o + 1] * h1[o + 1];
        }
        const double hsub = sqrt(fmax(h0[s], 0.0));
        const double* cs = d.cs + (size_t)s * m;
        const double2* sn = d.sn + (size_t)s * m;
        for (int i = 0; i < j; i++) {   // the earlier rotations
            const double ci = cs[i];
            const double2 si = sn[i], a0 = col[i], a1 = col[i + 1];
            // t = ci a0 + si a1; a1' = -conj(si) a0 + ci a1
            const double2 t = make_double2(ci * a0.x + si.x * a1.x - si.y * a1.y, ci * a0.y + si.x * a1.y + si.y * a1.x);
            col[i + 1] = make_double2(-(si.x * a0.x + si.y * a0.y) + ci * a1.x, -(si.x * a0.y - si.y * a0.x) + ci * a1.y);
            col[i] = t;
        }
        const double aa = hypot(col[j].x, col[j].y), rho = sqrt(aa * aa + hsub * hsub);
        if (rho == 0.0) {   // A v_j = 0: the operator is singular
            d.status[s] = 2;
            d.alive[s] = 0;
            continue;
        }
        const double2 ph = aa > 0.0 ? make_double2(col[j].x / aa, col[j].y / aa) : make_double2(1.0, 0.0);
        const double cj = aa / rho;
        const double2 sj = make_double2(ph.x * hsub / rho, ph.y * hsub / rho);
        d.cs[(size_t)s * m + j] = cj;
        d.sn[(size_t)s * m + j] = sj;
        col[j] = make_double2(ph.x * rho, ph.y * rho);
        double2* g = d.g + (size_t)s * m1;
        const double2 gj = g[j];
        g[j + 1] = make_double2(-(sj.x * gj.x + sj.y * gj.y), -(sj.x * gj.y - sj.y * gj.x));   // -conj(sj) gj
        g[j] = make_double2(cj * gj.x, cj * gj.y);
        d.kk[s] = j + 1;
        const double e2 = g[j + 1].x * g[j + 1].x + g[j + 1].y * g[j + 1].y;
        if (e2 >= d.target[s] && hsub > 1.0e-13 * sqrt(cn + hsub * hsub)) atomicAdd(&cnt, 1);
        else d.alive[s] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *d.j = j + 1;
        cudaGraphSetConditional(cond, (cnt > 0 && j + 1 < *d.jmax) ? 1u : 0u);
    }
}

// The cycle's least-squares solutions R y = g (back substitution per system,
// thread k for system act[k]) into y[i S + s] (complex as 2 doubles, zero past
// kk[s]; y zeroed by the caller), and *kmax = the largest kk.
__global__ void __launch_bounds__(256) gm_backsolve_kernel(int S, int m, int a, const int* act, GmDevState d, double* y, int* kmax)
{
    const int m1 = m + 1;
    for (int k = threadIdx.x + blockIdx.x * blockDim.x; k < a; k += blockDim.x * gridDim.x) {
        const int s = act[k], ks = d.kk[s];
        atomicMax(kmax, ks);
        const double2* R = d.Rm + (size_t)s * m * m1;   // column l at R + l m1
        const double2* g = d.g + (size_t)s * m1;
        for (int i = ks - 1; i >= 0; i--) {
            double2 t = g[i];
            for (int l = i + 1; l < ks; l++) {
                const double2 r = R[(size_t)l * m1 + i];
                const double yx = y[2 * ((size_t)l * S + s)], yy = y[2 * ((size_t)l * S + s) + 1];
                t.x -= r.x * yx - r.y * yy;
                t.y -= r.x * yy + r.y * yx;
            }
            const double2 d0 = R[(size_t)i * m1 + i];
            const double den = d0.x * d0.x + d0.y * d0.y;
            y[2 * ((size_t)i * S + s)] = (t.x * d0.x + t.y * d0.y) / den;
            y[2 * ((size_t)i * S + s) + 1] = (t.y * d0.x - t.x * d0.y) / den;
        }
    }
}

void launch_gm_gather_dev(int ld, int m1, int a, int apad, const int* act, const int* jp, const int* alive, const zf* V, zf* XP, int nsm,
                          cudaStream_t st)
{
    gm_gather_kernel<<<dim3(multi_grid(ld, apad, nsm), apad), MB, 0, st>>>(ld, m1, 0, a, act, V, XP, jp, alive);
    launch_counter() += 1;
}
void launch_eg_gather_dev(int ne, int ldv, int m1, int a, const int* act, const int* off, const int* len, const int* jp, const int* alive,
                          const zf* V, zf* XP, int nsm, cudaStream_t st)
{
    eg_gather_kernel<<<dim3(multi_grid(ldv, a, nsm), a), MB, 0, st>>>(ne, ldv, m1, 0, act, off, len, V, XP, jp, alive);
    launch_counter() += 1;
}
void launch_gm_dots_dev(int ld, int S, int m1, int a, const int* act, const int* jp, const zf* V, const zf* W, double* h, double* hacc,
                        int nsm, cudaStream_t st, const int* len)
{
    gm_dots_dev_kernel<<<4 * nsm, MB, 0, st>>>(ld, S, m1, a, act, jp, V, W, h, hacc, len, 8192);
    launch_counter() += 1;
}
void launch_gm_update_dev(int ld, int S, int m1, int a, const int* act, const int* jp, const zf* V, const double* h, zf* W, double* nrm,
                          int nsm, cudaStream_t st, const int* len)
{
    gm_update_kernel<<<dim3(multi_grid(ld, a, nsm), a), MB, 0, st>>>(ld, S, m1, 0, act, V, h, W, nrm, len, jp);
    launch_counter() += 1;
}
void launch_gm_scale_dev(int ld, int m1, int a, const int* act, const int* jp, const zf* Wsrc, const double* nrm, double tiny, zf* V,
                         int nsm, cudaStream_t st, const int* len)
{
    gm_scale_kernel<<<dim3(multi_grid(ld, a, nsm), a), MB, 0, st>>>(ld, m1, 0, act, 0, Wsrc, nrm, 1, tiny, V, len, jp);
    launch_counter() += 1;
}
void launch_gm_givens(int S, int m, int a, const int* act, const double* h0, const double* h1, const GmDevState& d,
                      cudaGraphConditionalHandle cond, cudaStream_t st)
{
    gm_givens_kernel<<<1, 256, 0, st>>>(S, m, a, act, h0, h1, d, cond);
    launch_counter() += 1;
}
void launch_gm_backsolve(int S, int m, int a, const int* act, const GmDevState& d, double* y, int* kmax, cudaStream_t st)
{
    gm_backsolve_kernel<<<(a + 255) / 256, 256, 0, st>>>(S, m, a, act, d, y, kmax);
    launch_counter() += 1;
}
void launch_gm_combine_dev(int ld, int S, int m1, int a, const int* act, const zf* V, const double* y, const int* kp1, zd* X, int nsm,
                           cudaStream_t st)
{
    gm_combine_kernel<<<dim3(multi_grid(ld, a, nsm), a), MB, 0, st>>>(ld, S, m1, 0, act, V, y, X, kp1);
    launch_counter() += 1;
}
void launch_eg_combine_dev(int ne, int ldv, int S, int m1, int a, const int* act, const int* off, const int* len, const zf* V, const double* y,
                           const int* kp1, zd* X, int nsm, cudaStream_t st)
{
    eg_combine_kernel<<<dim3(multi_grid(ldv, a, nsm), a), MB, 0, st>>>(ne, ldv, S, m1, 0, act, off, len, V, y, X, kp1);
    launch_counter() += 1;
}
