// bicg.cu -- device vector kernels of MSTM's complex biconjugate-gradient
// solver (cbicg, december2023/mstm-solver-8.f90:654-949).  The iteration
// keeps every vector and scalar on the device; the host reads back one small
// scalar block per iteration to decide termination exactly where cbicg does.
//
// Fortran dot_product(a,b) = sum(conj(a)*b); the reference's csk uses
// dot_product(conjg(cr),cr) = sum(cr*cr) (no conjugate).  All dot products
// accumulate in FP64 whatever the vector precision.
#include "common.cuh"
#include "bicg.cuh"

#define RB 256

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block reduction of K doubles; thread 0 writes K values to out.
template <int K> __device__ __forceinline__ void block_reduce_store(double (&v)[K], double* out)
{
    __shared__ double sh[K][RB / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        double s = warp_sum(v[k]);
        if (lane == 0) sh[k][w] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            double s = 0.0;
            for (int q = 0; q < RB / 32; q++) s += sh[k][q];
            out[k] = s;
        }
    }
}

template <typename T> __device__ __forceinline__ cpx<double> up(cpx<T> a) { return mk((double)a.x, (double)a.y); }

// cap = p - M*y0 (Mie multiply, idir=1), caw = w - conj(y1); partial sum conj(w)*cap.
// an == null: y0 already holds M*y0 (the host-sphere Mie multiply runs apart)
template <typename T>
__global__ void __launch_bounds__(RB) post_kernel(int nslots, const int* slot_sphere, const int* order, const int* offset,
                                                  const int* mie_offset, const cpx<T>* an, const cpx<T>* p, const cpx<T>* w,
                                                  const cpx<T>* y0, const cpx<T>* y1, cpx<T>* cap, cpx<T>* caw, double* part)
{
    double acc[2] = {0.0, 0.0};
    for (int e = blockIdx.x * RB + threadIdx.x; e < nslots; e += gridDim.x * RB) {
        int i = slot_sphere[e];
        int L = order[i], hb = L * (L + 2);
        int loc = e - offset[i] / 2;
        int row = loc % (L + 2), col = loc / (L + 2) + 1;
        int n = (row <= col) ? col : row - 1;
        int b0 = offset[i] + loc, b1 = b0 + hb;
        cpx<T> u0 = y0[b0], u1 = y0[b1];
        cpx<T> m0 = u0, m1 = u1;
        if (an) {
            const cpx<T>* A = an + mie_offset[i] + 4 * (n - 1);
            m0 = A[0] * u0 + A[2] * u1;
            m1 = A[1] * u0 + A[3] * u1;
        }
        cpx<T> c0 = p[b0] - m0, c1 = p[b1] - m1;
        cap[b0] = c0;
        cap[b1] = c1;
        caw[b0] = w[b0] - cj(y1[b0]);
        caw[b1] = w[b1] - cj(y1[b1]);
        cpx<double> w0 = up(w[b0]), w1 = up(w[b1]), d0 = up(c0), d1 = up(c1);
        acc[0] += w0.x * d0.x + w0.y * d0.y + w1.x * d1.x + w1.y * d1.y;
        acc[1] += w0.x * d0.y - w0.y * d0.x + w1.x * d1.y - w1.y * d1.x;
    }
    block_reduce_store<2>(acc, part + 2 * blockIdx.x);
}

// Initial residual: cr = b - x + M*y0 ; cq = conj(cr) ; cw = cq ; cp = cr.
// Partials: sum cr*cr (complex, no conjugate) and sum |b|^2.  an == null:
// y0 already holds M*y0.
template <typename T>
__global__ void __launch_bounds__(RB) init_kernel(int nslots, const int* slot_sphere, const int* order, const int* offset,
                                                  const int* mie_offset, const cpx<T>* an, const cpx<T>* b, const cpx<T>* x,
                                                  const cpx<T>* y0, int have_y, cpx<T>* r, cpx<T>* p, cpx<T>* w, cpx<T>* q,
                                                  double* part)
{
    double acc[3] = {0.0, 0.0, 0.0};
    for (int e = blockIdx.x * RB + threadIdx.x; e < nslots; e += gridDim.x * RB) {
        int i = slot_sphere[e];
        int L = order[i], hb = L * (L + 2);
        int loc = e - offset[i] / 2;
        int row = loc % (L + 2), col = loc / (L + 2) + 1;
        int n = (row <= col) ? col : row - 1;
        int bb[2] = {offset[i] + loc, offset[i] + loc + hb};
        cpx<T> m[2] = {mk((T)0, (T)0), mk((T)0, (T)0)};
        if (have_y) {
            cpx<T> u0 = y0[bb[0]], u1 = y0[bb[1]];
            m[0] = u0;
            m[1] = u1;
            if (an) {
                const cpx<T>* A = an + mie_offset[i] + 4 * (n - 1);
                m[0] = A[0] * u0 + A[2] * u1;
                m[1] = A[1] * u0 + A[3] * u1;
            }
        }
        for (int h = 0; h < 2; h++) {
            int k = bb[h];
            cpx<T> bv = b[k];
            cpx<T> rv = have_y ? (bv - x[k]) + m[h] : bv;
            r[k] = rv;
            p[k] = rv;
            q[k] = cj(rv);
            w[k] = cj(rv);
            cpx<double> rd = up(rv), bd = up(bv);
            acc[0] += rd.x * rd.x - rd.y * rd.y;
            acc[1] += 2.0 * rd.x * rd.y;
            acc[2] += bd.x * bd.x + bd.y * bd.y;
        }
    }
    block_reduce_store<3>(acc, part + 3 * blockIdx.x);
}

// x += a p ; r -= a cap ; q -= conj(a) caw ; partials sum conj(q)*r, sum |r|^2
template <typename T>
__global__ void __launch_bounds__(RB) upd1_kernel(int n, const BicgScalars* sc, cpx<T>* x, cpx<T>* r, cpx<T>* q, const cpx<T>* p,
                                                  const cpx<T>* cap, const cpx<T>* caw, double* part)
{
    double acc[3] = {0.0, 0.0, 0.0};
    if (!sc->breakdown) {
        cpx<T> a = mk((T)sc->alpha[0], (T)sc->alpha[1]);
        cpx<T> ac = cj(a);
        for (int k = blockIdx.x * RB + threadIdx.x; k < n; k += gridDim.x * RB) {
            x[k] = x[k] + a * p[k];
            cpx<T> rv = r[k] - a * cap[k];
            cpx<T> qv = q[k] - ac * caw[k];
            r[k] = rv;
            q[k] = qv;
            cpx<double> rd = up(rv), qd = up(qv);
            acc[0] += qd.x * rd.x + qd.y * rd.y;
            acc[1] += qd.x * rd.y - qd.y * rd.x;
            acc[2] += rd.x * rd.x + rd.y * rd.y;
        }
    }
    block_reduce_store<3>(acc, part + 3 * blockIdx.x);
}

// p = r + b p ; w = q + conj(b) w   (skipped once the system stopped)
template <typename T>
__global__ void __launch_bounds__(RB) upd2_kernel(int n, const BicgScalars* sc, cpx<T>* p, cpx<T>* w, const cpx<T>* r, const cpx<T>* q)
{
    if (sc->stop || sc->breakdown) return;
    cpx<T> b = mk((T)sc->beta[0], (T)sc->beta[1]);
    cpx<T> bc = cj(b);
    for (int k = blockIdx.x * RB + threadIdx.x; k < n; k += gridDim.x * RB) {
        p[k] = r[k] + b * p[k];
        w[k] = q[k] + bc * w[k];
    }
}

// mode 0: after init   (csk = sum cr*cr, enorm = sum |b|^2; stop if csk == 0)
// mode 1: after post   (cak = sum conj(w) cap; alpha = csk/cak or breakdown)
// mode 2: after upd1   (csk2, eerr; stop test; beta = csk2/csk; csk = csk2)
__global__ void fin_kernel(int mode, int nparts, const double* part, BicgScalars* sc, double eps, int normalize)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int K = (mode == 1) ? 2 : 3;
    double s[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < nparts; b++)
        for (int k = 0; k < K; k++) s[k] += part[K * b + k];
    if (mode == 0) {
        sc->csk[0] = s[0];
        sc->csk[1] = s[1];
        sc->enorm = normalize ? s[2] : 1.0;
        sc->stop = (s[0] == 0.0 && s[1] == 0.0) ? 1 : 0;
        sc->breakdown = 0;
        sc->eerr = 0.0;
    } else if (mode == 1) {
        zd cak = mk(s[0], s[1]);
        if (cabsd(cak) != 0.0) {
            zd a = cdiv(mk(sc->csk[0], sc->csk[1]), cak);
            sc->alpha[0] = a.x;
            sc->alpha[1] = a.y;
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

// partials sum conj(q) r, sum |r|^2 (residual replacement)
template <typename T>
__global__ void __launch_bounds__(RB) rr_dot_kernel(int n, const cpx<T>* q, const cpx<T>* r, double* part)
{
    double acc[3] = {0.0, 0.0, 0.0};
    for (int k = blockIdx.x * RB + threadIdx.x; k < n; k += gridDim.x * RB) {
        cpx<double> rd = up(r[k]), qd = up(q[k]);
        acc[0] += qd.x * rd.x + qd.y * rd.y;
        acc[1] += qd.x * rd.y - qd.y * rd.x;
        acc[2] += rd.x * rd.x + rd.y * rd.y;
    }
    block_reduce_store<3>(acc, part + 3 * blockIdx.x);
}
__global__ void sum3_last_kernel(int nparts, const double* part, double* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int b = 0; b < nparts; b++) s += part[3 * b + 2];
    out[0] = s;
}

// r = b - x + M*y (FP64 true residual of the refinement loop); partials |r|^2, |b|^2
template <typename T, typename TB>
__global__ void __launch_bounds__(RB) resid_kernel(int nslots, const int* slot_sphere, const int* order, const int* offset,
                                                   const int* mie_offset, const cpx<T>* an, const cpx<T>* b, const cpx<T>* x,
                                                   const cpx<T>* y, cpx<TB>* rout, double* part)
{
    double acc[2] = {0.0, 0.0};
    for (int e = blockIdx.x * RB + threadIdx.x; e < nslots; e += gridDim.x * RB) {
        int i = slot_sphere[e];
        int L = order[i], hb = L * (L + 2);
        int loc = e - offset[i] / 2;
        int row = loc % (L + 2), col = loc / (L + 2) + 1;
        int n = (row <= col) ? col : row - 1;
        int bb[2] = {offset[i] + loc, offset[i] + loc + hb};
        const cpx<T>* A = an + mie_offset[i] + 4 * (n - 1);
        cpx<T> u0 = y[bb[0]], u1 = y[bb[1]];
        cpx<T> m[2] = {A[0] * u0 + A[2] * u1, A[1] * u0 + A[3] * u1};
        for (int h = 0; h < 2; h++) {
            int k = bb[h];
            cpx<T> rv = (b[k] - x[k]) + m[h];
            rout[k] = mk((TB)rv.x, (TB)rv.y);
            acc[0] += (double)rv.x * rv.x + (double)rv.y * rv.y;
            acc[1] += (double)b[k].x * b[k].x + (double)b[k].y * b[k].y;
        }
    }
    block_reduce_store<2>(acc, part + 2 * blockIdx.x);
}

__global__ void sum2_kernel(int nparts, const double* part, double* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s0 = 0.0, s1 = 0.0;
    for (int b = 0; b < nparts; b++) { s0 += part[2 * b]; s1 += part[2 * b + 1]; }
    out[0] = s0;
    out[1] = s1;
}

// x64 += d (lower precision correction)
template <typename TL>
__global__ void add_correction_kernel(int n, zd* x, const cpx<TL>* d)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        x[k] = x[k] + mk((double)d[k].x, (double)d[k].y);
}
template <typename T>
__global__ void conj_copy_kernel(int n, const cpx<T>* a, cpx<T>* b)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) b[k] = cj(a[k]);
}
__global__ void d2f_kernel(int n, const zd* a, zf* b)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) b[k] = mk((float)a[k].x, (float)a[k].y);
}

static int grid_for(int n, int nsm)
{
    int g = (n + RB - 1) / RB;
    int cap = nsm * 4;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return g;
}

int reduce_grid(int n, int nsm) { return grid_for(n, nsm); }

template <typename T>
void launch_post(const SlotMaps& sm, const cpx<T>* an, const cpx<T>* p, const cpx<T>* w, const cpx<T>* y0, const cpx<T>* y1,
                 cpx<T>* cap, cpx<T>* caw, double* part, BicgScalars* sc, int nsm, cudaStream_t st)
{
    int g = grid_for(sm.nslots, nsm);
    post_kernel<T><<<g, RB, 0, st>>>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, an, p, w, y0, y1, cap, caw, part);
    fin_kernel<<<1, 32, 0, st>>>(1, g, part, sc, 0.0, 1);
    launch_counter() += 2;
}
template <typename T>
void launch_init(const SlotMaps& sm, const cpx<T>* an, const cpx<T>* b, const cpx<T>* x, const cpx<T>* y0, int have_y, cpx<T>* r,
                 cpx<T>* p, cpx<T>* w, cpx<T>* q, double* part, BicgScalars* sc, int normalize, int nsm, cudaStream_t st)
{
    int g = grid_for(sm.nslots, nsm);
    init_kernel<T><<<g, RB, 0, st>>>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, an, b, x, y0, have_y, r, p, w, q, part);
    fin_kernel<<<1, 32, 0, st>>>(0, g, part, sc, 0.0, normalize);
    launch_counter() += 2;
}
template <typename T>
void launch_upd(int n, cpx<T>* x, cpx<T>* r, cpx<T>* q, cpx<T>* p, cpx<T>* w, const cpx<T>* cap, const cpx<T>* caw, double* part,
                BicgScalars* sc, double eps, int nsm, cudaStream_t st)
{
    int g = grid_for(n, nsm);
    upd1_kernel<T><<<g, RB, 0, st>>>(n, sc, x, r, q, p, cap, caw, part);
    fin_kernel<<<1, 32, 0, st>>>(2, g, part, sc, eps, 1);
    upd2_kernel<T><<<g, RB, 0, st>>>(n, sc, p, w, r, q);
    launch_counter() += 3;
}

template <typename T, typename TB>
void launch_resid(const SlotMaps& sm, const cpx<T>* an, const cpx<T>* b, const cpx<T>* x, const cpx<T>* y, cpx<TB>* rout, double* part,
                  double* out2, int nsm, cudaStream_t st)
{
    int g = grid_for(sm.nslots, nsm);
    resid_kernel<T, TB><<<g, RB, 0, st>>>(sm.nslots, sm.slot, sm.order, sm.offset, sm.mie_offset, an, b, x, y, rout, part);
    sum2_kernel<<<1, 32, 0, st>>>(g, part, out2);
    launch_counter() += 2;
}
// out[0] = sum |v|^2 (one block-reduction pass and a fixed-order finish)
void launch_rr_dot_norm(int n, const zd* v, double* part, double* out, int nsm, cudaStream_t st)
{
    int g = grid_for(n, nsm);
    rr_dot_kernel<double><<<g, RB, 0, st>>>(n, v, v, part);
    sum3_last_kernel<<<1, 32, 0, st>>>(g, part, out);
    launch_counter() += 2;
}
void launch_add_correction_f(int n, zd* x, const zf* d, cudaStream_t st) { add_correction_kernel<float><<<296, 256, 0, st>>>(n, x, d); launch_counter() += 1; }
void launch_add_correction_d(int n, zd* x, const zd* d, cudaStream_t st) { add_correction_kernel<double><<<296, 256, 0, st>>>(n, x, d); launch_counter() += 1; }
template <typename T> void launch_conj_copy(int n, const cpx<T>* a, cpx<T>* b, cudaStream_t st) { conj_copy_kernel<T><<<296, 256, 0, st>>>(n, a, b); launch_counter() += 1; }
void launch_d2f(int n, const zd* a, zf* b, cudaStream_t st) { d2f_kernel<<<296, 256, 0, st>>>(n, a, b); launch_counter() += 1; }

template void launch_post<double>(const SlotMaps&, const zd*, const zd*, const zd*, const zd*, const zd*, zd*, zd*, double*, BicgScalars*, int, cudaStream_t);
template void launch_post<float>(const SlotMaps&, const zf*, const zf*, const zf*, const zf*, const zf*, zf*, zf*, double*, BicgScalars*, int, cudaStream_t);
template void launch_init<double>(const SlotMaps&, const zd*, const zd*, const zd*, const zd*, int, zd*, zd*, zd*, zd*, double*, BicgScalars*, int, int, cudaStream_t);
template void launch_init<float>(const SlotMaps&, const zf*, const zf*, const zf*, const zf*, int, zf*, zf*, zf*, zf*, double*, BicgScalars*, int, int, cudaStream_t);
template void launch_upd<double>(int, zd*, zd*, zd*, zd*, zd*, const zd*, const zd*, double*, BicgScalars*, double, int, cudaStream_t);
template void launch_upd<float>(int, zf*, zf*, zf*, zf*, zf*, const zf*, const zf*, double*, BicgScalars*, double, int, cudaStream_t);
template void launch_resid<double, double>(const SlotMaps&, const zd*, const zd*, const zd*, const zd*, zd*, double*, double*, int, cudaStream_t);
template void launch_resid<double, float>(const SlotMaps&, const zd*, const zd*, const zd*, const zd*, zf*, double*, double*, int, cudaStream_t);
template void launch_conj_copy<double>(int, const zd*, zd*, cudaStream_t);
template void launch_conj_copy<float>(int, const zf*, zf*, cudaStream_t);
