// fftpath.cu -- MSTM's FFT translation for large clusters
// (fft_translation-5.f90): near pairs go through the pair kernels; the rest
// travels sphere -> cell node (regular translation), node -> node (outgoing
// translation as a convolution on the zero-padded cell grid, evaluated with
// FFTs), node -> sphere (regular translation).
//
//   fft_j_kernel       per sphere, the dense regular translations to and from
//                      its node (gentranmatrix, vswf_type 1; the identity
//                      for translations shorter than 1e-3, the reference's
//                      zero_translation)                         fft:482-652
//   fft_hbuild_kernel  per slot of the (2 cell_dim)^3 grid, the outgoing
//                      translation matrices of the node offsets that map to
//                      it, summed in single precision in the reference's
//                      octant order (fft:901-974); a batched double FFT then
//                      gives the stored single-precision spectra
//   fft_s2n_kernel     x (shifted for conjugate-transpose columns) -> node
//                      coefficients on the padded grid (atomic adds: a cell
//                      holds several spheres)
//   fft_mul_kernel     per frequency: g(l) = sum_n H(l, n) a(n), both modes,
//                      all columns                                 fft:827-899
//   fft_n2s_kernel     node coefficients -> sphere (1/N of the inverse FFT
//                      folded in), shifted back, added to y
#include "common.cuh"
#include "gentran.cuh"
#include "fftpath.cuh"
#include "tables.h"
#include <algorithm>
#include <cmath>

void gentran_constants(int nmax, std::vector<double>& tc)
{
    mstmg::Tables tb(6 * nmax + 6);
    const int nd = nmax * (nmax + 2);
    tc.assign((size_t)nd * nd * (2 * nmax + 1), 0.0);
    std::vector<double> vc1(2 * nmax + 2), vc2(2 * nmax + 2);
    for (int l = 1; l <= nmax; l++)
        for (int n = 1; n <= nmax; n++) {
            const int wmax = n + l;
            tb.vcfunc(-1, n, 1, l, vc2.data());
            // c = -i^(n-l) sqrt(2n+1) sqrt(2l+1)
            int e0 = ((n - l) % 4 + 4) % 4;
            double ire = (e0 == 0) ? 1.0 : (e0 == 2 ? -1.0 : 0.0), iim = (e0 == 1) ? 1.0 : (e0 == 3 ? -1.0 : 0.0);
            double cre = (-ire * tb.fnr[n + n + 1]) * tb.fnr[l + l + 1], cim = (-iim * tb.fnr[n + n + 1]) * tb.fnr[l + l + 1];
            for (int k = -l; k <= l; k++) {
                const int kl = l * (l + 1) + k;
                for (int m = -n; m <= n; m++) {
                    const int mn = n * (n + 1) + m;
                    const double m1m = (m & 1) ? -1.0 : 1.0;
                    const int v = k - m;
                    tb.vcfunc(-m, n, k, l, vc1.data());
                    const int wmin = std::max(std::abs(v), std::abs(n - l));
                    for (int w = wmax; w >= wmin; w--) {
                        // i^w c exactly, then times (-1)^m, vc1(w), vc2(w) in the reference's order
                        int e = w % 4;
                        double are, aim;
                        if (e == 0) { are = cre; aim = cim; }
                        else if (e == 1) { are = -cim; aim = cre; }
                        else if (e == 2) { are = -cre; aim = -cim; }
                        else { are = cim; aim = -cre; }
                        are = ((are * m1m) * vc1[w]) * vc2[w];
                        aim = ((aim * m1m) * vc1[w]) * vc2[w];
                        tc[(size_t)(mn - 1) + (size_t)nd * ((size_t)(kl - 1) + (size_t)nd * w)] = ((wmax - w) % 2 == 0) ? are : aim;
                    }
                }
            }
        }
}

// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(FFT_NT) fft_j_kernel(FftJArgs a)
{
    __shared__ GtShared gs;
    const int i = blockIdx.x;
    if (i >= a.nsph) return;
    const int L = a.order[i], nb = L * (L + 2), No = a.No, nbN = No * (No + 2);
    double rv[3], r2 = 0.0;
    for (int m = 0; m < 3; m++) {
        int nd = a.snode[3 * i + m];   // 1-based cell
        rv[m] = a.dcell * ((double)nd - 0.5) - a.pos[3 * i + m] + a.cb[m];
        r2 += rv[m] * rv[m];
    }
    const bool ident = r2 < 1.0e-6;   // the reference's zero_translation
    zd* Jsn = a.Jsn + a.joff[i];       // nbN x nb x 2 (target node, source sphere)
    zd* Jns = a.Jns + a.joff[i];       // nb x nbN x 2
    const zd ri = mk(a.rimed_re, a.rimed_im);
    for (int pass = 0; pass < 2; pass++) {
        const int ns = pass == 0 ? L : No, nt = pass == 0 ? No : L;
        const int nbs = ns * (ns + 2), nbt = nt * (nt + 2);
        zd* out = pass == 0 ? Jsn : Jns;
        if (ident) {
            for (int e = threadIdx.x; e < nbt * nbs; e += FFT_NT) {
                int t = e % nbt, s = e / nbt;
                zd v = (t == s) ? mk(1.0, 0.0) : mk(0.0, 0.0);
                out[e] = v;
                out[e + (size_t)nbt * nbs] = v;
            }
            continue;
        }
        double xp[3] = {pass == 0 ? rv[0] : -rv[0], pass == 0 ? rv[1] : -rv[1], pass == 0 ? rv[2] : -rv[2]};
        const int wmaxt = ns + nt;
        gt_prepare(gs, a.g, xp, 1, ri, wmaxt);
        for (int e = threadIdx.x; e < nbt * nbs; e += FFT_NT) {
            int t = e % nbt, s = e / nbt;
            int m, n, k, l;
            gt_mn(s, ns, m, n);
            gt_mn(t, nt, k, l);
            zd e1, e2;
            gt_element(gs, a.g, 1, wmaxt, n, m, l, k, e1, e2);
            out[e] = e1;
            out[e + (size_t)nbt * nbs] = e2;
        }
        __syncthreads();
    }
    (void)nb;
    (void)nbN;
}

// One CTA per slot of the padded grid: the node offset that maps to the slot
// and the octants that reach it (fft_translation_initialization's loops),
// each octant's H(xp) added in single precision in octant order.
__global__ void __launch_bounds__(FFT_NT) fft_hbuild_kernel(FftHArgs a)
{
    __shared__ GtShared gs;
    const int N0 = 2 * a.cd[0], N1 = 2 * a.cd[1], N2 = 2 * a.cd[2];
    const int nslot = N0 * N1 * N2, No = a.No, nbN = No * (No + 2);
    const zd ri = mk(a.rimed_re, a.rimed_im);
    for (int slot = blockIdx.x; slot < nslot; slot += gridDim.x) {
        const int j0 = slot % N0, j1 = (slot / N0) % N1, j2 = slot / (N0 * N1);
        const int jj[3] = {j0, j1, j2};
        int off[3];
        bool okp[3], okm[3];
        for (int d = 0; d < 3; d++) {
            const int cd = a.cd[d];
            okp[d] = jj[d] <= cd;                     // is = +1: slot = offset
            okm[d] = jj[d] >= cd && jj[d] < 2 * cd;    // is = -1: slot = 2 cd - offset (offset >= 1)
            off[d] = jj[d] <= cd ? jj[d] : 2 * cd - jj[d];
        }
        // the neighbour stencil is a hole in the kernel
        bool hole = false;
        for (int q = 0; q < a.nnb; q++)
            if (off[0] == a.nbv[3 * q] && off[1] == a.nbv[3 * q + 1] && off[2] == a.nbv[3 * q + 2]) hole = true;
        // element (p, target t, source s) of this slot at ((p nbN + t) nbN + s) nslot + slot
        const int nel = 2 * nbN * nbN;
        for (int e = threadIdx.x; e < nel; e += FFT_NT) a.hr[(size_t)e * nslot + slot] = mk(0.0, 0.0);
        __syncthreads();
        if (hole) continue;
        for (int is = 0; is < 8; is++) {
            const int sx = (is & 1) ? -1 : 1, sy = (is & 2) ? -1 : 1, sz = (is & 4) ? -1 : 1;
            if ((sx > 0 ? !okp[0] : !okm[0]) || (sy > 0 ? !okp[1] : !okm[1]) || (sz > 0 ? !okp[2] : !okm[2])) continue;
            double xp[3] = {sx * a.dcell * (double)off[0], sy * a.dcell * (double)off[1], sz * a.dcell * (double)off[2]};
            gt_prepare(gs, a.g, xp, 3, ri, 2 * No);
            for (int e = threadIdx.x; e < nbN * nbN; e += FFT_NT) {
                int t = e % nbN, s = e / nbN;   // target (row l), source (column n)
                int m, n, k, l;
                gt_mn(s, No, m, n);
                gt_mn(t, No, k, l);
                zd e1, e2;
                gt_element(gs, a.g, 3, 2 * No, n, m, l, k, e1, e2);
                // complex(4) accumulation: (float)(acc + h)
                zd* h1 = &a.hr[((size_t)(0 * nbN + t) * nbN + s) * nslot + slot];
                zd* h2 = &a.hr[((size_t)(1 * nbN + t) * nbN + s) * nslot + slot];
                *h1 = mk((double)(float)(h1->x + e1.x), (double)(float)(h1->y + e1.y));
                *h2 = mk((double)(float)(h2->x + e2.x), (double)(float)(h2->y + e2.y));
            }
            __syncthreads();
        }
    }
}

__global__ void fft_round_kernel(size_t n, const zd* in, float2* out)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        out[e] = make_float2((float)in[e].x, (float)in[e].y);
}

template <typename T> struct c2 { typedef double2 t; };
template <> struct c2<float> { typedef float2 t; };

// sphere -> node: A[col][p][k][slot_i] += sum_m Jsn_i(k, m, p) (S x_i)(m, p)
template <typename T>
__global__ void __launch_bounds__(FFT_NT) fft_s2n_kernel(FftMArgs a, const cpx<T>* J, const cpx<T>* x, int ld, int ncol, unsigned contran,
                                                         cpx<T>* A)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cpx<T>* xs = reinterpret_cast<cpx<T>*>(smraw);   // ncol x 2 nb
    const int i = blockIdx.x;
    const int L = a.order[i], nb = L * (L + 2), No = a.No, nbN = No * (No + 2);
    const size_t N8 = a.N8;
    for (int e = threadIdx.x; e < ncol * 2 * nb; e += FFT_NT) {
        int c = e / (2 * nb), el = e % (2 * nb);
        int p = el / nb, idx = el % nb;
        cpx<T> v = x[(size_t)c * ld + a.offset[i] + el];
        if ((contran >> c) & 1u) {
            // shiftcoefficient(-1, -1): a'(+-m, n) = (-1)^m a(-+m, n)
            int m, n;
            gt_mn(idx, L, m, n);
            int src = (m == 0) ? idx : aidx(-m, n, 0, L);
            v = x[(size_t)c * ld + a.offset[i] + p * nb + src];
            if (m & 1) v = mk(-v.x, -v.y);
        }
        xs[e] = v;
    }
    __syncthreads();
    const cpx<T>* Ji = J + a.joff[i];
    const int slot = a.slot[i];
    for (int e = threadIdx.x; e < 2 * nbN; e += FFT_NT) {
        int p = e / nbN, k = e % nbN;
        cpx<T> acc[4];
        for (int c = 0; c < ncol; c++) acc[c] = mk((T)0, (T)0);
        for (int m = 0; m < nb; m++) {
            cpx<T> j = Ji[k + (size_t)nbN * (m + (size_t)nb * p)];
            for (int c = 0; c < ncol; c++) acc[c] = acc[c] + j * xs[c * 2 * nb + p * nb + m];
        }
        for (int c = 0; c < ncol; c++) {
            cpx<T>* dst = A + ((size_t)(c * 2 + p) * nbN + k) * N8 + slot;
            atomicAdd(&dst->x, acc[c].x);
            atomicAdd(&dst->y, acc[c].y);
        }
    }
}

// per frequency f: G[col][p][l][f] = sum_n H[p][l][n][f] A[col][p][n][f].
// Row (p, l) = blockIdx.y, frequencies over threads: every H element is read
// once, coalesced along f, and the A rows are shared through the caches by
// the 2 nbN rows of a frequency block.
template <typename T>
__global__ void __launch_bounds__(FFT_NT) fft_mul_kernel(int nbN, size_t N8, int ncol, const float2* H, const cpx<T>* A, cpx<T>* G)
{
    const int pl = blockIdx.y, p = pl / nbN, l = pl - p * nbN;
    const float2* h = H + (size_t)pl * nbN * N8;
    for (size_t f = blockIdx.x * (size_t)FFT_NT + threadIdx.x; f < N8; f += (size_t)gridDim.x * FFT_NT) {
        cpx<T> acc[4];
        for (int c = 0; c < ncol; c++) acc[c] = mk((T)0, (T)0);
        for (int n = 0; n < nbN; n++) {
            const float2 hh = h[(size_t)n * N8 + f];
            const cpx<T> hv = mk((T)hh.x, (T)hh.y);
            for (int c = 0; c < ncol; c++) acc[c] = acc[c] + hv * A[((size_t)(c * 2 + p) * nbN + n) * N8 + f];
        }
        for (int c = 0; c < ncol; c++) G[((size_t)(c * 2 + p) * nbN + l) * N8 + f] = acc[c];
    }
}

// node -> sphere: y_i += S (Jns_i g_node / N8)
template <typename T>
__global__ void __launch_bounds__(FFT_NT) fft_n2s_kernel(FftMArgs a, const cpx<T>* J, const cpx<T>* G, int ncol, unsigned contran, cpx<T>* y,
                                                         int ld)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const int i = blockIdx.x;
    const int L = a.order[i], nb = L * (L + 2), No = a.No, nbN = No * (No + 2);
    cpx<T>* gs = reinterpret_cast<cpx<T>*>(smraw);   // ncol x 2 nbN
    cpx<T>* ys = gs + 4 * 2 * nbN;                    // ncol x 2 nb
    const size_t N8 = a.N8;
    const int slot = a.slot[i];
    const T inv = (T)(1.0 / (double)N8);
    for (int e = threadIdx.x; e < ncol * 2 * nbN; e += FFT_NT) {
        int c = e / (2 * nbN), el = e % (2 * nbN);
        cpx<T> v = G[((size_t)c * 2 * nbN + el) * N8 + slot];
        gs[e] = mk(v.x * inv, v.y * inv);
    }
    __syncthreads();
    const cpx<T>* Ji = J + a.joff[i];
    for (int e = threadIdx.x; e < 2 * nb; e += FFT_NT) {
        int p = e / nb, m = e % nb;
        cpx<T> acc[4];
        for (int c = 0; c < ncol; c++) acc[c] = mk((T)0, (T)0);
        for (int k = 0; k < nbN; k++) {
            cpx<T> j = Ji[m + (size_t)nb * (k + (size_t)nbN * p)];
            for (int c = 0; c < ncol; c++) acc[c] = acc[c] + j * gs[c * 2 * nbN + p * nbN + k];
        }
        for (int c = 0; c < ncol; c++) ys[c * 2 * nb + e] = acc[c];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ncol * 2 * nb; e += FFT_NT) {
        int c = e / (2 * nb), el = e % (2 * nb);
        int p = el / nb, idx = el % nb;
        cpx<T> v = ys[e];
        if ((contran >> c) & 1u) {
            int m, n;
            gt_mn(idx, L, m, n);
            int src = (m == 0) ? idx : aidx(-m, n, 0, L);
            v = ys[c * 2 * nb + p * nb + src];
            if (m & 1) v = mk(-v.x, -v.y);
        }
        cpx<T>* dst = y + (size_t)c * ld + a.offset[i] + el;
        *dst = *dst + v;
    }
}

// ---------------------------------------------------------------------------

void launch_fft_j(const FftJArgs& a, cudaStream_t st)
{
    fft_j_kernel<<<a.nsph, FFT_NT, 0, st>>>(a);
    launch_counter() += 1;
}
void launch_fft_hbuild(const FftHArgs& a, int nsm, cudaStream_t st)
{
    int nslot = 8 * a.cd[0] * a.cd[1] * a.cd[2];
    fft_hbuild_kernel<<<std::min(nslot, nsm * 8), FFT_NT, 0, st>>>(a);
    launch_counter() += 1;
}
void launch_fft_round(size_t n, const zd* in, float2* out, cudaStream_t st)
{
    fft_round_kernel<<<(int)std::min<size_t>((n + 255) / 256, 148 * 32), 256, 0, st>>>(n, in, out);
    launch_counter() += 1;
}
template <typename T>
void launch_fft_s2n(const FftMArgs& a, const cpx<T>* J, const cpx<T>* x, int ld, int ncol, unsigned contran, cpx<T>* A, cudaStream_t st)
{
    size_t smem = sizeof(cpx<T>) * 4 * 2 * a.nbmax;
    cudaFuncSetAttribute(fft_s2n_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    fft_s2n_kernel<T><<<a.nsph, FFT_NT, smem, st>>>(a, J, x, ld, ncol, contran, A);
    launch_counter() += 1;
}
template <typename T> void launch_fft_mul(int nbN, size_t N8, int ncol, const float2* H, const cpx<T>* A, cpx<T>* G, int nsm, cudaStream_t st)
{
    const int rows = 2 * nbN;
    const int want = std::max(1, nsm * 16 / rows);   // about 16 CTAs per SM over all rows
    int g = (int)std::min<size_t>((N8 + FFT_NT - 1) / FFT_NT, (size_t)want);
    fft_mul_kernel<T><<<dim3(g, rows), FFT_NT, 0, st>>>(nbN, N8, ncol, H, A, G);
    launch_counter() += 1;
}
template <typename T>
void launch_fft_n2s(const FftMArgs& a, const cpx<T>* J, const cpx<T>* G, int ncol, unsigned contran, cpx<T>* y, int ld, cudaStream_t st)
{
    const int nbN = a.No * (a.No + 2);
    size_t smem = sizeof(cpx<T>) * 4 * 2 * (nbN + a.nbmax);
    cudaFuncSetAttribute(fft_n2s_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    fft_n2s_kernel<T><<<a.nsph, FFT_NT, smem, st>>>(a, J, G, ncol, contran, y, ld);
    launch_counter() += 1;
}

template void launch_fft_s2n<double>(const FftMArgs&, const zd*, const zd*, int, int, unsigned, zd*, cudaStream_t);
template void launch_fft_s2n<float>(const FftMArgs&, const zf*, const zf*, int, int, unsigned, zf*, cudaStream_t);
template void launch_fft_mul<double>(int, size_t, int, const float2*, const zd*, zd*, int, cudaStream_t);
template void launch_fft_mul<float>(int, size_t, int, const float2*, const zf*, zf*, int, cudaStream_t);
template void launch_fft_n2s<double>(const FftMArgs&, const zd*, const zd*, int, unsigned, zd*, int, cudaStream_t);
template void launch_fft_n2s<float>(const FftMArgs&, const zf*, const zf*, int, unsigned, zf*, int, cudaStream_t);
