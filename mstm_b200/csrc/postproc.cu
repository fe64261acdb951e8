// postproc.cu -- FP64 device post-processing of a solved cluster:
//   * translation orders of each sphere to the cluster origin
//     (tranordertest, december2023/mstm-modules-33.f90:1896-1942);
//   * merge to the common origin: regular (J) translation of every sphere's
//     expansion to the origin, converted from the LR to the TE/TM basis and
//     summed (merge_to_common_origin, mstm-scatprops-26.f90:447-559), and the
//     reverse translation of an origin expansion to every sphere
//     (distribute_from_common_origin, mstm-scatprops-26.f90:561-669);
//   * GSF expansion of the azimuth-averaged scattering matrix
//     (fosmexpansion, mstm-scatprops-26.f90:1820-1951);
//   * its evaluation at polar angles (fosmcalc, mstm-scatprops-26.f90:1750-1810);
//   * the scattering matrix at single directions without azimuthal averaging
//     (scatteringmatrix, mstm-scatprops-26.f90:1498-1573).
// Orders reach t_matrix_order (up to 100), so the per-sphere translation keeps
// its Wigner-d rows, Bessel values and axial blocks in global scratch.
#include "common.cuh"
#include "special.cuh"
#include "postproc.cuh"
#include "vcoupling.cuh"
#include <algorithm>

#define PP_NT 128

// vector-coupling coefficients: vc_func / vc_uprec of vcoupling.cuh

__device__ __forceinline__ zd ipow_z(int k)
{
    int e = ((k % 4) + 4) % 4;
    return (e == 0) ? mk(1.0, 0.0) : (e == 1 ? mk(0.0, 1.0) : (e == 2 ? mk(-1.0, 0.0) : mk(0.0, -1.0)));
}

// ---------------------------------------------------------------------------
// tranordertest per sphere: a warp per sphere, its lanes evaluating the
// terms of 32 consecutive orders n at a time; one lane adds them in order of
// n, exactly as the reference's loop does, and stops at the first order whose
// partial sum meets the criterion.
// ---------------------------------------------------------------------------
#define TRANORDER_WPB 4
__global__ void __launch_bounds__(32 * TRANORDER_WPB) tranorder_kernel(int nsph, const double* pos, const int* order, double ox,
                                                                       double oy, double oz, double rire, double eps, int maxt,
                                                                       VCTab tab, zd* scratch, int sstride, int* tord)
{
    __shared__ double terms[TRANORDER_WPB][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * TRANORDER_WPB + wib, nw = gridDim.x * TRANORDER_WPB;
    const int nlim = 200;
    zd* xi = scratch + ((size_t)gw * 32 + lane) * sstride;
    zd* scr = xi + (nlim + MSTMG_LMAX + 2);
    double* vc1 = (double*)(scr + (nlim + MSTMG_LMAX + 2));
    for (int i = gw; i < nsph; i += nw) {
        const int lmax = order[i];
        const double dx = pos[3 * i] - ox, dy = pos[3 * i + 1] - oy, dz = pos[3 * i + 2] - oz;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        int nmax = lmax;
        if (r != 0.0) {
            const zd z = mk(r * rire, 0.0);
            double sum = 0.0;
            int found = 0;
            for (int n0 = 1; n0 <= nlim && !found; n0 += 32) {
                const int n = n0 + lane;
                double term = 0.0;
                if (n <= nlim) {
                    mstm_cricbessel(n + lmax, z, xi, scr);
                    for (int l = 0; l <= n + lmax; l++) xi[l] = cdiv(xi[l], z) * ipow_z(l);
                    const int l = lmax;
                    const zd c = (tab.fr(n + n + 1) * tab.fr(l + l + 1)) * ipow_z(n - l);
                    vc_func(tab, -1, n, 1, l, vc1);
                    const int wmin = abs(n - l), wmax = n + l;
                    zd a = mk(0.0, 0.0), b = mk(0.0, 0.0);
                    for (int w = wmin; w <= wmax; w++) {
                        const double alnw = vc1[w] * vc1[w];
                        if ((n + l + w) % 2 == 0) a = a + alnw * xi[w];
                        else b = b + alnw * xi[w];
                    }
                    a = c * a;
                    b = c * b;
                    term = (a * cj(a) + b * cj(b)).x;
                }
                terms[wib][lane] = term;
                __syncwarp();
                if (lane == 0)
                    for (int k = 0; k < 32 && n0 + k <= nlim; k++) {
                        sum = sum + terms[wib][k];
                        if (fabs(1.0 - sum) < eps) {
                            found = n0 + k;
                            break;
                        }
                    }
                found = __shfl_sync(0xffffffffu, found, 0);
                __syncwarp();
            }
            nmax = found ? found : nlim;
            nmax = max(nmax, lmax);
        }
        if (lane == 0) tord[i] = min(nmax, maxt);
    }
}

// ---------------------------------------------------------------------------
// merge to / distribute from the common origin: CTAs over (sphere, chunk of
// MERGE_PC columns), spheres grid-strided, scratch per CTA.  Per sphere the
// translation's tables are made once -- e^{i m phi} powers, the regular
// radial functions, the Wigner-d rows (rotcoef recurrence) and the axial
// blocks of every degree m (first row and last column by the
// vector-coupling sums, the interior by the three-term recurrence, as
// axialtrancoefrecurrence fills them) -- and then applied to the chunk's
// columns together: forward rotation, axial translation, back rotation,
// each phase one barrier for all the columns.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(PP_NT) merge_kernel(MergeArgs a)
{
    const int tid = threadIdx.x;
    const int T = a.T;
    zd* base = a.scratch + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * a.scratch_stride;
    const bool dist = (a.mode == 1);
    const int p0 = blockIdx.y * MERGE_PC, np = min(MERGE_PC, a.npol - p0);
    if (np <= 0) return;
    for (int i = blockIdx.x; i < a.nsph; i += gridDim.x) {
        if (a.active && !a.active[i]) continue;   // uniform over the CTA
        const int Li = a.order[i];
        const int L = dist ? T : Li;                       // source order
        const int nt = dist ? Li : min(T, a.tord[i]);      // target order
        const int nmin = min(L, nt), nmax = max(L, nt);
        const int W = 2 * nmin + 1;
        const double sv = dist ? -1.0 : 1.0;               // translation vector: target - source
        const double rv0 = sv * (a.r0[0] - a.pos[3 * i]), rv1 = sv * (a.r0[1] - a.pos[3 * i + 1]), rv2 = sv * (a.r0[2] - a.pos[3 * i + 2]);
        const size_t soff = dist ? 0 : (size_t)a.offset[i];
        const double rr = rv0 * rv0 + rv1 * rv1 + rv2 * rv2;
        // scratch layout
        zd* xi = base;                                        // nt+L+2
        zd* hs = xi + (nmax + L + 4);                         // Bessel scratch 2*(nt+L+2)
        zd* eph = hs + 2 * (nmax + L + 4);                    // e^{i m phi}, m = -nmax..nmax
        double* D = (double*)(eph + (2 * nmax + 1));          // Wigner rows: per degree n, W x (2n+1), restricted index first
        size_t dsz = 0;
        for (int n = 0; n <= nmax; n++) dsz += (size_t)W * (2 * n + 1);
        double* dk0 = D + dsz + 1 + (nmax + 1);
        double* dk01 = dk0 + (2 * nmax + 3);
        int* dofs = (int*)(dk01 + (nmax + 2));                // offsets of D per degree, nmax + 2 ints
        zd* Zall = (zd*)(dofs + ((nmax + 3 + 3) & ~3));       // axial blocks, per degree ma: 2 x nt x L
        zd* AP = Zall + (size_t)(nmin + 1) * 2 * nt * L;      // a'(k, l, q) per column: PC x 2 x L x W
        zd* G = AP + (size_t)MERGE_PC * 2 * L * W;            // g(m, n, q) per column: PC x 2 x nt x W
        const zd* src = a.amnp;
        __syncthreads();
        if (rr < 1.0e-12) {
            // zero translation of regular functions: copy the overlapping orders (mtransfer)
            int nc = min(L, nt);
            for (int e = tid; e < np * nc * (nc + 2); e += PP_NT) {
                const int pc = e / (nc * (nc + 2)), ee = e - pc * (nc * (nc + 2));
                const int p = p0 + pc;
                int n = 1;
                while (n * (n + 2) <= ee) n++;
                int m = ee - (n * n - 1) - n;   // ee = n(n+1)-1+m ... -> m in -n..n
                zd v1 = src[(size_t)p * a.ld + soff + aidx(m, n, 0, L)];
                zd v2 = src[(size_t)p * a.ld + soff + aidx(m, n, 1, L)];
                if (dist) {
                    zd* o = a.out + (size_t)p * a.ldo + a.offset[i];
                    o[aidx(m, n, 0, nt)] = v1;
                    o[aidx(m, n, 1, nt)] = v2;
                    continue;
                }
                int s_ = aidx(m, n, 0, T);
                atomicAdd(&a.amnp0[(size_t)p * a.ld0 + s_].x, v1.x + v2.x);
                atomicAdd(&a.amnp0[(size_t)p * a.ld0 + s_].y, v1.y + v2.y);
                atomicAdd(&a.amnp0[(size_t)p * a.ld0 + s_ + T * (T + 2)].x, v1.x - v2.x);
                atomicAdd(&a.amnp0[(size_t)p * a.ld0 + s_ + T * (T + 2)].y, v1.y - v2.y);
            }
            __syncthreads();
            continue;
        }
        const double r = sqrt(rr);
        const double ct = rv2 / r;
        const zd ephi = (rv0 == 0.0 && rv1 == 0.0) ? mk(1.0, 0.0) : mk(rv0 / sqrt(rv0 * rv0 + rv1 * rv1), rv1 / sqrt(rv0 * rv0 + rv1 * rv1));
        // Bessel functions psi_n(r)/r (cricbessel), n = 0..nt+L; e^{i m phi}; degree offsets of D
        if (tid == 0) {
            zd z = mk(r * a.rimed_re, r * a.rimed_im);
            mstm_cricbessel(nt + L, z, xi, hs);
            for (int k = 0; k <= nt + L; k++) xi[k] = cdiv(xi[k], z);
        }
        if (tid == 32) {
            zd* e = eph + nmax;
            e[0] = mk(1.0, 0.0);
            for (int m = 1; m <= nmax; m++) {
                e[m] = ephi * e[m - 1];
                e[-m] = cj(e[m]);
            }
        }
        if (tid == 64) {
            int o = W;   // degree 0 occupies W x 1 but only its centre matters
            dofs[0] = 0;
            for (int n = 1; n <= nmax; n++) {
                dofs[n] = o;
                o += W * (2 * n + 1);
            }
        }
        // Wigner-d rows by the rotcoef recurrence (kmax = nmin, nmax)
        {
            double sbe = (fabs(ct) >= 1.0) ? 0.0 : sqrt(fabs((1.0 + ct) * (1.0 - ct)));
            double cbe2 = 0.5 * (1.0 + ct), sbe2 = 0.5 * (1.0 - ct);
            for (int k = tid; k < 2 * nmax + 3; k += PP_NT) { dk0[k - (nmax + 1)] = 0.0; dk01[k - (nmax + 1)] = 0.0; }
            __syncthreads();
            if (tid == 0) { dk0[0] = 1.0; D[0] = 1.0; }
            __syncthreads();
            int sgn = 1;
            double sben = 1.0;
            size_t doff = (size_t)W;
            for (int n = 1; n <= nmax; n++) {
                int kk = min(n, nmin);
                int ld = 2 * n + 1;
                double* Dn = D + doff;
                sgn = -sgn;
                sben = sben * sbe / 2.0;
                if (sben < 1.0e-30) sben = 0.0;
                double newv[4];
                int cnt = 0;
                for (int k = -n + 1 + tid; k <= n - 1; k += PP_NT) {
                    newv[cnt++] = (ct * (double)(n + n - 1) * dk0[k] - a.fnr[n - k - 1] * a.fnr[n + k - 1] * dk01[k]) / (a.fnr[n + k] * a.fnr[n - k]);
                }
                __syncthreads();
                cnt = 0;
                for (int k = -n + 1 + tid; k <= n - 1; k += PP_NT) {
                    dk01[k] = dk0[k];
                    dk0[k] = newv[cnt++];
                }
                if (tid == 0) {
                    dk0[n] = sgn * sben * a.bcofd[n];
                    dk0[-n] = sgn * dk0[n];
                    dk01[n] = 0.0;
                    dk01[-n] = 0.0;
                }
                __syncthreads();
                for (int k = -n + tid; k <= n; k += PP_NT) Dn[(0 + nmin) * ld + (k + n)] = dk0[k];
                __syncthreads();
                int im = 1;
                for (int m = 1; m <= kk; m++) {
                    im = -im;
                    double fmn = 1.0 / a.fnr[n - m + 1] / a.fnr[n + m];
                    for (int k = -n + tid; k <= n; k += PP_NT) {
                        double dkm1 = (k == -n) ? 0.0 : Dn[(m - 1 + nmin) * ld + (k - 1 + n)];
                        double dkn1 = (k == n) ? 0.0 : Dn[(m - 1 + nmin) * ld + (k + 1 + n)];
                        double v = (a.fnr[n + k] * a.fnr[n - k + 1] * cbe2 * dkm1 - a.fnr[n - k] * a.fnr[n + k + 1] * sbe2 * dkn1 -
                                    (double)k * sbe * Dn[(m - 1 + nmin) * ld + (k + n)]) * fmn;
                        Dn[(m + nmin) * ld + (k + n)] = v;
                        Dn[(-m + nmin) * ld + (-k + n)] = v * pm1(k) * im;
                    }
                    __syncthreads();
                }
                doff += (size_t)W * ld;
            }
        }
        __syncthreads();
        // axial blocks of every degree ma (regular functions), kept for all columns
        for (int ma = 0; ma <= nmin; ma++) {
            zd* Z = Zall + (size_t)ma * 2 * nt * L;
            int m1 = max(1, ma);
            int rows = nt - m1 + 1, cols = L - m1 + 1;
            // first row n = m1 and last column l = L
            for (int e = tid; e < cols + (rows - 1); e += PP_NT) {
                int n, l;
                if (e < cols) { n = m1; l = m1 + e; }
                else { n = m1 + 1 + (e - cols); l = L; }
                int wmin = abs(n - l), wmax = n + l, ml = l * (l + 1) + ma;
                zd s1 = mk(0.0, 0.0), s2 = mk(0.0, 0.0);
                for (int w = wmin; w <= wmax; w += 2) s1 = s1 + a.vcc[(n - 1) + (size_t)a.vcT * ((ml - 1) + (size_t)a.vcML * w)] * xi[w];
                for (int w = wmin + 1; w <= wmax - 1; w += 2) s2 = s2 + a.vcc[(n - 1) + (size_t)a.vcT * ((ml - 1) + (size_t)a.vcML * w)] * xi[w];
                s2 = imul(s2);
                Z[(0 * nt + (n - 1)) * L + (l - 1)] = s1 + s2;
                Z[(1 * nt + (n - 1)) * L + (l - 1)] = s1 - s2;
            }
            __syncthreads();
            if (m1 < min(nt, L)) {
                for (int n = m1; n <= nt - 1; n++) {
                    for (int e = tid; e < 2 * (L - m1); e += PP_NT) {
                        int pp = e / (L - m1), l = m1 + e % (L - m1);
                        double sp = (pp == 0) ? 1.0 : -1.0;
#define ZA(nn, ll) Z[(pp * nt + ((nn) - 1)) * L + ((ll) - 1)]
#define FC(arr, mm, ll) arr[((mm) + a.fcN) + (2 * a.fcN + 1) * ((ll) - 1)]
                        zd v = -(ZA(n, l + 1) * FC(a.fnp1, ma, l)) + imul(sp * (FC(a.fnc, ma, l) - FC(a.fnc, ma, n)) * ZA(n, l));
                        if (l >= m1 + 1) v = v + ZA(n, l - 1) * FC(a.fnm1, ma, l);
                        if (n > m1) v = v + ZA(n - 1, l) * FC(a.fnm1, ma, n);
                        double dd = FC(a.fnp1, ma, n);
                        ZA(n + 1, l) = mk(v.x / dd, v.y / dd);
#undef ZA
#undef FC
                    }
                    __syncthreads();
                }
            }
        }
        __syncthreads();
        const zd* e = eph + nmax;
        // phase (shift_op = F: e^{+i m phi} on the source) and forward rotation of degrees l <= L, every column
        for (int it = tid; it < np * 2 * L * W; it += PP_NT) {
            const int pc = it / (2 * L * W), ee = it - pc * (2 * L * W);
            int q = ee / (L * W);
            int rem = ee - q * L * W;
            int l = rem / W + 1;
            int k = rem % W - nmin;
            int n1 = min(l, nt);
            zd acc = mk(0.0, 0.0);
            if (abs(k) <= n1) {
                const double* Dl = D + dofs[l];
                const zd* x = src + (size_t)(p0 + pc) * a.ld + soff;
                for (int m = -l; m <= l; m++) acc = acc + Dl[(k + nmin) * (2 * l + 1) + (m + l)] * (x[aidx(m, l, q, L)] * e[m]);
            }
            AP[(((size_t)pc * 2 + q) * L + (l - 1)) * W + (k + nmin)] = acc;
        }
        __syncthreads();
        // g(+ma, n, p) = Z[mode p] a'(+ma) ; g(-ma, n, p) = Z[mode 1-p] a'(-ma), every degree ma and column
        {
            // items (column, ma, sign, mode, n) with n = max(1, ma) .. nt
            const int per_col = 2 * 2 * (nt + nt * nmin - (nmin * (nmin - 1)) / 2);   // 4 x sum over ma of the rows
            for (int it = tid; it < np * per_col; it += PP_NT) {
                const int pc = it / per_col;
                int rem = it - pc * per_col;
                int ma = 0;
                for (;; ma++) {
                    const int rows = nt - max(1, ma) + 1;
                    if (rem < 4 * rows) break;
                    rem -= 4 * rows;
                }
                const int m1 = max(1, ma), rows = nt - m1 + 1;
                const int sg = rem / (2 * rows);
                rem -= sg * 2 * rows;
                const int pm = rem / rows, n = m1 + rem % rows;
                if (ma == 0 && sg == 1) continue;
                const int mm = sg ? -ma : ma;
                const int pz = (ma == 0) ? 0 : (sg == 0 ? pm : 1 - pm);
                const zd* Z = Zall + (size_t)ma * 2 * nt * L;
                const zd* ap = AP + ((size_t)pc * 2 + pm) * L * W;
                zd acc = mk(0.0, 0.0);
                for (int l = m1; l <= L; l++) acc = acc + Z[(pz * nt + (n - 1)) * L + (l - 1)] * ap[(l - 1) * W + (mm + nmin)];
                G[(((size_t)pc * 2 + pm) * nt + (n - 1)) * W + (mm + nmin)] = acc;
            }
        }
        __syncthreads();
        // back rotation per target degree n, phase back, LR -> TE/TM, accumulate
        for (int it = tid; it < np * nt * (nt + 2); it += PP_NT) {
            const int pc = it / (nt * (nt + 2)), ee = it - pc * (nt * (nt + 2));
            const int p = p0 + pc;
            int n = 1;
            while (n * (n + 2) <= ee) n++;
            int k = ee - (n * n - 1) - n;   // -n..n
            int n1 = min(n, L);
            const double* Dn = D + dofs[n];
            zd gq[2];
            for (int pm = 0; pm < 2; pm++) {
                const zd* g = G + ((size_t)pc * 2 + pm) * nt * W;
                zd acc = mk(0.0, 0.0);
                for (int m = -n1; m <= n1; m++) acc = acc + Dn[(m + nmin) * (2 * n + 1) + (k + n)] * g[(n - 1) * W + (m + nmin)];
                gq[pm] = acc * e[-k];   // phase back: e^{-i k phi}
            }
            if (dist) {
                zd* od = a.out + (size_t)p * a.ldo + a.offset[i];
                od[aidx(k, n, 0, nt)] = gq[0];
                od[aidx(k, n, 1, nt)] = gq[1];
                continue;
            }
            int s_ = aidx(k, n, 0, T);
            zd* o = a.amnp0 + (size_t)p * a.ld0;
            atomicAdd(&o[s_].x, gq[0].x + gq[1].x);
            atomicAdd(&o[s_].y, gq[0].y + gq[1].y);
            atomicAdd(&o[s_ + T * (T + 2)].x, gq[0].x - gq[1].x);
            atomicAdd(&o[s_ + T * (T + 2)].y, gq[0].y - gq[1].y);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// fosmexpansion: one warp per (n, l); lanes over m, 32 at a time.  For each
// (p, q, w) the lanes' contributions go to the same few table elements, so
// the warp adds them up first (a butterfly over the lanes) and one lane
// issues the atomics into the global tables.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_allsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(32) fosm_kernel(int ntot, const zd* a0, VCTab tab, double* s00, double* s02, double* sp22, double* sm22, double* vscr)
{
  const int lane = threadIdx.x;
  double* base = vscr + ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 5 * (2 * ntot + 2);
  double* cm1p1 = base;
  double* cm1m1 = cm1p1 + (2 * ntot + 2);
  double* cmmpm = cm1m1 + (2 * ntot + 2);
  double* cmmm2pm = cmmpm + (2 * ntot + 2);
  double* cmmp2pm = cmmm2pm + (2 * ntot + 2);
  for (int nl = blockIdx.x; nl < ntot * ntot; nl += gridDim.x) {
    int n = nl / ntot + 1, l = nl % ntot + 1;
    const int nb = 2 * ntot * (ntot + 2);
    const int half = ntot * (ntot + 2);
    int wmin = abs(n - l), wmax = n + l;
    zd fnl = sqrt((double)((n + n + 1) * (l + l + 1))) * ipow_z(l - n);
    int mm = min(n, l + 2);
    // the m-independent couplings, once per (n, l)
    vc_func(tab, -1, n, 1, l, cm1p1);
    vc_func(tab, -1, n, -1, l, cm1m1);
    for (int m0 = -mm; m0 <= mm; m0 += 32) {
        const int m = m0 + lane;
        const bool act = m <= mm;
        if (act && abs(m) <= l) vc_func(tab, -m, n, m, l, cmmpm);
        else for (int w = 0; w <= n + l; w++) cmmpm[w] = 0.0;
        if (act && abs(-2 + m) <= l) vc_func(tab, -m, n, -2 + m, l, cmmm2pm);
        else for (int w = 0; w <= n + l; w++) cmmm2pm[w] = 0.0;
        if (act && abs(2 + m) <= l) vc_func(tab, -m, n, 2 + m, l, cmmp2pm);
        else for (int w = 0; w <= n + l; w++) cmmp2pm[w] = 0.0;
        double m1m = pm1(m);
        auto A = [&](int pol, int mq, int nq, int p) -> zd {
            if (!act || mq < -nq || mq > nq) return mk(0.0, 0.0);
            return a0[(size_t)pol * nb + aidx(mq, nq, 0, ntot) + (size_t)half * p];
        };
        for (int p = 1; p <= 2; p++)
            for (int q = 1; q <= 2; q++) {
                double m1mq = pm1(m + q);
                double m1mnpl = pm1(m + n + p + l);
                zd a1n = A(0, m, n, p - 1), a2n = A(1, m, n, p - 1);
                zd a1l = A(0, m, l, q - 1), a2l = A(1, m, l, q - 1);
                zd a1122 = a1n * cj(a1l) + a2n * cj(a2l);
                zd a2112 = a2n * cj(a1l) - a1n * cj(a2l);
                zd a1p2 = (a1n + imul(a2n)) * cj(A(0, m - 2, l, q - 1) - imul(A(1, m - 2, l, q - 1)));
                zd a1m2 = (a1n - imul(a2n)) * cj(A(0, m + 2, l, q - 1) + imul(A(1, m + 2, l, q - 1)));
                for (int w = wmin; w <= wmax; w++) {
                    double m1w = pm1(w);
                    bool ev = ((n + l + w + p + q) % 2 == 0);   // one parity for the whole warp
#define SS(arr, i, j) (&arr[((i) - 1) + 4 * ((j) - 1) + 16 * w])
                    // this lane's terms of the five elements (n, l, w, p, q) feeds
                    double v0, v1 = 0.0, v2 = 0.0, v3 = 0.0, v4 = 0.0;
                    if (ev) v0 = -((m1m * fnl) * a1122 * (cm1p1[w] * cmmpm[w])).x / 2.0;
                    else v0 = (imul(mk(0.5, 0.0)) * (m1m * fnl) * a2112 * (cm1p1[w] * cmmpm[w])).x;
                    if (w >= 2) {
                        if (ev) {
                            v1 = -((m1mq * a1122) * fnl * (cm1m1[w] * cmmpm[w])).x / 2.0;
                            v2 = -((m1m * a1p2) * fnl * (cm1p1[w] * cmmm2pm[w])).x / 4.0
                                 - ((m1m * a1m2) * fnl * (cm1p1[w] * cmmp2pm[w])).x / 4.0;
                        } else {
                            v1 = (imul(mk(-0.5, 0.0)) * (m1mq * a2112) * fnl * (cm1m1[w] * cmmpm[w])).y;
                            v2 = ((m1m * a1p2) * fnl * (cm1p1[w] * cmmm2pm[w])).y / 4.0
                                 - ((m1m * a1m2) * fnl * (cm1p1[w] * cmmp2pm[w])).y / 4.0;
                        }
                        v3 = -((m1mnpl * m1w * a1p2) * fnl * (cm1m1[w] * cmmm2pm[w])).x / 8.0
                             - ((m1mq * a1m2) * fnl * (cm1m1[w] * cmmp2pm[w])).x / 8.0;
                        v4 = -((m1mq * a1p2) * fnl * (cm1m1[w] * cmmm2pm[w])).x / 8.0
                             - ((m1mnpl * m1w * a1m2) * fnl * (cm1m1[w] * cmmp2pm[w])).x / 8.0;
                    }
                    v0 = warp_allsum(v0);
                    if (w >= 2) {
                        v1 = warp_allsum(v1);
                        v2 = warp_allsum(v2);
                        v3 = warp_allsum(v3);
                        v4 = warp_allsum(v4);
                    }
                    if (lane == 0) {
                        atomicAdd(ev ? SS(s00, 1, 1) : SS(s00, 4, 4), v0);
                        if (w >= 2) {
                            atomicAdd(ev ? SS(s02, 2, 1) : SS(s02, 3, 4), v1);
                            atomicAdd(ev ? SS(s02, 1, 2) : SS(s02, 4, 3), v2);
                            atomicAdd(SS(sm22, 2, 2), v3);
                            atomicAdd(SS(sp22, 2, 2), v4);
                        }
                    }
#undef SS
                }
            }
    }
  }
}

// the sign patches and the 1/(2 m_medium) factor of fosmexpansion
__global__ void fosm_patch_kernel(int ntot, double* s00, double* s02, double* sp22, double* sm22, double scale)
{
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w > 2 * ntot) return;
    double* S[4] = {s00, s02, sm22, sp22};
    for (int k = 0; k < 4; k++)
        for (int i = 3; i <= 4; i++)
            for (int j = 1; j <= i; j++) S[k][(j - 1) + 4 * (i - 1) + 16 * w] = -S[k][(j - 1) + 4 * (i - 1) + 16 * w];
    sm22[(3 - 1) + 4 * (3 - 1) + 16 * w] = -sm22[(2 - 1) + 4 * (2 - 1) + 16 * w];
    sp22[(3 - 1) + 4 * (3 - 1) + 16 * w] = sp22[(2 - 1) + 4 * (2 - 1) + 16 * w];
    for (int k = 0; k < 4; k++)
        for (int e = 0; e < 16; e++) S[k][e + 16 * w] = 0.5 * S[k][e + 16 * w] / scale;
}

// fosmcalc at each angle: one CTA per angle; rotcoef(ct, 2, 2ntot) by the
// degree recurrence, then the sum over w and the element patches
__global__ void fosmcalc_kernel(int ntot, int nang, const double* s00, const double* s02, const double* sp22,
                                const double* sm22, const double* fnr, const double* bcofd, double* dscr, double* smat)
{
    int ia = blockIdx.x;
    if (ia >= nang) return;
    const int nmax = 2 * ntot, kmax = 2;
    // polar angle as scattering_matrix_calculation forms it (input:3039-3043), pi as MSTM stores it
    double ct = cos(MSTMG_REF_PI / 180.0 * (0.0 + (180.0 - 0.0) * (double)ia / (double)(nang - 1)));
    if (ct == 1.0) ct = 0.9999999;
    if (ct == -1.0) ct = -0.9999999;
    double* dk0 = dscr + (size_t)ia * (16 * nmax + 40) + (nmax + 1);
    double* dk01 = dk0 + (2 * nmax + 3);
    double* dc = dk01 + (2 * nmax + 3);   // rows m = -2..2 of the current degree, columns k = -nmax..nmax
    const int W = 2 * nmax + 1;
#define DCR(m, k) dc[((m) + 2) * W + ((k) + nmax)]
    __shared__ double acc[16];
    if (threadIdx.x < 16) acc[threadIdx.x] = 0.0;
    double sbe = (fabs(ct) >= 1.0) ? 0.0 : sqrt(fabs((1.0 + ct) * (1.0 - ct)));
    double cbe2 = 0.5 * (1.0 + ct), sbe2 = 0.5 * (1.0 - ct);
    for (int k = threadIdx.x; k < 2 * nmax + 3; k += blockDim.x) { dk0[k - (nmax + 1)] = 0.0; dk01[k - (nmax + 1)] = 0.0; }
    __syncthreads();
    if (threadIdx.x == 0) dk0[0] = 1.0;
    __syncthreads();
    // degree 0: dc(0,0) = 1 -> the w = 0 term
    if (threadIdx.x < 16) acc[threadIdx.x] += s00[threadIdx.x] * 1.0;
    int sgn = 1;
    double sben = 1.0;
    for (int n = 1; n <= nmax; n++) {
        int kk = min(n, kmax);
        sgn = -sgn;
        sben = sben * sbe / 2.0;
        if (sben < 1.0e-30) sben = 0.0;
        double newv[8];
        int cnt = 0;
        for (int k = -n + 1 + (int)threadIdx.x; k <= n - 1; k += blockDim.x)
            newv[cnt++] = (ct * (double)(n + n - 1) * dk0[k] - fnr[n - k - 1] * fnr[n + k - 1] * dk01[k]) / (fnr[n + k] * fnr[n - k]);
        __syncthreads();
        cnt = 0;
        for (int k = -n + 1 + (int)threadIdx.x; k <= n - 1; k += blockDim.x) {
            dk01[k] = dk0[k];
            dk0[k] = newv[cnt++];
        }
        if (threadIdx.x == 0) {
            dk0[n] = sgn * sben * bcofd[n];
            dk0[-n] = sgn * dk0[n];
            dk01[n] = 0.0;
            dk01[-n] = 0.0;
        }
        __syncthreads();
        for (int k = -n + (int)threadIdx.x; k <= n; k += blockDim.x) DCR(0, k) = dk0[k];
        __syncthreads();
        int im = 1;
        for (int m = 1; m <= kk; m++) {
            im = -im;
            double fmn = 1.0 / fnr[n - m + 1] / fnr[n + m];
            for (int k = -n + (int)threadIdx.x; k <= n; k += blockDim.x) {
                double dkm1 = (k == -n) ? 0.0 : DCR(m - 1, k - 1);
                double dkn1 = (k == n) ? 0.0 : DCR(m - 1, k + 1);
                double v = (fnr[n + k] * fnr[n - k + 1] * cbe2 * dkm1 - fnr[n - k] * fnr[n + k + 1] * sbe2 * dkn1 -
                            (double)k * sbe * DCR(m - 1, k)) * fmn;
                DCR(m, k) = v;
                DCR(-m, -k) = v * pm1(k) * im;
            }
            __syncthreads();
        }
        // terms: w = n uses dc(0, n(n+1)) [k=0 column]; dc(0,n(n+1)+2), dc(+-2, n(n+1)+2) [k=2]
        if (threadIdx.x < 16) {
            int e = threadIdx.x;
            double v = s00[e + 16 * n] * DCR(0, 0);
            if (n >= 2) v += s02[e + 16 * n] * DCR(0, 2) + sp22[e + 16 * n] * DCR(2, 2) + sm22[e + 16 * n] * DCR(-2, 2);
            acc[e] += v;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double sm[16];
        for (int e = 0; e < 16; e++) sm[e] = acc[e];
#define SM(i, j) sm[((i) - 1) + 4 * ((j) - 1)]
        SM(3, 1) = -SM(3, 1);
        SM(1, 3) = -SM(1, 3);
        SM(4, 3) = -SM(4, 3);
        double temp = SM(4, 1);
        SM(4, 1) = SM(4, 2);
        SM(4, 2) = temp;
        SM(1, 2) = (SM(1, 2) + SM(2, 1)) / 2.0;
        SM(2, 1) = SM(1, 2);
        SM(3, 4) = (SM(3, 4) - SM(4, 3)) / 2.0;
        SM(4, 3) = -SM(3, 4);
#undef SM
        for (int e = 0; e < 16; e++) smat[(size_t)ia * 16 + e] = sm[e];
    }
#undef DCR
}

// scatteringmatrix (scatprops:1498-1573) with normalize_s11 = .false. at the
// directions of scattering_matrix_calculation (input:3038-3061): one CTA per
// direction.  rotcoef(ct, 1, T) advances degree by degree in shared memory;
// per degree the threads take the orders m = -n..n, form the two tau
// functions of taufunc (modules:1324-1344) and add their terms to the four
// amplitude sums, which are reduced over the CTA at the end; thread 0 forms
// the 4x4 matrix (amplitude_to_scattering_matrix, scatprops:1410-1436).
#define PS_NT 128
__global__ void __launch_bounds__(PS_NT) planesm_kernel(PlaneSmArgs a)
{
    const int ia = blockIdx.x;
    const int i = a.ldim + ia;
    if (i > a.udim) return;
    const int T = a.T;
    __shared__ double dk0s[2 * PS_TMAX + 3], dk01s[2 * PS_TMAX + 3], dcs[3 * (2 * PS_TMAX + 1)];
    __shared__ double red[8][PS_NT / 32];
    double* dk0 = dk0s + (T + 1);
    double* dk01 = dk01s + (T + 1);
    const int W = 2 * T + 1;
#define DCR(m, k) dcs[((m) + 1) * W + ((k) + T)]
    double ct = cos(MSTMG_REF_PI / 180.0 * (a.amin + (a.amax - a.amin) * (double)(i - a.ldim) / (double)(a.udim - a.ldim)));
    if (ct == 1.0) ct = 0.9999999;
    if (ct == -1.0) ct = -0.9999999;
    const double phi = (i < 0) ? a.alpha + MSTMG_REF_PI : a.alpha;
    double cphi, sphi;
    sincos(phi, &sphi, &cphi);
    const double* fnr = a.fnr;
    double sbe = (fabs(ct) >= 1.0) ? 0.0 : sqrt(fabs((1.0 + ct) * (1.0 - ct)));
    double cbe2 = 0.5 * (1.0 + ct), sbe2 = 0.5 * (1.0 - ct);
    for (int k = threadIdx.x; k < 2 * T + 3; k += blockDim.x) { dk0s[k] = 0.0; dk01s[k] = 0.0; }
    __syncthreads();
    if (threadIdx.x == 0) dk0[0] = 1.0;
    __syncthreads();
    zd sa[4];
    for (int e = 0; e < 4; e++) sa[e] = mk(0.0, 0.0);
    const size_t ld = 2 * (size_t)T * (T + 2);
    int sgn = 1;
    double sben = 1.0;
    for (int n = 1; n <= T; n++) {
        sgn = -sgn;
        sben = sben * sbe / 2.0;
        if (sben < 1.0e-30) sben = 0.0;
        double newv[(2 * PS_TMAX + PS_NT - 1) / PS_NT];
        int cnt = 0;
        for (int k = -n + 1 + (int)threadIdx.x; k <= n - 1; k += blockDim.x)
            newv[cnt++] = (ct * (double)(n + n - 1) * dk0[k] - fnr[n - k - 1] * fnr[n + k - 1] * dk01[k]) / (fnr[n + k] * fnr[n - k]);
        __syncthreads();
        cnt = 0;
        for (int k = -n + 1 + (int)threadIdx.x; k <= n - 1; k += blockDim.x) {
            dk01[k] = dk0[k];
            dk0[k] = newv[cnt++];
        }
        if (threadIdx.x == 0) {
            dk0[n] = sgn * sben * a.bcofd[n];
            dk0[-n] = sgn * dk0[n];
            dk01[n] = 0.0;
            dk01[-n] = 0.0;
        }
        __syncthreads();
        for (int k = -n + (int)threadIdx.x; k <= n; k += blockDim.x) DCR(0, k) = dk0[k];
        __syncthreads();
        {
            const double fmn = 1.0 / fnr[n] / fnr[n + 1];
            for (int k = -n + (int)threadIdx.x; k <= n; k += blockDim.x) {
                double dkm1 = (k == -n) ? 0.0 : DCR(0, k - 1);
                double dkn1 = (k == n) ? 0.0 : DCR(0, k + 1);
                double v = (fnr[n + k] * fnr[n - k + 1] * cbe2 * dkm1 - fnr[n - k] * fnr[n + k + 1] * sbe2 * dkn1 -
                            (double)k * sbe * DCR(0, k)) * fmn;
                DCR(1, k) = v;
                DCR(-1, -k) = -v * pm1(k);
            }
        }
        __syncthreads();
        // (-i)^n
        const zd cin = (n & 3) == 0 ? mk(1.0, 0.0) : (n & 3) == 1 ? mk(0.0, -1.0) : (n & 3) == 2 ? mk(-1.0, 0.0) : mk(0.0, 1.0);
        const double fnm = sqrt((double)(n + n + 1) / 2.0) / 4.0;
        for (int m = -n + (int)threadIdx.x; m <= n; m += blockDim.x) {
            const double tau[2] = {-fnm * (-DCR(-1, m) + DCR(1, m)), -fnm * (DCR(-1, m) + DCR(1, m))};
            const int m1 = (m <= -1) ? n + 1 : m, n1 = (m <= -1) ? -m : n;
            double sm_, cm_;
            sincos((double)m * phi, &sm_, &cm_);
            const zd ce = cin * mk(cm_, sm_);
            for (int p = 0; p < 2; p++) {
                const size_t ix = (size_t)aidx(m1, n1, p, T);
                const zd a1 = a.a0[ix], a2 = a.a0[ix + ld];
                zd av, bv;
                if (a.rotate) {
                    av = cphi * a1 + sphi * a2;
                    bv = sphi * a1 - cphi * a2;
                } else {
                    av = a1;
                    bv = -a2;
                }
                const zd tb = ce * bv, ta = ce * av;
                sa[0] = sa[0] + tau[1 - p] * tb;
                sa[1] = sa[1] + tau[p] * imul(ta);
                sa[2] = sa[2] + tau[p] * imul(tb);
                sa[3] = sa[3] + tau[1 - p] * ta;
            }
        }
        __syncthreads();
    }
#undef DCR
    // CTA reduction of the 8 doubles
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double v8[8] = {sa[0].x, sa[0].y, sa[1].x, sa[1].y, sa[2].x, sa[2].y, sa[3].x, sa[3].y};
    for (int e = 0; e < 8; e++) {
        double v = v8[e];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[e][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        zd s[4];
        for (int e = 0; e < 4; e++) {
            double re = 0.0, im = 0.0;
            for (int w = 0; w < PS_NT / 32; w++) { re += red[2 * e][w]; im += red[2 * e + 1][w]; }
            s[e] = (4.0 / sqrt(2.0 * (1.0 / MSTMG_REF_PI))) * mk(re, im);
        }
        zd sp[4][4];
        for (int r = 0; r < 4; r++)
            for (int q = 0; q < 4; q++) sp[r][q] = s[r] * cj(s[q]);
        double sm[16];
#define SP(r, q) sp[(r) - 1][(q) - 1]
#define SM(r, q) sm[((r) - 1) + 4 * ((q) - 1)]
        SM(1, 1) = (SP(1, 1) + SP(2, 2) + SP(3, 3) + SP(4, 4)).x;
        SM(1, 2) = (-SP(1, 1) + SP(2, 2) - SP(3, 3) + SP(4, 4)).x;
        SM(2, 1) = (-SP(1, 1) + SP(2, 2) + SP(3, 3) - SP(4, 4)).x;
        SM(2, 2) = (SP(1, 1) + SP(2, 2) - SP(3, 3) - SP(4, 4)).x;
        SM(3, 3) = 2.0 * (SP(1, 2) + SP(3, 4)).x;
        SM(3, 4) = 2.0 * (SP(2, 1) + SP(4, 3)).y;
        SM(4, 3) = 2.0 * (SP(1, 2) - SP(3, 4)).y;
        SM(4, 4) = 2.0 * (SP(1, 2) - SP(3, 4)).x;
        SM(1, 3) = 2.0 * (SP(2, 3) + SP(1, 4)).x;
        SM(3, 1) = 2.0 * (SP(2, 4) + SP(1, 3)).x;
        SM(1, 4) = -2.0 * (SP(2, 3) - SP(1, 4)).y;
        SM(4, 1) = -2.0 * (SP(4, 2) + SP(1, 3)).y;
        SM(2, 3) = -2.0 * (SP(2, 3) - SP(1, 4)).x;
        SM(3, 2) = -2.0 * (SP(2, 4) - SP(1, 3)).x;
        SM(2, 4) = -2.0 * (SP(2, 3) + SP(1, 4)).y;
        SM(4, 2) = -2.0 * (SP(4, 2) - SP(1, 3)).y;
#undef SP
#undef SM
        for (int e = 0; e < 16; e++) a.smat[(size_t)ia * 16 + e] = sm[e] / (4.0 * MSTMG_REF_PI) / a.rimed_re;
    }
}

// blocks of TRANORDER_WPB warps, at most one warp per SM's worth (148) in all
int tranorder_blocks(int nsph) { return std::max(1, (std::min(nsph, 148) + TRANORDER_WPB - 1) / TRANORDER_WPB); }
size_t tranorder_scratch(int nsph, int sstride) { return (size_t)tranorder_blocks(nsph) * TRANORDER_WPB * 32 * (size_t)sstride; }

void launch_tranorder(int nsph, const double* pos, const int* order, const double* origin, double rire, double eps, int maxt,
                      const double* bcof, const double* fnr, int nbc, zd* scratch, int sstride, int* tord, cudaStream_t st)
{
    VCTab t{bcof, fnr, nbc};
    tranorder_kernel<<<tranorder_blocks(nsph), 32 * TRANORDER_WPB, 0, st>>>(nsph, pos, order, origin[0], origin[1], origin[2], rire,
                                                                            eps, maxt, t, scratch, sstride, tord);
    launch_counter() += 1;
}

size_t merge_scratch_per_cta(int T, int L)
{
    int nmin = std::min(T, L), nmax = std::max(T, L), W = 2 * nmin + 1;
    size_t dsz = 0;
    for (int n = 0; n <= nmax; n++) dsz += (size_t)W * (2 * n + 1);
    size_t z = (size_t)(nmax + L + 4) * 3 + (2 * nmax + 1);             // xi + Bessel scratch + e^{i m phi}
    size_t dbl = dsz + 1 + 2 * (2 * nmax + 3) + 8 + (nmax + 8) / 2 + 2;  // D + dk arrays + degree offsets
    size_t zz = (size_t)(nmin + 1) * 2 * T * L + (size_t)MERGE_PC * (2 * (size_t)L * W + 2 * (size_t)T * W);
    return z + (dbl + 1) / 2 + zz + 8;                                  // in zd units
}
int merge_chunks(int npol) { return (npol + MERGE_PC - 1) / MERGE_PC; }

void launch_merge(const MergeArgs& a, int grid, cudaStream_t st)
{
    merge_kernel<<<dim3(grid, merge_chunks(a.npol)), PP_NT, 0, st>>>(a);
    launch_counter() += 1;
}

int fosm_grid(int ntot) { return std::min(ntot * ntot, 148 * 8); }
size_t fosm_scratch_doubles(int ntot) { return (size_t)fosm_grid(ntot) * 32 * 5 * (2 * ntot + 2); }
size_t fosmcalc_scratch_doubles(int ntot, int nang) { return (size_t)nang * (16 * (2 * ntot) + 40); }

void launch_fosm(int ntot, const zd* a0, const double* bcof, const double* fnr, int nbc, double* s00, double* s02, double* sp22,
                 double* sm22, double* vscr, cudaStream_t st)
{
    VCTab t{bcof, fnr, nbc};
    fosm_kernel<<<fosm_grid(ntot), 32, 0, st>>>(ntot, a0, t, s00, s02, sp22, sm22, vscr);
    fosm_patch_kernel<<<(2 * ntot + 1 + 63) / 64, 64, 0, st>>>(ntot, s00, s02, sp22, sm22, 1.0);
    launch_counter() += 2;
}

void launch_fosmcalc(int ntot, int nang, const double* s00, const double* s02, const double* sp22, const double* sm22,
                     const double* fnr, const double* bcofd, double* dscr, double* smat, cudaStream_t st)
{
    fosmcalc_kernel<<<nang, 128, 0, st>>>(ntot, nang, s00, s02, sp22, sm22, fnr, bcofd, dscr, smat);
    launch_counter() += 1;
}

void launch_planesm(const PlaneSmArgs& a, cudaStream_t st)
{
    planesm_kernel<<<a.udim - a.ldim + 1, PS_NT, 0, st>>>(a);
    launch_counter() += 1;
}
