// mrhs.cuh -- many-system BiCG vector kernels and T-matrix helpers (mrhs.cu).
#pragma once
#include "common.cuh"
#include "bicg.cuh"

// S systems are the columns of ld x S column-major blocks.  A launch works on
// the a active systems listed in act[0..a) (device), system act[k] in grid row k.
template <typename T> struct MultiVecs {
    cpx<T> *X, *R, *P, *W, *Q, *CAP, *CAW;   // ld x S each
};

int multi_grid(int nslots, int a, int nsm);   // CTAs per system
// XP[:, k] = X[:, act[k]] for k < a, zero for a <= k < apad
template <typename T> void launch_m_gather(int ld, int a, int apad, const int* act, const cpx<T>* X, cpx<T>* XP, int nsm, cudaStream_t st);
// XP[:, 2k] = P[:, act[k]], XP[:, 2k+1] = A^T conj(W[:, act[k]]); columns 2a .. 2apad-1 zeroed
template <typename T>
void launch_m_pack(const SlotMaps& sm, const cpx<T>* an, int ld, int a, int apad, const int* act, const cpx<T>* P, const cpx<T>* W,
                   cpx<T>* XP, int nsm, cudaStream_t st);
template <typename T>
void launch_m_init(const SlotMaps& sm, const cpx<T>* an, int ld, int a, const int* act, const cpx<T>* B, const MultiVecs<T>& v,
                   const cpx<T>* YP, int have_y, double* part, BicgScalars* sc, int nsm, cudaStream_t st);
template <typename T>
void launch_m_post(const SlotMaps& sm, const cpx<T>* an, int ld, int a, const int* act, const MultiVecs<T>& v, const cpx<T>* YP,
                   double* part, BicgScalars* sc, int nsm, cudaStream_t st, unsigned* cnt = nullptr);
template <typename T>
void launch_m_upd(int ld, int a, const int* act, const MultiVecs<T>& v, double* part, BicgScalars* sc, const double* epsv, int nsm,
                  cudaStream_t st, unsigned* cnt = nullptr);   // epsv[s]: stopping threshold of system s (device)
// cnt (one zeroed counter per active position k, left zeroed): the last CTA of
// each system does the scalar finish instead of a separate launch
// the two halves of launch_m_upd for residual replacement: x, r, q update and
// the scalar finish with no stopping threshold (csk_prev kept), then p, w
template <typename T>
void launch_m_upd1(int ld, int a, const int* act, const MultiVecs<T>& v, double* part, BicgScalars* sc, int nsm, cudaStream_t st,
                   unsigned* cnt = nullptr);
template <typename T> void launch_m_upd2(int ld, int a, const int* act, const MultiVecs<T>& v, const BicgScalars* sc, int nsm, cudaStream_t st);
// residual replacement of the systems in act: csk, beta = csk / csk_prev and enorm from the replaced r
template <typename T>
void launch_m_rrfix(int ld, int a, const int* act, const MultiVecs<T>& v, double* part, BicgScalars* sc, int nsm, cudaStream_t st);
// FP64 true residual of system act[k]: Rout[:, k] (Rout[:, act[k]] when by_sys)
// = B - X + M YP[:, k] (rounded to TB); out2[2 act[k]] = |r|^2, out2[2 act[k] + 1] = |b|^2
template <typename TB>
void launch_m_resid(const SlotMaps& sm, const zd* an, int ld, int a, const int* act, const zd* B, const zd* X, const zd* YP, cpx<TB>* Rout,
                    double* part, double* out2, int nsm, cudaStream_t st, int by_sys = 0);
// X[:, dst[k]] += D[:, src[k]], k < a
template <typename TL> void launch_m_addcorr(int ld, int a, const int* dst, const int* src, zd* X, const cpx<TL>* D, cudaStream_t st);
// Y[:, k] = M X[:, k] for k < ncols (Mie multiply, idir = 1)
void launch_m_mie(const SlotMaps& sm, const zd* an, int ld, int ncols, const zd* X, zd* Y, cudaStream_t st);

// ---- restarted GMRES for many systems (FP32 vectors, FP64 sums).  Basis
//      vector i of system s at V + (s m1 + i) ld; a launch works on the a
//      systems act[0..a) (device), packed work columns by position k, basis,
//      h and norms by system s = act[k]; complex h, y as 2 doubles ----
// XP[:, k] = V_{act[k], j}, k < a; zero columns a .. apad-1
void launch_gm_gather(int ld, int m1, int j, int a, int apad, const int* act, const zf* V, zf* XP, int nsm, cudaStream_t st);
// W[:, k] = XP[:, k] - M Y[:, k]
void launch_gm_apply(const SlotMaps& sm, const zf* an, int ld, int a, const zf* XP, const zf* Y, zf* W, int nsm, cudaStream_t st);
// (len, when given: system s's vectors hold len[s] <= ld elements)
// h[i S + s] += V_{s,i}^H W[:, k] for i < kp1 (hacc too when given; both zeroed by the caller)
void launch_gm_dots(int ld, int S, int m1, int kp1, int a, const int* act, const zf* V, const zf* W, double* h, double* hacc, int nsm,
                    cudaStream_t st, const int* len = nullptr);
// W[:, k] -= sum_{i < kp1} V_{s,i} h[i S + s]; nrm[s] += |W[:, k]|^2 after it when nrm is given
void launch_gm_update(int ld, int S, int m1, int kp1, int a, const int* act, const zf* V, const double* h, zf* W, double* nrm, int nsm,
                      cudaStream_t st, const int* len = nullptr);
// V_{s,jd} = Wsrc[:, by_sys ? s : k] / sqrt(nrm[s stride]), zero when the norm is below tiny
void launch_gm_scale(int ld, int m1, int jd, int a, const int* act, int by_sys, const zf* Wsrc, const double* nrm, int stride, double tiny,
                     zf* V, int nsm, cudaStream_t st, const int* len = nullptr);
// X[:, s] += sum_{i < kp1} y[i S + s] V_{s,i} in FP64
void launch_gm_combine(int ld, int S, int m1, int kp1, int a, const int* act, const zf* V, const double* y, zd* X, int nsm, cudaStream_t st);

// ---- ensembles of independent configurations in one index space: system
//      s = 2 c + p is polarisation p (column p of ne x 2 blocks) over the
//      elements [off[s], off[s] + len[s]) of configuration c; basis vector i
//      of s at V + (s m1 + i) ldv, work column k at W + k ldv (ldv >= len) ----
// R[p, seg] = B - X + M YP (FP32); rr[2s] += |r|^2, rr[2s+1] += |b|^2 (rr zeroed by the caller)
void launch_eg_resid(const SlotMaps& sm, const zd* an, int ne, int ldv, int a, const int* act, const int* off, const int* len, const zd* B,
                     const zd* X, const zd* YP, zf* R, double* rr, int nsm, cudaStream_t st);
// V_{s,0} = R[p, seg] / sqrt(rr[2s])
void launch_eg_start(int ne, int ldv, int m1, int a, const int* act, const int* off, const int* len, const zf* R, const double* rr, double tiny,
                     zf* V, int nsm, cudaStream_t st);
// XP[p, seg] = V_{s,j} (XP zeroed by the caller)
void launch_eg_gather(int ne, int ldv, int m1, int j, int a, const int* act, const int* off, const int* len, const zf* V, zf* XP, int nsm,
                      cudaStream_t st);
// W[:, k] = (XP - M Y)[p, seg]
void launch_eg_apply(const SlotMaps& sm, const zf* an, int ne, int ldv, int a, const int* act, const int* off, const int* len, const zf* XP,
                     const zf* Y, zf* W, int nsm, cudaStream_t st);
// X[p, seg] += sum_{i < kp1} y[i S + s] V_{s,i} (FP64)
void launch_eg_combine(int ne, int ldv, int S, int m1, int kp1, int a, const int* act, const int* off, const int* len, const zf* V,
                       const double* y, zd* X, int nsm, cudaStream_t st);

// ---- Arnoldi cycles driven on the device (one CUDA graph per cycle: the
//      step under a conditional WHILE node); state in device memory ----
struct GmDevState {
    int* j;          // step index of the cycle
    int* jmax;       // steps the cycle may take
    int* alive;      // per system: still iterating in this cycle
    int* kk;         // per system: steps taken in this cycle
    int* status;     // per system: 2 when the operator was found singular
    double* target;  // per system: squared residual estimate that ends its cycle
    double* cs;      // per system: m rotation cosines
    double2* sn;     // per system: m rotation sines
    double2* g;      // per system: m + 1 least-squares right-hand side
    double2* Rm;     // per system: m rotated Hessenberg columns of m + 1
};
void launch_gm_gather_dev(int ld, int m1, int a, int apad, const int* act, const int* jp, const int* alive, const zf* V, zf* XP, int nsm,
                          cudaStream_t st);
void launch_eg_gather_dev(int ne, int ldv, int m1, int a, const int* act, const int* off, const int* len, const int* jp, const int* alive,
                          const zf* V, zf* XP, int nsm, cudaStream_t st);
void launch_gm_dots_dev(int ld, int S, int m1, int a, const int* act, const int* jp, const zf* V, const zf* W, double* h, double* hacc,
                        int nsm, cudaStream_t st, const int* len = nullptr);
void launch_gm_update_dev(int ld, int S, int m1, int a, const int* act, const int* jp, const zf* V, const double* h, zf* W, double* nrm,
                          int nsm, cudaStream_t st, const int* len = nullptr);
void launch_gm_scale_dev(int ld, int m1, int a, const int* act, const int* jp, const zf* Wsrc, const double* nrm, double tiny, zf* V,
                         int nsm, cudaStream_t st, const int* len = nullptr);
void launch_gm_givens(int S, int m, int a, const int* act, const double* h0, const double* h1, const GmDevState& d,
                      cudaGraphConditionalHandle cond, cudaStream_t st);
void launch_gm_backsolve(int S, int m, int a, const int* act, const GmDevState& d, double* y, int* kmax, cudaStream_t st);
void launch_gm_combine_dev(int ld, int S, int m1, int a, const int* act, const zf* V, const double* y, const int* kp1, zd* X, int nsm,
                           cudaStream_t st);
void launch_eg_combine_dev(int ne, int ldv, int S, int m1, int a, const int* act, const int* off, const int* len, const zf* V, const double* y,
                           const int* kp1, zd* X, int nsm, cudaStream_t st);

// ---- T matrix (tmatrix_solution, mstm-solver-8.f90:22-332) ----
// columns of order l: unit TE (q=1) / TM (q=2) field of degree k in the LR basis
void launch_tm_rhs(int l, zd* P0, cudaStream_t st);
// per-column, per-sphere efficiencies (qefficiencyfactors with npol = 1): qcol[3 (i + N c)]
void launch_tm_qeff(int nsph, int ncols, const int* order, const int* offset, const int* mie_offset, const double* radius, zd rimed,
                    const zd* an_inv, const zd* A, const zd* P, int ld, double* qcol, cudaStream_t st, const zd* G = nullptr,
                    const double* rext = nullptr);
// sphere_qeff(3,N) += sum over the columns (fixed order); qsum[0..2] = sum_i sphere_qeff r_i^2 / xv^2
void launch_tm_qsum(int nsph, int ncols, const double* qcol, const double* radius, double xv, double* sphere_qeff, double* qsum,
                    cudaStream_t st);
// T-matrix columns of order l from the merged TE/TM coefficients A0 (nb(l) x 2(2l+1))
void launch_tm_store(int l, int tmo, const zd* A0, zd* tmat, cudaStream_t st);
// orientation-averaged Qext, Qsca from the single-precision symmetrised T matrix
void launch_tm_qext_qsca(int tmo, const zd* tmat, double xv, float* tc, double* out2, cudaStream_t st);
