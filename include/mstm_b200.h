/*
 * mstm_b200.h -- C ABI of the B200 (sm_100a) multiple-sphere interaction solve.
 *
 * Drop-in boundary for MSTM's solver path (dmckwski/MSTM, december2023 tree).
 * The reference has no FFI; its boundary is the Fortran subroutine interface.
 * Each entry point below replaces one Fortran routine, called from Fortran
 * through an ISO_C_BINDING interface module that declares them bind(c):
 *
 *   mstmg_ctx_create         replaces the spheredata/mie module set-up:
 *                            miecoefcalc (mstm-modules-33.f90:5301-5407) and
 *                            the sphere arrays of spheredata (mstm-modules-33.f90:5088-5131)
 *   mstmg_interaction        sphereinteraction (mstm-scatprops-26.f90:25-180)
 *   mstmg_bicg               cbicg (mstm-solver-8.f90:654-949)
 *   mstmg_planewave          sphereplanewavecoef (mstm-scatprops-26.f90:217-284)
 *   mstmg_fixed_orientation  fixedorsoln (mstm-solver-8.f90:350-569) + qtotcalc
 *                            (mstm-scatprops-26.f90:872-912)
 *
 * Conventions
 *   - Complex arrays are interleaved (re, im) doubles, i.e. Fortran complex(8)
 *     or C double _Complex; vectors use MSTM's layout: each sphere's block is
 *     a(0:L+1,1:L,1:2) column-major, blocks in sphere order; multi-column
 *     arrays are column-major with leading dimension neqns.
 *   - Pointers may be host memory or device memory (detected per call).
 *   - Every call returns an int status: 0 ok; 1 not converged (MSTM's istat=1,
 *     mstm-solver-8.f90:524); negative values are errors (see MSTMG_ERR_*),
 *     with a message from mstmg_last_error().  Nothing calls exit().
 *   - One host thread per context.  The context replaces MSTM's module globals.
 *   - Lengths are dimensionless (k = 1): a sphere's radius is its size parameter.
 */
#ifndef MSTM_B200_H
#define MSTM_B200_H
#ifdef __cplusplus
extern "C" {
#endif

#define MSTMG_OK 0
#define MSTMG_NOT_CONVERGED 1
#define MSTMG_ERR_ARG (-1)
#define MSTMG_ERR_CUDA (-2)
#define MSTMG_ERR_UNSUPPORTED (-3)
#define MSTMG_ERR_BREAKDOWN (-4)

#define MSTMG_PRECISION_FP64 0    /* drop-in: FP64 operators and BiCG, the reference's iteration */
#define MSTMG_PRECISION_MIXED 1   /* FP32 Krylov passes from FP64 true residuals (mixed_solver), systems batched */

typedef struct mstmg_ctx mstmg_ctx;

typedef struct {
    int precision;                 /* MSTMG_PRECISION_* */
    int device;                    /* CUDA device ordinal */
    double medium_re, medium_im;   /* host medium refractive index (MSTM layer_ref_index(0)); 1 in free space */
    int translation_switch_order;  /* MSTM translation_switch_order (mstm-modules-33.f90:5126), default 3 */
    double inner_eps;              /* mixed mode: squared residual reduction a GMRES cycle (or inner BiCG solve)
                                      aims at, at most (default 1e-8) */
    int max_outer;                 /* mixed mode: GMRES cycles (mixed_solver 2) or refinement steps
                                      (mixed_solver 1) at most (default 30) */
    int generic_kernel;            /* 1: always use the order-generic translation kernel (default 0) */
    int tile_ctas_per_sm;          /* tiled kernels' CTAs per SM, 1..3 caps it (0: as many as shared memory and
                                      the kernel's register budget allow: 2 for the row kernel and FP64 passes,
                                      3 for the rotation-tiled kernel's FP32 passes of 1 or 2 columns) */
    int fp32_chunk;                /* columns per chunk of FP32 tiled passes, 2 or 4 (0: chosen per context by
                                      timing one pass of each on the first pass of 4 or more columns) */
    int mixed_solver;              /* MSTMG_PRECISION_MIXED solver of the fixed-orientation and T-matrix
                                      systems: 2 restarted GMRES, FP32 Arnoldi cycles from FP64 true
                                      residuals (default; iterations then count Arnoldi steps in pairs);
                                      0 FP32 BiCG with FP64 residual replacement; 1 restarted FP32 BiCG
                                      inside FP64 refinement */
    int gmres_restart;             /* mixed_solver 2: Arnoldi steps per cycle at most (0: up to 200, fewer
                                      when a quarter of the free device memory cannot hold the basis) */
    int tile_pairs;                /* FP32 passes of clusters of one sphere order: 0 (default) the row kernel
                                      (operator rows broadcast from shared memory to the columns of up to two
                                      pairs a step, FP32 operators in row records); 1 or 2 the rotation-tiled
                                      kernel with that many pairs a step (FP32 operators in the FP64 layout) */
    int tensor_core;               /* FP32 passes of 12 or more plain columns (the T-matrix GMRES) on the
                                      tensor cores with dense TF32 hi/lo pair operators: 0 when the context
                                      qualifies (one sphere order 5..10, direct pairs) and the operators fit
                                      in a third of the free device memory (default), -1 never */
} mstmg_opts;

/* Fill opts with the defaults above. */
void mstmg_default_opts(mstmg_opts *opts);

/* Create a context for nsphere external spheres.
 * pos: 3*nsphere (x,y,z per sphere); radius: nsphere; ref_index: 2*nsphere (re,im).
 * mie_epsilon as MSTM's mie_epsilon: >0 converge orders, <0 force order ceil(-mie_epsilon).
 * Replaces miecoefcalc (mstm-modules-33.f90:5301-5407) and the spheredata set-up. */
int mstmg_ctx_create(mstmg_ctx **ctx, int nsphere, const double *pos, const double *radius, const double *ref_index,
                     double mie_epsilon, const mstmg_opts *opts);
void mstmg_ctx_destroy(mstmg_ctx *ctx);

/* Replace the sphere positions (same count, radii and indices) without
 * reallocating; operators are regenerated on the next solve. */
int mstmg_ctx_set_positions(mstmg_ctx *ctx, const double *pos);

int mstmg_neqns(const mstmg_ctx *ctx);
int mstmg_npairs(const mstmg_ctx *ctx);
/* order: nsphere sphere orders; offset: nsphere+1 sphere_offset values (complex units). */
int mstmg_sphere_orders(const mstmg_ctx *ctx, int *order, int *offset);
/* an: 2 * 4*sum(L) doubles (MSTM an_mie layout); qext, qabs: nsphere (may be NULL). */
int mstmg_mie_coefficients(const mstmg_ctx *ctx, double *an, double *qext, double *qabs);
/* (sum r^3)^.333333 as MSTM forms vol_radius (mstm-input-37.f90:1218-1225),
 * over the spheres outside every other sphere. */
double mstmg_vol_radius(const mstmg_ctx *ctx);

/* Host spheres (MSTM spheredata findhostspheres, mstm-modules-33.f90:5230-5276):
 * a sphere whose centre lies inside a larger sphere is held by the smallest
 * such sphere, sits in that sphere's refractive index, and couples to the
 * other spheres of the same host directly and to its host through the
 * regular field inside the host (external_to_internal_expansion,
 * mstm-modules-33.f90:6533-6608).  A host's equations are its own block
 * followed by the block of the field inside it (number_field_expansions 2),
 * as sphere_offset lays them out.  mstmg_ctx_create detects hosts always.
 * host (may be NULL): nsphere entries, the holding sphere (0-based) or -1.
 * Returns the number of spheres that have a host (number_host_spheres).
 * With hosts, mstmg_bicg, mstmg_fixed_orientation and mstmg_tmatrix
 * (precision FP64, or mixed with mixed_solver 2), mstmg_t_matrix_order,
 * mstmg_interaction(_ex), mstmg_planewave, mstmg_fixed_orientation_rhs,
 * mstmg_efficiencies, mstmg_scattering and the FP64 / FP32 translation
 * passes are available; the FFT path, pair shards, ensembles, the
 * tensor-core pass and mstmg_ctx_set_positions return MSTMG_ERR_UNSUPPORTED. */
int mstmg_host_spheres(const mstmg_ctx *ctx, int *host);
/* The D, U, V Mie coefficients of the host spheres (mieoa's dnp_mie, unp_mie,
 * vnp_mie, mstm-modules-33.f90:5495-5528), laid out as an (zero for spheres
 * holding no others). */
int mstmg_host_mie_coefficients(const mstmg_ctx *ctx, double *dn, double *un, double *vn);

/* sphereinteraction (mstm-scatprops-26.f90:25-180).  ain, aout: neqns x nrhs complex.
 * con_tran[r] != 0: column r gets conj((Mie*H)^T conj(x)); mie_mult[r] == 0 skips the
 * Mie multiply.  Either array may be NULL (all 0 / all 1).  initial_run != 0
 * (re)generates the stored pair operators. */
int mstmg_interaction(mstmg_ctx *ctx, int nrhs, const double *ain, double *aout, const int *con_tran, const int *mie_mult,
                      int initial_run);

/* sphereinteraction with the rest of its optional arguments
 * (mstm-scatprops-26.f90:25-27): rhs_list[r] == 0 leaves column r out (its
 * output is zero; NULL: all columns); fft_option -1 uses the context's set-up,
 * 0 / 1 demand the direct / FFT path and return MSTMG_ERR_UNSUPPORTED when the
 * context was set up the other way; store_matrix_option is accepted and ignored
 * (the operators are always stored); skip_external_translation != 0 skips the
 * pair translation, which leaves a zero interaction on this path (no host
 * spheres or plane boundaries). */
int mstmg_interaction_ex(mstmg_ctx *ctx, int nrhs, const double *ain, double *aout, const int *con_tran, const int *mie_mult,
                         int initial_run, const int *rhs_list, int fft_option, int store_matrix_option,
                         int skip_external_translation);

/* cbicg (mstm-solver-8.f90:654-949), FP64.  Solves (I - Mie*H) x = pnp from the
 * initial guess in anp; stops when ||r||^2/||pnp||^2 < eps.  iter, err as cbicg's. */
int mstmg_bicg(mstmg_ctx *ctx, int niter, double eps, const double *pnp, double *anp, int initialize, int *iter, double *err);

/* sphereplanewavecoef (mstm-scatprops-26.f90:217-284), no plane boundaries: pmnp neqns x 2. */
int mstmg_planewave(mstmg_ctx *ctx, double alpha, double sinc, int dir, double *pmnp);

/* fixedorsoln (mstm-solver-8.f90:350-569) and qtotcalc.  amnp: neqns x 2 (out);
 * qeff: 3 x 3 x nsphere (out, may be NULL); qtot: 3 x 3 (out, may be NULL):
 * [ext, abs, sca] x [unpolarised, par, perp].  maxerr/maxiter as fixedorsoln's
 * (FP64: BiCG iterations, the reference's count; mixed with mixed_solver 2:
 * Arnoldi steps in pairs, maxerr the FP64 true residual). */
int mstmg_fixed_orientation(mstmg_ctx *ctx, double alpha, double sinc, int dir, double eps, int niter, double *amnp,
                            double *qeff, double *qtot, double *maxerr, int *maxiter);

/* Scattering post-processing of a fixed-orientation solution, the free-space
 * single-origin branch of main_calling_program (mstm-input-37.f90:1159-1197,
 * 1497-1532): translation orders of each sphere to the cluster origin
 * (tranordertest, mstm-modules-33.f90:1896-1942) with trans_eps
 * (translation_epsilon) and cap max_t_order (max_t_matrix_order); the merge to
 * the common origin (merge_to_common_origin, mstm-scatprops-26.f90:447-559);
 * the GSF expansion of the azimuth-averaged scattering matrix (fosmexpansion,
 * mstm-scatprops-26.f90:1820-1951) and its values at nangles polar angles
 * evenly spaced over 0..180 degrees (fosmcalc, mstm-scatprops-26.f90:1750-1810,
 * as scattering_matrix_calculation, mstm-input-37.f90:3015-3118, calls it).
 *   amnp: neqns x 2 (the fixed_orientation output); smat: 16 x nangles
 *   (Fortran sm(4,4) per angle, may be NULL); g = s00(1,1,1)/(3 s00(1,1,0));
 *   amnp0: optional 2*T(T+2) x 2 common-origin coefficients if amnp0_cap >= 2*T(T+2). */
int mstmg_scattering(mstmg_ctx *ctx, const double *amnp, double trans_eps, int max_t_order, int nangles, double *smat, double *g,
                     int *t_matrix_order, double *amnp0, int amnp0_cap);

/* The GSF expansion of the azimuth-averaged scattering matrix of a
 * common-origin expansion (fosmexpansion, mstm-scatprops-26.f90:1820-1951):
 * coef = s00, s02, sp22, sm22 in turn, each 16 x (2T+1) (Fortran sm(4,4) per
 * degree w = 0..2T).  amnp0 as for mstmg_scattering_plane. */
int mstmg_gsf_coefficients(mstmg_ctx *ctx, int t_matrix_order, const double *amnp0, double *coef);

/* The scattering matrix of the common-origin expansion at single directions,
 * without azimuthal averaging (azimuthal_average = .false., the reference's
 * default for fixed orientation): scatteringmatrix
 * (mstm-scatprops-26.f90:1498-1573) with normalize_s11 = .false., at the
 * directions of scattering_matrix_calculation (mstm-input-37.f90:3038-3061):
 * i = ldim..udim, theta_i = amin + (amax - amin)(i - ldim)/(udim - ldim)
 * degrees, azimuth alpha + pi for i < 0 and alpha otherwise (the reference
 * takes udim = floor(180.00001/scattering_map_increment), ldim = -udim,
 * amin = -180, amax = 180).
 *   amnp0: 2T(T+2) x 2 TE/TM coefficients (mstmg_scattering's amnp0 output),
 *   T = t_matrix_order <= 200; sm: 16 x (udim - ldim + 1), Fortran sm(4,4)
 *   per direction, divided by the medium's real index as the reference does. */
int mstmg_scattering_plane(mstmg_ctx *ctx, int t_matrix_order, const double *amnp0, int ldim, int udim, double amin, double amax,
                           double alpha, int rotate_plane, double *sm);

/* Order of the cluster T matrix about the cluster origin (the mean sphere
 * position): replaces the t_matrix_order set-up of main_calling_program
 * (mstm-input-37.f90:1179-1197), tranordertest (mstm-modules-33.f90:1896-1942)
 * per sphere with trans_eps (translation_epsilon), capped at max_t_order
 * (max_t_matrix_order).  Keeps each sphere's translation order in the context
 * for mstmg_tmatrix. */
int mstmg_t_matrix_order(mstmg_ctx *ctx, double trans_eps, int max_t_order, int *t_matrix_order);

/* Replaces tmatrix_solution (mstm-solver-8.f90:22-332) with the iterative
 * solver, one process: for l = 1..t_matrix_order the 2(2l+1) unit TE/TM
 * common-origin fields of order l are distributed to the spheres
 * (distribute_from_common_origin, mstm-scatprops-26.f90:561-669), multiplied by
 * the Mie coefficients and solved together (each column stops where cbicg
 * stops it, solution_eps, max_iterations), merged back to the origin
 * (merge_to_common_origin) and stored as T-matrix columns; the order loop stops
 * after the order at which the summed extinction changes by less than
 * convergence_eps (signed difference, as the reference; <= 0 disables).
 * mstmg_t_matrix_order must have been called on the context.  With
 * MSTMG_PRECISION_MIXED the column solves are FP32 BiCG inside FP64
 * refinement.
 *   tmat: nblkt x nblkt complex, column-major, nblkt = 2 T (T+2), T =
 *     t_matrix_order: column 2(l(l+1)+k-1)+q-1, row 2(n(n+1)+m-1)+p-1, rows with
 *     n > l zero (the entries the reference's T-matrix file holds);
 *   sphere_qeff: 3 x N (ext, abs, sca) summed over the columns (the
 *     reference's sphere_qeff); qtot[3]: their area-weighted totals with
 *     Qsca = Qext + Qinc - Qabs (qtotcalc); order_used: the order kept;
 *   maxiter, maxerr: over all column solves.
 * Returns 0, MSTMG_NOT_CONVERGED (solution_status = 1) or an error. */
int mstmg_tmatrix(mstmg_ctx *ctx, int t_matrix_order, double solution_eps, double convergence_eps, int max_iterations,
                  double *tmat, double *sphere_qeff, double *qtot, int *order_used, int *maxiter, double *maxerr);

/* Orientation-averaged Qext and Qsca from a T matrix as ranorientscatmatrix
 * forms them after reading the T-matrix file (mstm-scatprops-26.f90:2031-2122):
 * entries rounded to single precision, rows of order n > l filled by the
 * T-matrix symmetry, Qext = -2/xv^2 sum Re T(q,kl,q,kl), Qsca = 2/xv^2 sum |T|^2,
 * xv = the context's volume-equivalent radius (cross_section_radius). */
int mstmg_tmatrix_qext_qsca(mstmg_ctx *ctx, int t_matrix_order, const double *tmat, double *qext, double *qsca);

/* Replaces ranorientscatmatrix (mstm-scatprops-26.f90:1963-2530, no Gaussian
 * beam) and its evaluation ranorienscatmatrixcalc (:2538-2592) as
 * main_calling_program calls them (mstm-input-37.f90:1431-1445): the GSF
 * expansion of the orientation-averaged scattering matrix from a T matrix of
 * order t_matrix_order (<= 60; layout as mstmg_tmatrix writes it), with the
 * entries rounded to single precision and the symmetric rows filled as the
 * reference's T-matrix reader does.
 *   sm, smcf: 16 x (2T+1) expansion coefficients, Fortran sm(4,4,0:2T), total
 *     and coherent part (either may be NULL); smcf(1,1,0) is the coherent
 *     scattering ratio;
 *   smat: 16 x nangles elements at theta_i = i pi/(nangles-1) (may be NULL,
 *     nangles 0 to skip). */
int mstmg_ranorient_scattering(mstmg_ctx *ctx, int t_matrix_order, const double *tmat, int nangles, double *sm, double *smcf,
                               double *smat);

/* Switch the context to MSTM's FFT translation (fft_translation_option=t;
 * node_selection, fft_translation-5.f90:654-825, with the target box spanned
 * by the sphere centres, as main_calling_program sets it up,
 * mstm-input-37.f90:1238-1261): spheres are binned in cubic cells; pairs in
 * cells within the neighbour stencil (neighbor_node_model 0/1/2: 1/7/19 cells)
 * are translated directly, all other interactions go through regular
 * expansions of order node_order about the cell centres and the node-to-node
 * outgoing translation, applied as an FFT convolution on the zero-padded
 * (2 cell_dim)^3 grid with kernels stored in single precision, as the
 * reference stores them (fft:72-336, 827-974).  d_cell > 0 fixes the cell
 * edge, otherwise cell_volume_fraction (<= 0: from the spheres' volume) sets
 * it; node_order <= 0 means -node_order + ceiling(d_cell).  Every later
 * interaction, BiCG, fixed-orientation and T-matrix call uses it (positions
 * set later rebuild it).
 *   cell_dim[3], d_cell_out, node_order_out, near_pairs: the chosen grid. */
int mstmg_fft_setup(mstmg_ctx *ctx, double cell_volume_fraction, double d_cell, int node_order, int neighbor_node_model, int *cell_dim,
                    double *d_cell_out, int *node_order_out, int *near_pairs);

/* mstmg_fixed_orientation from a caller's initial guess x0 (neqns x 2, the
 * learned warm start) instead of MSTM's Mie-solution start (fixedorsoln,
 * mstm-solver-8.f90:482-483).  Each polarisation's guess is used only if its
 * FP64 relative residual ||b - (I - M H) x0|| / ||b|| is at most
 * fallback_residual, else that polarisation starts from the Mie solution.
 * used_guess[2], guess_residual[2]: the decision and the residuals (may be
 * NULL).  No counterpart in MSTM. */
int mstmg_fixed_orientation_guess(mstmg_ctx *ctx, double alpha, double sinc, int dir, double eps, int niter, const double *x0,
                                  double fallback_residual, int *used_guess, double *guess_residual, double *amnp, double *qeff,
                                  double *qtot, double *maxerr, int *maxiter);

/* Ensembles of independent configurations in one context; no counterpart in
 * MSTM, which solves one configuration per run (its configuration_average_*
 * drivers, input:1789, 2185, loop over configurations).  Configuration c holds
 * spheres config_start[c] .. config_start[c+1]-1 (config_start[0] = 0,
 * config_start[nconfig] = nsphere, every configuration non-empty); the
 * context has no pairs between configurations, so its interaction matrix is
 * block-diagonal.  Other arguments as mstmg_ctx_create.  Entry points that
 * treat a context as one cluster (mstmg_bicg, mstmg_fixed_orientation*,
 * mstmg_scattering, mstmg_t_matrix_order, mstmg_tmatrix, mstmg_fft_setup)
 * return MSTMG_ERR_UNSUPPORTED on it; mstmg_interaction applies the
 * block-diagonal operator. */
int mstmg_ensemble_create(mstmg_ctx **ctx, int nconfig, const int *config_start, int nsphere, const double *pos, const double *radius,
                          const double *ref_index, double mie_epsilon, const mstmg_opts *opts);
/* fixedorsoln (solver:350-569) of every configuration at once: per
 * configuration and polarisation the mixed GMRES (precision mixed,
 * mixed_solver 2; MSTMG_ERR_UNSUPPORTED otherwise) from x0 = Mie f to the
 * reference's criterion ||r||^2 / ||b||^2 < eps on that configuration's own
 * system, all systems advancing together (one translation pass a step for
 * the whole ensemble).  amnp: neqns x 2; qeff: 3 x 3 x nsphere (may be NULL);
 * qtot: 3 x 3 per configuration, as qtotcalc forms it with the
 * configuration's own volume radius (may be NULL); iterations, errors:
 * 2 per configuration (polarisation fastest; may be NULL), iterations in
 * Arnoldi-step pairs.  Returns 0, or 1 when any system missed the criterion
 * within niter. */
int mstmg_ensemble_fixed_orientation(mstmg_ctx *ctx, double alpha, double sinc, int dir, double eps, int niter, double *amnp,
                                     double *qeff, double *qtot, int *iterations, double *errors);

/* Learned warm start network primitives (warmstart.cu), all on device memory
 * and the given stream; no counterpart in MSTM.
 *   gemm: C[M x N] (+)= op(A)[M x K] op(B)[K x N]; A FP32 (lda), B BF16
 *         (b_bf16 = 1) or FP32 (ldb), FP32 accumulation; op = transpose if set;
 *   bias_act: Y = act(Z + b), act 0 identity / 1 SiLU; act_back: dZ = dY act'(Z + b);
 *   colsum: db = column sums; edge_concat: rows [h_dst, h_src, ef] and its
 *   backward (atomic); scatter_add: out[dst[e]] += in[e]; gather: out[e] = in[idx[e]];
 *   mse: masked mean-square loss (*loss) and gradient; adam: Adam step on FP32
 *   weights with an optional BF16 copy; to_bf16; knn: k <= 32 nearest
 *   neighbours of each sphere within its configuration. */
int mstmg_nn_gemm(int M, int N, int K, const float *A, int lda, int transA, const void *B, int ldb, int transB, int b_bf16, float *C,
                  int ldc, int accumulate, void *stream);
int mstmg_nn_bias_act(int M, int N, const float *Z, const float *b, float *Y, int act, void *stream);
int mstmg_nn_act_back(int M, int N, const float *Z, const float *b, const float *dY, float *dZ, int act, void *stream);
int mstmg_nn_colsum(int M, int N, const float *dZ, float *db, void *stream);
int mstmg_nn_edge_concat(int E, int H, int F, const int *dst, const int *src, const float *h, const float *ef, float *Z, void *stream);
int mstmg_nn_edge_concat_back(int E, int H, int F, const int *dst, const int *src, const float *dZ, float *dh, void *stream);
int mstmg_nn_scatter_add(int E, int H, const int *dst, const float *in, float *out, void *stream);
int mstmg_nn_gather(int E, int H, const int *idx, const float *in, float *out, int accumulate, void *stream);
int mstmg_nn_mse(long long n, const float *y, const float *t, const float *mask, float msum, float *dy, double *loss, void *stream);
int mstmg_nn_adam(long long n, float *p, const float *g, float *m, float *v, void *pb, float lr, float b1, float b2, float eps, int step,
                  void *stream);
int mstmg_nn_to_bf16(long long n, const float *p, void *pb, void *stream);
int mstmg_nn_axpy(long long n, float a, const float *x, float *y, void *stream);   /* y += a x */
int mstmg_nn_knn(int n, int k, const int *cfg_start, const int *sphere_cfg, const double *pos, int *nbr, void *stream);

/* Statistics of the last solve: iterations per polarisation, refinement steps,
 * FP64 and FP32 operator passes. */
int mstmg_last_stats(const mstmg_ctx *ctx, int *iters2, int *outer, int *passes64, int *passes32);

/* Host synchronisations of the last mixed GMRES solve on the context.  The
 * two-column solves (a fixed orientation, an ensemble) run each restart
 * cycle as one CUDA graph whose Arnoldi step repeats on the device under a
 * conditional WHILE node, so they synchronise once per cycle (the FP64 true
 * residual that starts it) and once at the end. */
int mstmg_last_host_syncs(const mstmg_ctx *ctx);

/* Bytes of one FP64 (prec=0) or FP32 (prec=1) operator pass, and the
 * reference's canonical per-pass operator bytes (translation_data layout). */
int mstmg_operator_bytes(const mstmg_ctx *ctx, int prec, double *stored_bytes, double *canonical_bytes);

/* The pair translation pass alone, y = H x (external_to_external_expansion,
 * mstm-modules-33.f90:6390-6525, no Mie multiply): ncols columns (<= 256) of
 * neqns complex values, column k a conjugate-transpose product when
 * con_tran[k] != 0 (NULL: none), with the FP64 (prec 0) or FP32 (prec 1)
 * operators and kernels the solvers use, or (prec 2) the tensor-core pass
 * with dense TF32 hi/lo operators, which takes no conjugate-transpose columns
 * and returns MSTMG_ERR_UNSUPPORTED where the context does not qualify (see
 * mstmg_opts.tensor_core); FP32 results are returned widened. */
int mstmg_translation_pass(mstmg_ctx *ctx, int prec, int ncols, const int *con_tran, const double *x, double *y);

/* Diagnostic, no counterpart in the reference: runs the bounded mbarrier
 * wait that the translation kernels use on a barrier that no copy ever
 * completes, with `limit` polls per thread (1 .. 4194304, the kernels' own
 * limit), and stores the status the kernel records: MSTMG_ERR_CUDA when the
 * wait gave up.  Returns MSTMG_OK when the launch ran and the device is still
 * usable afterwards. */
int mstmg_selftest_bounded_wait(int device, int limit, int *status);

/* Time `reps` translation passes (nrhs right-hand sides, FP64 (prec 0) or
 * FP32 (prec 1) with every second column a conjugate-transpose product, or
 * (prec 2) plain FP32 columns on the tensor cores) with CUDA events on the
 * context stream; returns the average milliseconds per pass. */
int mstmg_time_translation(mstmg_ctx *ctx, int prec, int nrhs, int reps, double *ms_per_pass);

/* Run this context's work on the caller's CUDA stream (a cudaStream_t; NULL
 * restores the context's own stream).  Lets a caller time a solve with its
 * own events on the stream the kernels are launched on. */
int mstmg_set_stream(mstmg_ctx *ctx, void *stream);

/* Kernel timing: when enabled, every translation launch is bracketed by CUDA
 * events; mstmg_kernel_time returns the summed milliseconds and launch counts
 * of the FP64 and FP32 translation kernels since the last reset. */
int mstmg_set_timing(mstmg_ctx *ctx, int enable);
int mstmg_kernel_time(mstmg_ctx *ctx, double *ms64, int *n64, double *ms32, int *n32);
/* The same for the tensor-core passes (mstmg_opts.tensor_core): summed
 * milliseconds and count since the last call. */
int mstmg_kernel_time_tc(mstmg_ctx *ctx, double *ms, int *n);

/* Number of kernels this library has launched in the process so far. */
long long mstmg_kernel_launches(void);

/* Incident plane-wave coefficients for callers that cannot allocate device
 * memory: no context and no cudaMalloc.  This entry point has no counterpart
 * in the reference.  It is meant for callers that own all device memory
 * themselves (e.g. a host code with its own memory manager or a fixed
 * device-memory budget).  The same values as mstmg_planewave on a context in
 * free space: the medium's refractive index is 1 here.
 *   nsphere spheres, all of order `order` (1..16); pos: device array 3*nsphere
 *   of the current device; pmnp: device array of the current device, neqns x 2
 *   complex (neqns = nsphere*2*order*(order+2)), written in MSTM's layout;
 *   dir 1 or 2 as mstmg_planewave's; stream: a cudaStream_t or NULL.
 * Intermediate tables live in a fixed ~32 KB device array inside the library
 * (held by every GPU that loads it until the process exits).  Every call made
 * outside stream capture looks up that array's address in the current
 * context (cudaGetSymbolAddress); a call on a stream being captured reuses
 * the last address found on its device, so make the first call on each
 * device before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller.  Orders
 * above 16 are rejected with MSTMG_ERR_UNSUPPORTED; host pointers, or memory
 * of another device, with MSTMG_ERR_ARG. */
int mstmg_planewave_noalloc(int nsphere, int order, const double *pos, double alpha, double sinc, int dir, double *pmnp,
                            void *stream);

/* Single-cluster sharding over ranks (the reference's MPI partition of the
 * pair translations: pairs dealt round-robin to the ranks of the group,
 * mstm-modules-33.f90:6466-6474, and an allreduce of the results,
 * mstm-scatprops-26.f90:152-156).  After mstmg_set_pair_shard(ctx, s, n) the
 * context translates the tiles t of its pair list with t % n == s, so
 * mstmg_interaction(_ex) and mstmg_translation_pass (prec 0, 1) return this
 * shard's part of H x (times the Mie coefficients where asked; the Mie
 * multiply is linear, so the parts still sum to the whole).  The caller sums
 * the parts over its ranks and drives the iteration (mstm_b200.shard does
 * both with torch.distributed); the solver entry points (mstmg_bicg,
 * mstmg_fixed_orientation(_guess), mstmg_tmatrix) and the tensor-core pass
 * refuse a sharded context.  Contexts of one sphere order without dense
 * pairs (MSTMG_ERR_UNSUPPORTED otherwise); on the FFT path the near-pair
 * tiles are dealt and shard 0 adds the far field.  n = 1 restores the whole
 * pair set.
 * Replaces the reference's MPI task loop inside external_to_external_expansion. */
int mstmg_set_pair_shard(mstmg_ctx *ctx, int shard, int nshards);

/* Right-hand sides of the fixed-orientation system (Mie x plane wave, both
 * polarisations: neqns x 2, fixedorsoln's pmnpan, mstm-solver-8.f90:465-483)
 * and the efficiencies of a given solution amnp (neqns x 2; qeff 3 x 3 x N,
 * qtot 3 x 3, either may be NULL; qefficiencyfactors / qtotcalc): the two
 * ends of mstmg_fixed_orientation for a caller that iterates itself. */
int mstmg_fixed_orientation_rhs(mstmg_ctx *ctx, double alpha, double sinc, int dir, double *pmnpan);
int mstmg_efficiencies(mstmg_ctx *ctx, double alpha, double sinc, int dir, const double *amnp, double *qeff, double *qtot);

/* Message of the last error on this thread. */
const char *mstmg_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
