/*
 * mstm_oracle.h -- CPU restatement of MSTM's multiple-sphere interaction solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product
 * (mstm_b200/libmstm_b200.so).  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  The product
 * never links, imports or calls anything here.
 *
 * It restates, in plain C99 with FP64 complex arithmetic, the Fortran-90
 * routines of dmckwski/MSTM (december2023 tree) that make up the hot path.
 * Every function cites the reference routine it follows (file:line, paths
 * relative to the MSTM project root; "modules" = december2023/mstm-modules-33.f90,
 * "scatprops" = december2023/mstm-scatprops-26.f90, "solver" =
 * december2023/mstm-solver-8.f90, "input" = december2023/mstm-input-37.f90).
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists on
 * either machine, so outputs of the reference itself cannot be produced.  The
 * reference ships no tests, golden vectors or expected outputs.  The oracle is
 * pinned by analytic identities (N=1 cluster == Mie, energy balance, Wigner-d
 * orthogonality, rotation/axial translation == the dense gentranmatrix
 * translation, BiCG == dense LU) in tests/test_oracle.py -- "parity unpinned"
 * against reference outputs.
 */
#ifndef MSTM_ORACLE_H
#define MSTM_ORACLE_H
#include <complex.h>

typedef double _Complex ocplx;
typedef struct orc_ctx orc_ctx;

/* pi exactly as the reference stores it (modules:18, a default-real literal). */
#define ORC_REF_PI 3.1415927410125732

orc_ctx *orc_create(int nsphere, const double *pos /*3*N*/, const double *radius,
                    const double *ri /*2*N re,im*/, double mie_eps, int store_matrix,
                    int nthreads);
void orc_destroy(orc_ctx *c);
int orc_neqns(const orc_ctx *c);
void orc_orders(const orc_ctx *c, int *order, int *offset, int *mie_offset);
void orc_mie_coefs(const orc_ctx *c, ocplx *an, ocplx *an_inv, double *qext, double *qabs);

void orc_sphereinteraction(orc_ctx *c, int nrhs, const ocplx *ain, ocplx *aout,
                           const int *con_tran, const int *mie_mult, int initial_run);
/* skip_external != 0: without external_to_external_expansion (the host
 * coupling alone, sphereinteraction's skip_external_translation) */
void orc_sphereinteraction_ex(orc_ctx *c, int nrhs, const ocplx *ain, ocplx *aout,
                              const int *con_tran, const int *mie_mult, int initial_run,
                              int skip_external);
/* Host spheres (findhostspheres, modules:5230-5276): host[i] is the sphere
 * holding sphere i, -1 for none; returns the number of spheres with a host.
 * A host's equations hold its scattered block and then the block of the
 * regular field inside it. */
int orc_hosts(const orc_ctx *c, int *host);
void orc_host_mie_coefs(const orc_ctx *c, ocplx *dn, ocplx *un, ocplx *vn);
int orc_cbicg(orc_ctx *c, int niter, double eps, const ocplx *pnp, ocplx *anp,
              int initialize, int *iter, double *err);
void orc_planewave(const orc_ctx *c, double alpha, double sinc, int dir, ocplx *pmnp);
int orc_fixedorsoln(orc_ctx *c, double alpha, double sinc, int dir, double eps, int niter,
                    ocplx *amnp, double *qeff, double *maxerr, int *maxiter, int direct);
void orc_qtotcalc(const orc_ctx *c, double *qeff, double *qtot);
void orc_last_iterations(const orc_ctx *c, int *iters2);
double orc_vol_radius(const orc_ctx *c);

#endif
