/*
 * mstm_oracle.c -- CPU restatement (FP64) of MSTM's multiple-sphere interaction
 * solve.  TEST INFRASTRUCTURE ONLY: the checker for the CUDA product and the
 * timed CPU baseline.  See mstm_oracle.h for the scope and parity status.
 *
 * Index conventions follow the reference exactly:
 *   - a sphere block of order L is the Fortran array a(0:L+1,1:L,1:2),
 *     column-major; degree m>=0 of order n sits at (m,n), m<0 at (n+1,-m);
 *     the mode index p (left/right helicity) is slowest (modules:2365-2377);
 *   - Mie matrices are an(2,2,L) per sphere (modules:5385-5403);
 *   - Wigner-d tables are dc(-kmax:kmax, 0:nmax*(nmax+2)) (modules:1098);
 *   - axial coefficient blocks are ordered m=0,-1,1,-2,2,... (modules:1566).
 */
#include "mstm_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef ocplx cplx;
#define CI (_Complex_I)

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }
static int iabs_(int a) { return a < 0 ? -a : a; }
static double pm1(int n) { return (n & 1) ? -1.0 : 1.0; } /* (-1)**n for any integer n */

/* ------------------------------------------------------------------------ */
/* numconstants: sqrt table and binomial roots (modules:23-113)             */
/* ------------------------------------------------------------------------ */
#define NBC 1206               /* 6*200+6: covers init(n) for n <= 200 */
static double g_fnr[2 * NBC + 1];
static double *g_bcof;         /* (NBC+1)^2 */
#define BCOF(n, l) g_bcof[(size_t)(n) * (NBC + 1) + (size_t)(l)]
#define FNR(n) g_fnr[(n)]

static void tables_init(void)
{
    if (g_bcof) return;
    g_bcof = (double *)calloc((size_t)(NBC + 1) * (NBC + 1), sizeof(double));
    g_fnr[0] = 0.0;
    for (int n = 1; n <= 2 * NBC; n++) g_fnr[n] = sqrt((double)n);
    BCOF(0, 0) = 1.0;
    for (int n = 0; n <= NBC - 1; n++) {
        for (int l = n + 1; l <= NBC; l++) {
            BCOF(n, l) = g_fnr[n + l] * BCOF(n, l - 1) / g_fnr[l];
            BCOF(l, n) = BCOF(n, l);
        }
        BCOF(n + 1, n + 1) = g_fnr[n + n + 2] * g_fnr[n + n + 1] * BCOF(n, n) / g_fnr[n + 1] / g_fnr[n + 1];
    }
}

/* ------------------------------------------------------------------------ */
/* Bessel / Hankel (modules:262-371, 873-942)                                */
/* ------------------------------------------------------------------------ */
/* envj modifies its integer argument in the reference (n=max(1,abs(n))). */
static double envj(int *n, double x)
{
    *n = imax(1, iabs_(*n));
    return 0.5 * log10(6.28 * (*n)) - (*n) * log10(1.36 * x / (*n));
}

/* msta1 (modules:873-893) */
static int msta1(double x, int mp)
{
    double a0 = fabs(x);
    int n0 = (int)(1.1 * a0) + 1;
    double f0 = envj(&n0, a0) - mp;
    int n1 = n0 + 5;
    double f1 = envj(&n1, a0) - mp;
    int nn = n1;
    for (int it = 1; it <= 20; it++) {
        nn = (int)(n1 - (n1 - n0) / (1.0 - f0 / f1));
        double f = envj(&nn, a0) - mp;
        if (iabs_(nn - n1) < 1) break;
        n0 = n1; f0 = f1; n1 = nn; f1 = f;
    }
    return nn;
}

/* msta2 (modules:907-934) */
static int msta2(double x, int n, int mp)
{
    double a0 = fabs(x);
    double hmp = 0.5 * (double)mp;
    int nt = n;
    double ejn = envj(&nt, a0);
    double obj;
    int n0;
    if (ejn <= hmp) { obj = mp; n0 = (int)(1.1 * a0); }
    else { obj = hmp + ejn; n0 = n; }
    double f0 = envj(&n0, a0) - obj;
    int n1 = n0 + 5;
    double f1 = envj(&n1, a0) - obj;
    int nn = n1;
    for (int it = 1; it <= 20; it++) {
        nn = (int)(n1 - (n1 - n0) / (1.0 - f0 / f1));
        double f = envj(&nn, a0) - obj;
        if (iabs_(nn - n1) < 1) break;
        n0 = n1; f0 = f1; n1 = nn; f1 = f;
    }
    return nn + 10;
}

/* cspherebessel: Jin's j_n(z), y_n(z) for complex z (modules:322-371) */
static void cspherebessel(int n, cplx z, cplx *csj, cplx *csy)
{
    double a0 = cabs(z);
    int nm = n;
    if (a0 < 1.0e-60) {
        for (int k = 0; k <= n; k++) { csj[k] = 0; csy[k] = -1.0e300; }
        csy[0] = 1.0;
        return;
    }
    for (int k = 0; k <= n; k++) csj[k] = 0;
    csj[0] = csin(z) / z;
    if (n >= 1) csj[1] = (csj[0] - ccos(z)) / z;
    if (n >= 2) {
        cplx csa = csj[0], csb = csj[1], cs = 0, cf0, cf1, cf = 0;
        int m = msta1(a0, 200);
        if (m < n) nm = m;
        else m = msta2(a0, n, 15);
        cf0 = 0.0;
        cf1 = 1.0 - 100;   /* the reference writes 1.0d0-100 (= -99) */
        for (int k = m; k >= 0; k--) {
            cf = (2.0 * k + 3.0) * cf1 / z - cf0;
            if (k <= nm) csj[k] = cf;
            cf0 = cf1;
            cf1 = cf;
        }
        if (cabs(csa) > cabs(csb)) cs = csa / cf;
        if (cabs(csa) <= cabs(csb)) cs = csb / cf0;
        for (int k = 0; k <= imin(nm, n); k++) csj[k] = cs * csj[k];
    }
    for (int k = 0; k <= n; k++) csy[k] = 1.0e200;
    csy[0] = -ccos(z) / z;
    if (n >= 1) csy[1] = (csy[0] - csin(z)) / z;
    for (int k = 2; k <= imin(nm, n); k++) {
        if (cabs(csj[k - 1]) > cabs(csj[k - 2]))
            csy[k] = (csj[k] * csy[k - 1] - 1.0 / (z * z)) / csj[k - 1];
        else
            csy[k] = (csj[k] * csy[k - 2] - (2.0 * k - 1.0) / (z * z * z)) / csj[k - 2];
    }
}

/* cricbessel: Riccati-Bessel psi_n(z) = z j_n(z) (modules:262-271) */
static void cricbessel(int n, cplx ds, cplx *psi)
{
    cplx *chi = (cplx *)malloc(sizeof(cplx) * (n + 1));
    cspherebessel(n, ds, psi, chi);
    for (int i = 0; i <= n; i++) psi[i] = psi[i] * ds;
    free(chi);
}

/* crichankel: Riccati-Hankel xi_n(z) (modules:281-300) */
static void crichankel(int n, cplx ds, cplx *xi)
{
    xi[0] = -CI * cexp(CI * ds);
    cplx psi0 = csin(ds);
    if (cabs(xi[0]) / cabs(psi0) < 1.0e-6) {
        if (n >= 1) xi[1] = -cexp(CI * ds) * (CI + ds) / ds;
        for (int i = 2; i <= n; i++) xi[i] = (double)(i + i + 1) / ds * xi[i - 1] - xi[i - 2];
    } else {
        cplx *psi = (cplx *)malloc(sizeof(cplx) * (n + 1));
        cplx *chi = (cplx *)malloc(sizeof(cplx) * (n + 1));
        cspherebessel(n, ds, psi, chi);
        for (int i = 1; i <= n; i++) xi[i] = (psi[i] + CI * chi[i]) * ds;
        free(psi); free(chi);
    }
}

/* ------------------------------------------------------------------------ */
/* 2x2 helpers (modules:2321-2335)                                          */
/* ------------------------------------------------------------------------ */
/* Fortran 2x2 complex stored column-major: m[s-1 + 2*(t-1)] = mat(s,t). */
#define M2(a, s, t) (a)[((s) - 1) + 2 * ((t) - 1)]
static void twobytwoinverse(const cplx *mat, cplx *imat)
{
    cplx tmat[4];
    memcpy(tmat, mat, sizeof(tmat));
    cplx det = M2(mat, 1, 1) * M2(mat, 2, 2) - M2(mat, 2, 1) * M2(mat, 1, 2);
    for (int s = 1; s <= 2; s++) {
        double ss = pm1(s);
        for (int t = 1; t <= 2; t++) {
            double st = pm1(t);
            M2(imat, s, t) = ss * st * M2(tmat, 3 - t, 3 - s) / det;
        }
    }
}
static void matmul22(const cplx *a, const cplx *b, cplx *c)
{
    cplx r[4];
    for (int i = 1; i <= 2; i++)
        for (int j = 1; j <= 2; j++)
            M2(r, i, j) = M2(a, i, 1) * M2(b, 1, j) + M2(a, i, 2) * M2(b, 2, j);
    memcpy(c, r, sizeof(r));
}

/* ------------------------------------------------------------------------ */
/* mieoa: LR-basis Mie coefficients, non-optically-active sphere in a        */
/* medium (modules:5438-5578).  qeps>0: order from the convergence test;     */
/* qeps<0: order forced to ceiling(-qeps); qeps==0: order = *nodr0.          */
/* anp/anpinv: (2,2,nodr) column-major, may be NULL.                         */
/* ------------------------------------------------------------------------ */
static void mieoa(double x, cplx ri, cplx rimed, int *nodr0, double qeps, double *qext_o,
                  double *qsca_o, double *qabs_o, cplx *anp, cplx *anpinv)
{
    cplx rii[2][2];   /* rii[p][i]: p helicity (both equal here), i=0 medium, i=1 sphere */
    rii[0][0] = rimed; rii[1][0] = rimed;
    rii[0][1] = ri; rii[1][1] = ri;
    cplx ribulk[2];
    for (int i = 0; i < 2; i++) ribulk[i] = 2.0 / (1.0 / rii[0][i] + 1.0 / rii[1][i]);
    cplx xri[2][2];
    for (int p = 0; p < 2; p++)
        for (int i = 0; i < 2; i++) xri[p][i] = x * rii[p][i];
    int nstop;
    if (qeps > 0.0) {
        /* nint(x+4.*x**(1./3.))+5. : 1./3. is a default-real (single) literal */
        double third = (double)(1.0f / 3.0f);
        nstop = (int)lround(x + 4.0 * pow(x, third)) + 5;
    } else if (qeps < 0.0) {
        nstop = (int)ceil(-qeps);
        *nodr0 = nstop;
    } else {
        nstop = *nodr0;
    }
    int nb = nstop + 1;
    cplx *psi = (cplx *)malloc(sizeof(cplx) * (nb + 1) * 4);
    cplx *xi = (cplx *)malloc(sizeof(cplx) * (nb + 1) * 4);
    double *qext1 = (double *)malloc(sizeof(double) * (nstop + 1));
#define PSI(n, p, i) psi[(n) + (nb + 1) * ((p) + 2 * (i))]
#define XI(n, p, i) xi[(n) + (nb + 1) * ((p) + 2 * (i))]
    for (int i = 0; i < 2; i++)
        for (int p = 0; p < 2; p++) {
            cricbessel(nb, xri[p][i], &PSI(0, p, i));
            crichankel(nb, xri[p][i], &XI(0, p, i));
        }
    double qsca = 0.0, qext = 0.0;
    for (int n = 1; n <= nstop; n++) {
        cplx psip[2][2], xip[2][2], psipn[2][2], xipn[2][2];
        for (int p = 0; p < 2; p++)
            for (int i = 0; i < 2; i++) {
                psip[p][i] = PSI(n - 1, p, i) - (double)n * PSI(n, p, i) / xri[p][i];
                xip[p][i] = XI(n - 1, p, i) - (double)n * XI(n, p, i) / xri[p][i];
                psipn[p][i] = PSI(n - 1, p, i) / PSI(n, p, i) - (double)n / xri[p][i];
                xipn[p][i] = XI(n - 1, p, i) / XI(n, p, i) - (double)n / xri[p][i];
            }
        cplx gmat[4], amat[4];
        for (int s = 1; s <= 2; s++) {
            double ss = pm1(s);
            for (int t = 1; t <= 2; t++) {
                double st = pm1(t);
                M2(gmat, s, t) = (ss * ribulk[0] + st * ribulk[1]) / (rii[s - 1][1] * rii[t - 1][0])
                                 * (psipn[s - 1][1] * XI(n, t - 1, 0) - ss * st * xip[t - 1][0]);
                M2(amat, s, t) = (ss * ribulk[0] + st * ribulk[1]) / (rii[s - 1][1] * rii[t - 1][0])
                                 * (psipn[s - 1][1] * PSI(n, t - 1, 0) - ss * st * psip[t - 1][0]);
            }
        }
        cplx gmatinv[4];
        twobytwoinverse(gmat, gmatinv);
        matmul22(gmatinv, amat, amat);
        for (int k = 0; k < 4; k++) amat[k] = -amat[k];
        if (anp) memcpy(anp + 4 * (n - 1), amat, sizeof(amat));
        if (anpinv) {
            cplx inv[4];
            twobytwoinverse(amat, inv);
            memcpy(anpinv + 4 * (n - 1), inv, sizeof(inv));
        }
        qext1[n] = 0.0;
        double fn1 = n + n + 1;
        for (int p = 1; p <= 2; p++) {
            for (int q = 1; q <= 2; q++) qsca = qsca + fn1 * cabs(M2(amat, p, q)) * cabs(M2(amat, p, q));
            qext1[n] = qext1[n] - fn1 * creal(M2(amat, p, p));
        }
        qext = qext + qext1[n];
    }
    int nlast = nstop;
    if (qeps > 0.0) {
        double qextt = qext;
        qext = 0.0;
        int n;
        for (n = 1; n <= nstop; n++) {
            qext = qext + qext1[n];
            double err = fabs(1.0 - qext / qextt);
            if (err < qeps || n == nstop) break;
        }
        *nodr0 = n;
        nlast = n;
    }
    (void)nlast;
    qsca = 2.0 / x / x * qsca;
    qext = 2.0 / x / x * qext;
    if (qext_o) *qext_o = qext;
    if (qsca_o) *qsca_o = qsca;
    if (qabs_o) *qabs_o = qext - qsca;
#undef PSI
#undef XI
    free(psi); free(xi); free(qext1);
}

/* The generalized Mie coefficients of a host sphere (mieoa's dnp_mie,
 * unp_mie, vnp_mie, modules:5495-5528) for orders 1..nodr: with the
 * sphere's scattered coefficients a and the regular coefficients f of the
 * field inside it, (a, f) = [[A, U], [D, V]] (g, b) for the exciting field g
 * outside and b inside (multmiecoeffmult, modules:5690-5747).  Each (2,2,nodr)
 * column-major; non-optically-active sphere. */
static void mieoa_host(double x, cplx ri, cplx rimed, int nodr, cplx *dnp, cplx *unp, cplx *vnp)
{
    cplx rii[2] = {rimed, ri};   /* region 0 outside, 1 inside; both helicities equal */
    cplx rb[2], xri[2];
    for (int i = 0; i < 2; i++) {
        rb[i] = 2.0 / (1.0 / rii[i] + 1.0 / rii[i]);
        xri[i] = x * rii[i];
    }
    int nb = nodr + 1;
    cplx *psi = (cplx *)malloc(sizeof(cplx) * (nb + 1) * 2);
    cplx *xi = (cplx *)malloc(sizeof(cplx) * (nb + 1) * 2);
    for (int i = 0; i < 2; i++) {
        cricbessel(nb, xri[i], psi + (nb + 1) * i);
        crichankel(nb, xri[i], xi + (nb + 1) * i);
    }
#define PS(n, i) psi[(n) + (nb + 1) * (i)]
#define XS(n, i) xi[(n) + (nb + 1) * (i)]
    for (int n = 1; n <= nodr; n++) {
        cplx psip[2], xip[2], psipn[2], xipn[2];
        for (int i = 0; i < 2; i++) {
            psip[i] = PS(n - 1, i) - (double)n * PS(n, i) / xri[i];
            xip[i] = XS(n - 1, i) - (double)n * XS(n, i) / xri[i];
            psipn[i] = PS(n - 1, i) / PS(n, i) - (double)n / xri[i];
            xipn[i] = XS(n - 1, i) / XS(n, i) - (double)n / xri[i];
        }
        cplx g[4], b[4], u[4], d[4], v[4];
        for (int s = 1; s <= 2; s++) {
            double ss = pm1(s);
            for (int t = 1; t <= 2; t++) {
                double st = pm1(t);
                M2(g, s, t) = (ss * rb[0] + st * rb[1]) / (rii[1] * rii[0]) * (psipn[1] * XS(n, 0) - ss * st * xip[0]);
                M2(u, s, t) = (ss * rb[1] + st * rb[1]) / (rii[1] * rii[1]) * CI / PS(n, 1);
                M2(b, s, t) = (ss * rb[1] + st * rb[0]) / (rii[0] * rii[1]) * (xipn[0] * PS(n, 1) - ss * st * psip[1]);
                M2(d, s, t) = -(ss * rb[0] + st * rb[0]) / (rii[0] * rii[0]) * CI / XS(n, 0);
                M2(v, s, t) = (ss * rb[1] + st * rb[0]) / (rii[0] * rii[1]) * (xipn[0] * XS(n, 1) - ss * st * xip[1]);
            }
        }
        cplx gi[4], bi[4];
        twobytwoinverse(g, gi);
        twobytwoinverse(b, bi);
        matmul22(gi, u, u);
        matmul22(bi, d, d);
        matmul22(bi, v, v);
        for (int k = 0; k < 4; k++) {
            unp[4 * (n - 1) + k] = -u[k];
            dnp[4 * (n - 1) + k] = -d[k];
            vnp[4 * (n - 1) + k] = -v[k];
        }
    }
#undef PS
#undef XS
    free(psi); free(xi);
}

/* ------------------------------------------------------------------------ */
/* vector coupling coefficients (modules:950-1056)                          */
/* vcn indexed 0..n+l                                                        */
/* ------------------------------------------------------------------------ */
static void vcfuncuprec(int m, int n, int k, int l, int wmax, double *vcn)
{
    int mk = iabs_(m + k), nl = iabs_(n - l), w, m1, n1, l1, k1;
    double vc1;
    (void)n1;
    if (nl >= mk) {
        w = nl;
        if (n >= l) { m1 = m; n1 = n; l1 = l; k1 = k; }
        else { m1 = k; n1 = l; k1 = m; l1 = n; }
        vc1 = pm1(k1 + l1) * BCOF(l1 + k1, w - m1 - k1) * BCOF(l1 - k1, w + m1 + k1) / BCOF(l1 + l1, w + w + 1);
    } else {
        w = mk;
        if (m + k >= 0)
            vc1 = pm1(n + m) * BCOF(n - l + w, l - k) * BCOF(l - n + w, n - m) / BCOF(w + w + 1, n + l - w);
        else
            vc1 = pm1(l + k) * BCOF(n - l + w, l + k) * BCOF(l - n + w, n + m) / BCOF(w + w + 1, n + l - w);
    }
    int w1 = w;
    vcn[w] = vc1;
    w = w1 + 1;
    mk = m + k;
    int w2 = imin(wmax, n + l);
    if (w2 > w1) {
        double t1 = 2 * w * FNR(w + w + 1) * FNR(w + w - 1)
                    / (FNR(w + mk) * FNR(w - mk) * FNR(n - l + w) * FNR(l - n + w) * FNR(n + l - w + 1) * FNR(n + l + w + 1));
        double t2;
        if (w1 == 0) t2 = 0.5 * (double)(m - k);
        else t2 = (double)((m - k) * w * (w - 1) - mk * n * (n + 1) + mk * l * (l + 1)) / (double)(2 * w * (w - 1));
        vcn[w] = t1 * t2 * vcn[w1];
    }
    for (w = w1 + 2; w <= w2; w++) {
        double t1 = 2 * w * FNR(w + w + 1) * FNR(w + w - 1)
                    / (FNR(w + mk) * FNR(w - mk) * FNR(n - l + w) * FNR(l - n + w) * FNR(n + l - w + 1) * FNR(n + l + w + 1));
        double t2 = (double)((m - k) * w * (w - 1) - mk * n * (n + 1) + mk * l * (l + 1)) / (double)(2 * w * (w - 1));
        double t3 = FNR(w - mk - 1) * FNR(w + mk - 1) * FNR(l - n + w - 1) * FNR(n - l + w - 1) * FNR(n + l - w + 2) * FNR(n + l + w)
                    / ((double)(2 * (w - 1)) * FNR(2 * w - 3) * FNR(2 * w - 1));
        vcn[w] = t1 * (t2 * vcn[w - 1] - t3 * vcn[w - 2]);
    }
}

static void vcfunc(int m, int n, int k, int l, double *vcn)
{
    for (int w = 0; w <= n + l; w++) vcn[w] = 0.0;
    int wmax = n + l;
    int wmin = imax(iabs_(n - l), iabs_(m + k));
    vcn[wmax] = BCOF(n + m, l + k) * BCOF(n - m, l - k) / BCOF(n + n, l + l);
    if (wmin == wmax) return;
    vcn[wmax - 1] = vcn[wmax] * (l * m - k * n) * FNR(2 * (l + n) - 1) / FNR(l) / FNR(n) / FNR(n + l + m + k) / FNR(n + l - m - k);
    if (wmin == wmax - 1) return;
    int mk = m + k;
    double vcmax = fabs(vcn[wmax]) + fabs(vcn[wmax - 1]);
    int w;
    for (w = wmax; w >= wmin + 2; w--) {
        double t1 = 2 * w * FNR(w + w + 1) * FNR(w + w - 1)
                    / (FNR(w + mk) * FNR(w - mk) * FNR(n - l + w) * FNR(l - n + w) * FNR(n + l - w + 1) * FNR(n + l + w + 1));
        double t2 = (double)((m - k) * w * (w - 1) - mk * n * (n + 1) + mk * l * (l + 1)) / (double)(2 * w * (w - 1));
        double t3 = FNR(w - mk - 1) * FNR(w + mk - 1) * FNR(l - n + w - 1) * FNR(n - l + w - 1) * FNR(n + l - w + 2) * FNR(n + l + w)
                    / ((double)(2 * (w - 1)) * FNR(2 * w - 3) * FNR(2 * w - 1));
        vcn[w - 2] = (t2 * vcn[w - 1] - vcn[w] / t1) / t3;
        if ((wmax - w) % 2 == 1) {
            double vctest = fabs(vcn[w - 2]) + fabs(vcn[w - 1]);
            vcmax = vcmax > vctest ? vcmax : vctest;
            double rat = vctest / vcmax;
            if (rat < 0.01) break;
        }
    }
    if (w - 2 > wmin) {
        wmax = w - 3;
        vcfuncuprec(m, n, k, l, wmax, vcn);
    }
}

/* ------------------------------------------------------------------------ */
/* axial translation constants (modules:1680-1722)                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int nmax;
    double *vcc;    /* vcc_const(nmax, nmax*(nmax+2), 0:2nmax) */
    double *fnm1, *fn, *fnp1;  /* (-nmax:nmax, 1:nmax) */
} axconst_t;
static axconst_t g_ax = {0, 0, 0, 0, 0};
#define VCC(n, ml, w) g_ax.vcc[((n) - 1) + (size_t)g_ax.nmax * (((ml) - 1) + (size_t)g_ax.nmax * (g_ax.nmax + 2) * (w))]
#define FCI(a, m, l) (a)[((m) + g_ax.nmax) + (2 * g_ax.nmax + 1) * ((l) - 1)]

static void axialtrancoefinit(int nmax)
{
    if (nmax <= g_ax.nmax) return;
    free(g_ax.vcc); free(g_ax.fnm1); free(g_ax.fn); free(g_ax.fnp1);
    g_ax.nmax = nmax;
    size_t nv = (size_t)nmax * nmax * (nmax + 2) * (2 * nmax + 1);
    g_ax.vcc = (double *)calloc(nv, sizeof(double));
    size_t nf = (size_t)(2 * nmax + 1) * nmax;
    g_ax.fnm1 = (double *)calloc(nf, sizeof(double));
    g_ax.fn = (double *)calloc(nf, sizeof(double));
    g_ax.fnp1 = (double *)calloc(nf, sizeof(double));
    double *vc1 = (double *)malloc(sizeof(double) * (2 * nmax + 2));
    double *vc2 = (double *)malloc(sizeof(double) * (2 * nmax + 2));
    for (int n = 1; n <= nmax; n++) {
        int n21 = n + n + 1;
        for (int l = 1; l <= nmax; l++) {
            double c1 = FNR(n21) * FNR(l + l + 1);
            int ll1 = l * (l + 1);
            vcfunc(-1, n, 1, l, vc2);
            int wmin = iabs_(n - l), wmax = n + l, nlmin = imin(l, n);
            for (int m = -nlmin; m <= nlmin; m++) {
                int ml = ll1 + m;
                double c2 = -c1 * pm1(m);
                vcfunc(-m, n, m, l, vc1);
                for (int w = wmin; w <= wmax; w++) {
                    /* inlw = ci**(n-l+w); (real(inlw)+imag(inlw)) */
                    int e = ((n - l + w) % 4 + 4) % 4;
                    double re = (e == 0) ? 1.0 : (e == 2 ? -1.0 : 0.0);
                    double im = (e == 1) ? 1.0 : (e == 3 ? -1.0 : 0.0);
                    VCC(n, ml, w) = c2 * vc1[w] * vc2[w] * (re + im);
                }
            }
        }
    }
    for (int m = -nmax; m <= nmax; m++) {
        for (int l = imax(1, iabs_(m)); l <= nmax; l++) {
            int lp1 = l + 1, lm1 = l - 1;
            FCI(g_ax.fnm1, m, l) = FNR(lm1) * FNR(lp1) * FNR(l - m) * FNR(l + m) / FNR(lm1 + l) / FNR(l + lp1) / (double)l;
            FCI(g_ax.fn, m, l) = (double)m / (double)l / (double)lp1;
            FCI(g_ax.fnp1, m, l) = FNR(l) * FNR(l + 2) * FNR(lp1 - m) * FNR(lp1 + m) / FNR(l + lp1) / FNR(l + l + 3) / (double)lp1;
        }
    }
    free(vc1); free(vc2);
}

/* atcdim (modules:1956-1962) */
static int atcdim(int ntot, int ltot)
{
    int nmin = imin(ntot, ltot), nmax = imax(ntot, ltot);
    return 2 * (nmin * (1 - nmin * nmin + 3 * nmax * (2 + nmin))) / 3;
}

/* moffset (modules:1966-1978) */
static int moffset(int m, int ntot, int ltot)
{
    if (m == 0) return 0;
    if (m < 0)
        return 2 * (-((1 + m) * (2 + m) * (3 + 2 * m + 3 * ntot)) - 3 * ltot * (2 + ntot + m * (3 + m + 2 * ntot))) / 3;
    return 2 * (-3 * ltot * (-1 + m) * (-1 + m) + 6 * ltot * m * ntot + (-1 + m) * (m * (-4 + 2 * m - 3 * ntot) + 3 * (1 + ntot))) / 3;
}

/* axialtrancoefrecurrence (modules:1566-1676).  ac has atcdim(nmax,lmax)
 * entries.  The caller must have run axialtrancoefinit(max(nmax,lmax)). */
static void axialtrancoefrecurrence(int itype, double r, cplx ri, int nmax, int lmax, cplx *ac)
{
    int nlmin = imin(nmax, lmax);
    int nl = nmax + lmax;
    if (r <= 1.0e-12) {
        int iadd0 = 0;
        for (int ma = 0; ma <= nlmin; ma++) {
            int m1 = imax(1, ma);
            for (int m = -ma; m <= ma; m += 2 * m1) {
                int rows = nmax - m1 + 1, cols = lmax - m1 + 1;
                int blockdim = rows * cols * 2;
                for (int k = 0; k < blockdim; k++) ac[iadd0 + k] = 0;
                if (itype == 1)
                    for (int p = 0; p < 2; p++)
                        for (int l = m1; l <= nlmin; l++) ac[iadd0 + (l - m1) + rows * (l - m1) + rows * cols * p] = 1.0;
                iadd0 += blockdim;
            }
        }
        return;
    }
    cplx z = r * ri;
    cplx *xi = (cplx *)malloc(sizeof(cplx) * (nl + 1));
    if (itype == 1) cricbessel(nl, z, xi);
    else crichankel(nl, z, xi);
    for (int k = 0; k <= nl; k++) xi[k] = xi[k] / z;
    /* both helicities share one refractive index here: xi(:,2)=xi(:,1) */
    int lm1 = lmax - 1;
    int iadd0 = 0;
    cplx *act = (cplx *)malloc(sizeof(cplx) * nmax * lmax * 2);
#define ACT(n, l, p) act[((n) - 1) + nmax * (((l) - 1) + lmax * ((p) - 1))]
    for (int ma = 0; ma <= nlmin; ma++) {
        int m1 = imax(1, ma);
        int lp1 = m1 + 1;
        for (int m = -ma; m <= ma; m += 2 * m1) {
            int blockdim = 2 * (nmax - m1 + 1) * (lmax - m1 + 1);
            int n = m1;
            for (int l = m1; l <= lmax; l++) {
                int wmin = iabs_(n - l), wmax = n + l, ml = l * (l + 1) + m;
                cplx s1 = 0, s2 = 0;
                for (int w = wmin; w <= wmax; w += 2) s1 += VCC(n, ml, w) * xi[w];
                for (int w = wmin + 1; w <= wmax - 1; w += 2) s2 += VCC(n, ml, w) * xi[w];
                s2 = CI * s2;
                ACT(n, l, 1) = s1 + s2;
                ACT(n, l, 2) = s1 - s2;
            }
            {
                int l = lmax, ml = l * (l + 1) + m;
                for (n = m1 + 1; n <= nmax; n++) {
                    int wmin = iabs_(n - l), wmax = n + l;
                    cplx s1 = 0, s2 = 0;
                    for (int w = wmin; w <= wmax; w += 2) s1 += VCC(n, ml, w) * xi[w];
                    for (int w = wmin + 1; w <= wmax - 1; w += 2) s2 += VCC(n, ml, w) * xi[w];
                    s2 = CI * s2;
                    ACT(n, l, 1) = s1 + s2;
                    ACT(n, l, 2) = s1 - s2;
                }
            }
            if (m1 < nlmin) {
                for (n = m1; n <= nmax - 1; n++) {
                    int np1 = n + 1, nm1 = n - 1;
                    for (int p = 1; p <= 2; p++) {
                        double sp = -pm1(p);
                        /* row np1 for columns m1..lmax-1 */
                        for (int l = m1; l <= lm1; l++) {
                            cplx v = -ACT(n, l + 1, p) * FCI(g_ax.fnp1, m, l)
                                     + sp * (FCI(g_ax.fn, m, l) - FCI(g_ax.fn, m, n)) * CI * ACT(n, l, p);
                            if (l >= lp1) v = v + ACT(n, l - 1, p) * FCI(g_ax.fnm1, m, l);
                            if (n > m1) v = v + ACT(nm1, l, p) * FCI(g_ax.fnm1, m, n);
                            ACT(np1, l, p) = v / FCI(g_ax.fnp1, m, n);
                        }
                    }
                }
            }
            /* reshape(act(m1:nmax,m1:lmax,1:2)) */
            int rows = nmax - m1 + 1, cols = lmax - m1 + 1;
            for (int p = 1; p <= 2; p++)
                for (int l = m1; l <= lmax; l++)
                    for (n = m1; n <= nmax; n++)
                        ac[iadd0 + (n - m1) + rows * ((l - m1) + cols * (p - 1))] = ACT(n, l, p);
            iadd0 += blockdim;
        }
    }
#undef ACT
    free(act);
    free(xi);
}

/* ------------------------------------------------------------------------ */
/* Wigner-d: rotcoef (modules:1098-1175), crotcoef (modules:1187-1246)       */
/* dc indexed dc[(m+kmax) + (2kmax+1)*nk], nk = n(n+1)+k                     */
/* ------------------------------------------------------------------------ */
static void rotcoef(double cbe, int kmax, int nmax, double *dc)
{
    int ld = 2 * kmax + 1;
#define DC(m, nk) dc[((m) + kmax) + ld * (nk)]
    memset(dc, 0, sizeof(double) * ld * (nmax * (nmax + 2) + 1));
    double sbe;
    if (fabs(cbe) >= 1.0) sbe = 0.0;
    else sbe = sqrt(fabs((1.0 + cbe) * (1.0 - cbe)));
    double cbe2 = 0.5 * (1.0 + cbe), sbe2 = 0.5 * (1.0 - cbe);
    double *dk0 = (double *)calloc(2 * nmax + 3, sizeof(double)) + (nmax + 1);
    double *dk01 = (double *)calloc(2 * nmax + 3, sizeof(double)) + (nmax + 1);
    int sgn = 1;
    dk0[0] = 1.0;
    double sben = 1.0;
    DC(0, 0) = 1.0;
    dk01[0] = 0.0;
    for (int n = 1; n <= nmax; n++) {
        int knmax = imin(n, kmax);
        int nn1 = n * (n + 1);
        sgn = -sgn;
        sben = sben * sbe / 2.0;
        if (sben < 1.0e-30) sben = 0.0;
        dk0[n] = sgn * sben * BCOF(n, n);
        dk0[-n] = sgn * dk0[n];
        dk01[n] = 0.0;
        dk01[-n] = 0.0;
        DC(0, nn1 + n) = dk0[n];
        DC(0, nn1 - n) = dk0[-n];
        for (int k = -n + 1; k <= n - 1; k++) {
            int kn = nn1 + k;
            double dkt = dk01[k];
            dk01[k] = dk0[k];
            dk0[k] = (cbe * (double)(n + n - 1) * dk01[k] - FNR(n - k - 1) * FNR(n + k - 1) * dkt) / (FNR(n + k) * FNR(n - k));
            DC(0, kn) = dk0[k];
        }
        int im = 1;
        for (int m = 1; m <= knmax; m++) {
            im = -im;
            double fmn = 1.0 / FNR(n - m + 1) / FNR(n + m);
            int m1 = m - 1;
            double dkm0 = 0.0;
            for (int k = -n; k <= n; k++) {
                int kn = nn1 + k;
                double dkm1 = dkm0;
                dkm0 = DC(m1, kn);
                double dkn1 = (k == n) ? 0.0 : DC(m1, kn + 1);
                DC(m, kn) = (FNR(n + k) * FNR(n - k + 1) * cbe2 * dkm1 - FNR(n - k) * FNR(n + k + 1) * sbe2 * dkn1
                             - (double)k * sbe * DC(m1, kn)) * fmn;
                DC(-m, nn1 - k) = DC(m, kn) * pm1(k) * im;
            }
        }
    }
#undef DC
    free(dk0 - (nmax + 1));
    free(dk01 - (nmax + 1));
}

static void crotcoef(cplx cbe, int kmax, int nmax, cplx *dc)
{
    int ld = 2 * kmax + 1;
#define DC(m, nk) dc[((m) + kmax) + ld * (nk)]
    for (int i = 0; i < ld * (nmax * (nmax + 2) + 1); i++) dc[i] = 0;
    cplx sbe = csqrt((1.0 + cbe) * (1.0 - cbe));
    cplx cbe2 = 0.5 * (1.0 + cbe), sbe2 = 0.5 * (1.0 - cbe);
    cplx *dk0 = (cplx *)calloc(2 * nmax + 3, sizeof(cplx)) + (nmax + 1);
    cplx *dk01 = (cplx *)calloc(2 * nmax + 3, sizeof(cplx)) + (nmax + 1);
    int in = 1;
    dk0[0] = 1.0;
    cplx sben = 1.0;
    DC(0, 0) = 1.0;
    dk01[0] = 0.0;
    for (int n = 1; n <= nmax; n++) {
        int knmax = imin(n, kmax);
        int nn1 = n * (n + 1);
        in = -in;
        sben = sben * sbe / 2.0;
        dk0[n] = (double)in * sben * BCOF(n, n);
        dk0[-n] = (double)in * dk0[n];
        dk01[n] = 0.0;
        dk01[-n] = 0.0;
        DC(0, nn1 + n) = dk0[n];
        DC(0, nn1 - n) = dk0[-n];
        for (int k = -n + 1; k <= n - 1; k++) {
            int kn = nn1 + k;
            cplx dkt = dk01[k];
            dk01[k] = dk0[k];
            dk0[k] = (cbe * (double)(n + n - 1) * dk01[k] - FNR(n - k - 1) * FNR(n + k - 1) * dkt) / (FNR(n + k) * FNR(n - k));
            DC(0, kn) = dk0[k];
        }
        int im = 1;
        for (int m = 1; m <= knmax; m++) {
            im = -im;
            double fmn = 1.0 / FNR(n - m + 1) / FNR(n + m);
            int m1 = m - 1;
            cplx dkm0 = 0.0;
            for (int k = -n; k <= n; k++) {
                int kn = nn1 + k;
                cplx dkm1 = dkm0;
                dkm0 = DC(m1, kn);
                cplx dkn1 = (k == n) ? 0.0 : DC(m1, kn + 1);
                DC(m, kn) = (FNR(n + k) * FNR(n - k + 1) * cbe2 * dkm1 - FNR(n - k) * FNR(n + k + 1) * sbe2 * dkn1
                             - (double)k * sbe * DC(m1, kn)) * fmn;
                DC(-m, nn1 - k) = DC(m, kn) * pm1(k) * (double)im;
            }
        }
    }
#undef DC
    free(dk0 - (nmax + 1));
    free(dk01 - (nmax + 1));
}

/* normalizedlegendre (modules:1061-1083): dc(-mmax:mmax, 0:nmax) */
static void normalizedlegendre(double cbe, int mmax, int nmax, double *dc)
{
    int ld = 2 * mmax + 1;
#define DL(m, n) dc[((m) + mmax) + ld * (n)]
    double sbe = sqrt((1.0 + cbe) * (1.0 - cbe));
    memset(dc, 0, sizeof(double) * ld * (nmax + 1));
    for (int m = 0; m <= mmax; m++) {
        DL(m, m) = pm1(m) * pow(0.5 * sbe, m) * BCOF(m, m);
        if (m == nmax) break;
        DL(m, m + 1) = FNR(m + m + 1) * cbe * DL(m, m);
        for (int n = m + 1; n <= nmax - 1; n++)
            DL(m, n + 1) = (-FNR(n - m) * FNR(n + m) * DL(m, n - 1) + (double)(n + n + 1) * cbe * DL(m, n)) / (FNR(n + 1 - m) * FNR(n + 1 + m));
    }
    for (int m = 1; m <= mmax; m++) {
        double im = pm1(m);
        for (int n = m; n <= nmax; n++) DL(-m, n) = im * DL(m, n);
    }
#undef DL
}

/* cartosphere (modules:1986-2004), ephicoef (modules:2075-2085) */
static void cartosphere(const double *xp, double *r, double *ct, cplx *ep)
{
    double rr = xp[0] * xp[0] + xp[1] * xp[1] + xp[2] * xp[2];
    if (rr == 0.0) { *r = 0.0; *ct = 1.0; *ep = 1.0; return; }
    rr = sqrt(rr);
    *r = rr;
    *ct = xp[2] / rr;
    if (xp[0] == 0.0 && xp[1] == 0.0) *ep = 1.0;
    else *ep = (xp[0] + CI * xp[1]) / sqrt(xp[0] * xp[0] + xp[1] * xp[1]);
}
static void ephicoef(cplx ep, int nodr, cplx *epm /* index m+nodr */)
{
    epm[nodr] = 1.0;
    for (int m = 1; m <= nodr; m++) {
        epm[nodr + m] = ep * epm[nodr + m - 1];
        epm[nodr - m] = conj(epm[nodr + m]);
    }
}

/* ------------------------------------------------------------------------ */
/* gentranmatrix (modules:1724-1888): dense LR-mode translation matrix,      */
/* index model 2.  ac(nblkt, nblks, 2) column-major.  Used by the dense LU   */
/* check, which is an independent route to the pair operator.                */
/* ------------------------------------------------------------------------ */
static int amnaddress2(int m, int n, int l) /* 1-based, model 2 */
{
    return (m >= 0) ? (n - 1) * (l + 2) + m + 1 : -(m + 1) * (l + 2) + n + 2;
}

static void gentranmatrix(int nodr_s, int nodr_t, const double *xp, cplx ri, int itype, cplx *ac)
{
    int nblks = nodr_s * (nodr_s + 2), nblkt = nodr_t * (nodr_t + 2);
    int nodrmax = imax(nodr_s, nodr_t);
    int wmaxt = nodr_s + nodr_t;
    size_t ntot = (size_t)nblkt * nblks * 2;
    double rr = xp[0] * xp[0] + xp[1] * xp[1] + xp[2] * xp[2];
    if (rr == 0.0) {
        for (size_t k = 0; k < ntot; k++) ac[k] = 0;
        if (itype == 1)
            for (int n = 1; n <= imin(nblks, nblkt); n++)
                for (int p = 0; p < 2; p++) ac[(n - 1) + (size_t)nblkt * ((n - 1) + (size_t)nblks * p)] = 1.0;
        return;
    }
    /* tran_coef constants (modules:1724-1760) for the orders needed */
    int nd = nodrmax * (nodrmax + 2);
    double *tc = (double *)calloc((size_t)nd * nd * (2 * nodrmax + 1), sizeof(double));
#define TC(mn, kl, w) tc[((mn) - 1) + (size_t)nd * (((kl) - 1) + (size_t)nd * (w))]
    double *vc1 = (double *)malloc(sizeof(double) * (2 * nodrmax + 2));
    double *vc2 = (double *)malloc(sizeof(double) * (2 * nodrmax + 2));
    for (int l = 1; l <= nodrmax; l++)
        for (int n = 1; n <= nodrmax; n++) {
            int wmax = n + l;
            vcfunc(-1, n, 1, l, vc2);
            int e0 = ((n - l) % 4 + 4) % 4;
            cplx ie = (e0 == 0) ? 1.0 : (e0 == 1 ? CI : (e0 == 2 ? -1.0 : -CI));
            cplx c = -ie * FNR(n + n + 1) * FNR(l + l + 1);
            for (int k = -l; k <= l; k++) {
                int kl = l * (l + 1) + k;
                for (int m = -n; m <= n; m++) {
                    int mn = n * (n + 1) + m;
                    double m1m = pm1(m);
                    int v = k - m;
                    vcfunc(-m, n, k, l, vc1);
                    int wmin = imax(iabs_(v), iabs_(n - l));
                    for (int w = wmax; w >= wmin; w--) {
                        int e = (w % 4 + 4) % 4;
                        cplx iw = (e == 0) ? 1.0 : (e == 1 ? CI : (e == 2 ? -1.0 : -CI));
                        cplx a = iw * c * m1m * vc1[w] * vc2[w];
                        if ((wmax - w) % 2 == 0) TC(mn, kl, w) = creal(a);
                        else TC(mn, kl, w) = cimag(a);
                    }
                }
            }
        }
    double r = sqrt(rr);
    double ct = xp[2] / r;
    cplx ephi = (xp[0] == 0.0 && xp[1] == 0.0) ? 1.0 : (xp[0] + CI * xp[1]) / sqrt(xp[0] * xp[0] + xp[1] * xp[1]);
    cplx *ephim = (cplx *)malloc(sizeof(cplx) * (2 * wmaxt + 1));
    ephim[wmaxt] = 1.0;
    for (int m = 1; m <= wmaxt; m++) { ephim[wmaxt + m] = ephi * ephim[wmaxt + m - 1]; ephim[wmaxt - m] = conj(ephim[wmaxt + m]); }
    double *ymn = (double *)malloc(sizeof(double) * (2 * wmaxt + 1) * (wmaxt + 1));
    normalizedlegendre(ct, wmaxt, wmaxt, ymn);
#define YMN(v, w) ymn[((v) + wmaxt) + (2 * wmaxt + 1) * (w)]
    cplx *hn = (cplx *)malloc(sizeof(cplx) * (wmaxt + 1));
    cplx rri = r * ri;
    if (itype == 3) {
        hn[0] = -CI * cexp(CI * rri) / rri;
        hn[1] = -cexp(CI * rri) * (CI + rri) / rri / rri;
        for (int n = 2; n <= wmaxt; n++) hn[n] = (double)(n + n - 1) / rri * hn[n - 1] - hn[n - 2];
    } else {
        cricbessel(wmaxt, rri, hn);
        for (int n = 0; n <= wmaxt; n++) hn[n] = hn[n] / rri;
    }
    for (int n = 1; n <= nodr_s; n++)
        for (int m = -n; m <= n; m++) {
            int mna = amnaddress2(m, n, nodr_s);
            int mn = n * (n + 1) + m;
            for (int l = 1; l <= nodr_t; l++) {
                int wmax = n + l;
                for (int k = -l; k <= l; k++) {
                    int kla = amnaddress2(k, l, nodr_t);
                    int kl = l * (l + 1) + k;
                    int v = m - k;
                    int wmin = imax(iabs_(v), iabs_(n - l));
                    cplx a1 = 0, a2 = 0, b1 = 0, b2 = 0;
                    for (int w = wmax; w >= wmin; w--) {
                        if ((wmax - w) % 2 == 0) {
                            a1 += hn[w] * YMN(v, w) * TC(kl, mn, w);
                            a2 += hn[w] * YMN(v, w) * TC(kl, mn, w);
                        } else {
                            b1 += hn[w] * YMN(v, w) * TC(kl, mn, w);
                            b2 += hn[w] * YMN(v, w) * TC(kl, mn, w);
                        }
                    }
                    ac[(kla - 1) + (size_t)nblkt * ((mna - 1) + (size_t)nblks * 0)] = ephim[wmaxt + v] * (a1 + CI * b1);
                    ac[(kla - 1) + (size_t)nblkt * ((mna - 1) + (size_t)nblks * 1)] = ephim[wmaxt + v] * (a2 - CI * b2);
                }
            }
        }
#undef TC
#undef YMN
    free(tc); free(vc1); free(vc2); free(ephim); free(ymn); free(hn);
}

/* ------------------------------------------------------------------------ */
/* coefficient translation (modules:6610-6787, shiftcoefficient 6789-6820)   */
/* ------------------------------------------------------------------------ */
#define AIDX(m, n, p, L) ((m) + ((L) + 2) * ((n) - 1) + ((L) + 2) * (L) * (p))   /* 0-based, m in 0..L+1 */

static void shiftcoefficient(int nodr, int msign, int mflip, const cplx *ain, cplx *aout)
{
    int nb = 2 * nodr * (nodr + 2);
    if (msign == 1 && mflip == 1) { if (aout != ain) memcpy(aout, ain, sizeof(cplx) * nb); return; }
    for (int p = 0; p < 2; p++)
        for (int n = 1; n <= nodr; n++) aout[AIDX(0, n, p, nodr)] = ain[AIDX(0, n, p, nodr)];
    double im = 1.0;
    for (int m = 1; m <= nodr; m++) {
        im = im * msign;
        for (int n = m; n <= nodr; n++)
            for (int p = 0; p < 2; p++) {
                if (mflip == -1) {
                    cplx at = ain[AIDX(n + 1, m, p, nodr)];
                    aout[AIDX(n + 1, m, p, nodr)] = im * ain[AIDX(m, n, p, nodr)];
                    aout[AIDX(m, n, p, nodr)] = im * at;
                } else {
                    aout[AIDX(m, n, p, nodr)] = im * ain[AIDX(m, n, p, nodr)];
                    aout[AIDX(n + 1, m, p, nodr)] = im * ain[AIDX(n + 1, m, p, nodr)];
                }
            }
    }
}

/* One pair operator in the reference's stored form (translation_data,
 * modules:5773-5780): rot_mat(-nmin:nmin, 0:nmax(nmax+2)), z_mat(atcdim),
 * phi_mat(-nmax:nmax).  nodrt = target order, nodrs = source order of the
 * first (shift_op=F) application; rvec = target - source position. */
typedef struct {
    int nodrt, nodrs, nmin, nmax, vtype;
    int zero;
    double *rot;
    cplx *z, *phi;
} pairop_t;

static void pairop_compute(pairop_t *op, int nodrt, int nodrs, const double *rvec, int vtype, cplx rimed)
{
    op->nodrt = nodrt; op->nodrs = nodrs; op->vtype = vtype;
    op->nmin = imin(nodrt, nodrs); op->nmax = imax(nodrt, nodrs);
    double r2 = rvec[0] * rvec[0] + rvec[1] * rvec[1] + rvec[2] * rvec[2];
    op->zero = (r2 < 1.0e-12);
    op->rot = NULL; op->z = NULL; op->phi = NULL;
    if (op->zero) return;
    int nmin = op->nmin, nmax = op->nmax;
    op->rot = (double *)malloc(sizeof(double) * (2 * nmin + 1) * (nmax * (nmax + 2) + 1));
    op->phi = (cplx *)malloc(sizeof(cplx) * (2 * nmax + 1));
    op->z = (cplx *)malloc(sizeof(cplx) * atcdim(nodrt, nodrs));
    double r, ct; cplx ephi;
    cartosphere(rvec, &r, &ct, &ephi);
    rotcoef(ct, nmin, nmax, op->rot);
    axialtrancoefrecurrence(vtype, r, rimed, nodrt, nodrs, op->z);
    ephicoef(ephi, nmax, op->phi);
}
static void pairop_free(pairop_t *op) { free(op->rot); free(op->z); free(op->phi); op->rot = NULL; op->z = NULL; op->phi = NULL; }

/* coefficient_translation, rotation path: gcoef += T(op) acoef. */
static void coefficient_translation(int nodra, int nodrg, const cplx *acoef, cplx *gcoef, const pairop_t *op, int sop, int top)
{
    if (op->zero) {
        if (op->vtype == 1) {
            /* mtransfer: copy the overlapping orders */
            int nmn = imin(nodra, nodrg);
            for (int p = 0; p < 2; p++)
                for (int n = 1; n <= nmn; n++) {
                    for (int m = 0; m <= n; m++) gcoef[AIDX(m, n, p, nodrg)] += acoef[AIDX(m, n, p, nodra)];
                    for (int m = 1; m <= n; m++) gcoef[AIDX(n + 1, m, p, nodrg)] += acoef[AIDX(n + 1, m, p, nodra)];
                }
        }
        return;
    }
    int nmin = op->nmin, nmax = op->nmax;
    int ldr = 2 * nmin + 1;
#define ROT(k, nk) op->rot[((k) + nmin) + ldr * (nk)]
#define PHI(m) op->phi[(m) + nmax]
    int sv = (sop != top) ? -1 : 1;
    int im = sop ? -1 : 1;
    int nba = 2 * nodra * (nodra + 2), nbg = 2 * nodrg * (nodrg + 2);
    cplx *a_t = (cplx *)malloc(sizeof(cplx) * nba);
    shiftcoefficient(nodra, sv, sv, acoef, a_t);
    int lda = 2 * nodra + 1, ldg = 2 * nodrg + 1;
    cplx *a_tt = (cplx *)calloc((size_t)lda * nodra * 2, sizeof(cplx));
    cplx *g_tt = (cplx *)calloc((size_t)ldg * nodrg * 2, sizeof(cplx));
    cplx *tmp = (cplx *)malloc(sizeof(cplx) * (2 * nmax + 1));
#define ATT(m, n, p) a_tt[((m) + nodra) + lda * (((n) - 1) + nodra * (p))]
#define GTT(m, n, p) g_tt[((m) + nodrg) + ldg * (((n) - 1) + nodrg * (p))]
    for (int p = 0; p < 2; p++) {
        for (int n = 1; n <= nodra; n++) ATT(0, n, p) = a_t[AIDX(0, n, p, nodra)];
        for (int m = 1; m <= nodra; m++)
            for (int n = m; n <= nodra; n++) {
                ATT(m, n, p) = a_t[AIDX(m, n, p, nodra)] * PHI(im * m);
                ATT(-m, n, p) = a_t[AIDX(n + 1, m, p, nodra)] * PHI(-im * m);
            }
        /* forward rotation */
        for (int n = 1; n <= nodra; n++) {
            int nn1 = n * n;   /* n(n+1)-n */
            int n1 = imin(n, nodrg);
            for (int k = -n1; k <= n1; k++) {
                cplx s = 0;
                for (int m = -n; m <= n; m++) s += ROT(k, nn1 + (m + n)) * ATT(m, n, p);
                tmp[k + n1] = s;
            }
            for (int k = -n1; k <= n1; k++) ATT(k, n, p) = tmp[k + n1];
        }
    }
    /* axial translation per degree m */
    for (int m = -nmin; m <= nmin; m++) {
        int m1 = imax(1, iabs_(m));
        if (sop) {
            int offset = moffset(m, nodra, nodrg);
            int rows = nodra - m1 + 1, cols = nodrg - m1 + 1;
            for (int p = 0; p < 2; p++)
                for (int l = m1; l <= nodrg; l++) {
                    cplx s = 0;
                    for (int n = m1; n <= nodra; n++)
                        s += ATT(m, n, p) * op->z[offset + (n - m1) + rows * ((l - m1) + cols * p)];
                    GTT(m, l, p) = s;
                }
        } else {
            int offset = moffset(m, nodrg, nodra);
            int rows = nodrg - m1 + 1, cols = nodra - m1 + 1;
            for (int p = 0; p < 2; p++)
                for (int n = m1; n <= nodrg; n++) {
                    cplx s = 0;
                    for (int l = m1; l <= nodra; l++)
                        s += op->z[offset + (n - m1) + rows * ((l - m1) + cols * p)] * ATT(m, l, p);
                    GTT(m, n, p) = s;
                }
        }
    }
    /* back rotation */
    for (int p = 0; p < 2; p++)
        for (int n = 1; n <= nodrg; n++) {
            int nn1 = n * n;
            int n1 = imin(n, nodra);
            for (int k = -n; k <= n; k++) {
                cplx s = 0;
                for (int m = -n1; m <= n1; m++) s += GTT(m, n, p) * ROT(m, nn1 + (k + n));
                tmp[k + n] = s;
            }
            for (int k = -n; k <= n; k++) GTT(k, n, p) = tmp[k + n];
        }
    cplx *g_t = (cplx *)malloc(sizeof(cplx) * nbg);
    for (int p = 0; p < 2; p++) {
        for (int n = 1; n <= nodrg; n++) g_t[AIDX(0, n, p, nodrg)] = GTT(0, n, p);
        for (int m = 1; m <= nodrg; m++)
            for (int n = m; n <= nodrg; n++) {
                g_t[AIDX(m, n, p, nodrg)] = GTT(m, n, p) * PHI(-im * m);
                g_t[AIDX(n + 1, m, p, nodrg)] = GTT(-m, n, p) * PHI(im * m);
            }
    }
    shiftcoefficient(nodrg, sv, sv, g_t, g_t);
    for (int k = 0; k < nbg; k++) gcoef[k] += g_t[k];
#undef ATT
#undef GTT
#undef ROT
#undef PHI
    free(a_t); free(a_tt); free(g_tt); free(tmp); free(g_t);
}

/* ------------------------------------------------------------------------ */
/* context = the reference's spheredata/mie module globals                   */
/* ------------------------------------------------------------------------ */
struct orc_ctx {
    int n;
    double *pos, *rad;
    cplx *ri;
    cplx rimed;
    int *order, *offset, *mie_offset;
    int neqns, max_order;
    cplx *an, *an_inv;
    double *qext_mie, *qabs_mie;
    int store;
    int nthreads;
    int npairs;
    int *pi_, *pj_;
    pairop_t *ops;     /* stored operators (store_translation_matrix) */
    int ops_ready;
    /* FFT translation (fft_translation-5.f90): set by orc_fft_setup */
    int fft, No, cd[3], nnb, nb_vec[27][3];
    double dcell, cb[3];
    int *snode;            /* 3N, 1-based cell of each sphere */
    cplx *Jsn, *Jns;       /* per sphere: dense J(node - pos) (nbN x nb_i x 2) and J(pos - node) (nb_i x nbN x 2) */
    size_t *joff;
    cplx *Hc;              /* dense H at every node offset (2cd-1)^3 x nbN x nbN x 2, zero inside the hole */
    int last_iter[2];      /* cbicg iterations of each polarisation in the last orc_fixedorsoln */
    /* host spheres (spheredata, modules:5088-5278): spheres inside others */
    int *host;             /* findhostspheres: the host of each sphere, -1 outside every sphere */
    int *nfe;              /* number_field_expansions: 2 for a sphere holding others, else 1 */
    int nhosted;           /* number_host_spheres: spheres that have a host */
    cplx *rext;            /* exteriorrefindex: the index around each sphere */
    cplx *dn, *un, *vn;    /* the host spheres' D, U, V Mie coefficients (mie_offset) */
    int nhp;               /* external_to_internal pairs: (host, sphere it holds) */
    int *hpi, *hpj;
    pairop_t *hops;        /* their regular translation operators */
};

/* findhostspheres (modules:5230-5276): the host of sphere i is the smallest
 * larger sphere whose surface encloses i's centre (the first in order among
 * equal radii); sphere_order then raised so that every host has at least the
 * order of the spheres inside it (miecoefcalc, modules:5331-5342). */
static void find_hosts(orc_ctx *c)
{
    int n = c->n;
    c->nhosted = 0;
    for (int i = 0; i < n; i++) {
        c->host[i] = -1;
        c->nfe[i] = 1;
    }
    for (int i = 0; i < n; i++) {
        double xspmin = 1.0e6;
        for (int j = 0; j < n; j++) {
            if (!(c->rad[j] > c->rad[i])) continue;
            double d0 = c->pos[3 * j] - c->pos[3 * i], d1 = c->pos[3 * j + 1] - c->pos[3 * i + 1], d2 = c->pos[3 * j + 2] - c->pos[3 * i + 2];
            double rij = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            if (rij <= c->rad[j] && c->rad[j] < xspmin) {
                c->host[i] = j;
                xspmin = c->rad[j];
            }
        }
    }
    for (int i = 0; i < n; i++)
        if (c->host[i] >= 0) {
            c->nfe[c->host[i]] = 2;
            c->nhosted++;
        }
    for (int i = 0; i < n; i++) c->rext[i] = c->host[i] >= 0 ? c->ri[c->host[i]] : c->rimed;
}

orc_ctx *orc_create(int nsphere, const double *pos, const double *radius, const double *ri,
                    double mie_eps, int store_matrix, int nthreads)
{
    tables_init();
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
    c->n = nsphere;
    c->pos = (double *)malloc(sizeof(double) * 3 * nsphere);
    c->rad = (double *)malloc(sizeof(double) * nsphere);
    c->ri = (cplx *)malloc(sizeof(cplx) * nsphere);
    memcpy(c->pos, pos, sizeof(double) * 3 * nsphere);
    memcpy(c->rad, radius, sizeof(double) * nsphere);
    for (int i = 0; i < nsphere; i++) c->ri[i] = ri[2 * i] + CI * ri[2 * i + 1];
    c->rimed = 1.0;
    c->host = (int *)malloc(sizeof(int) * (nsphere + 1));
    c->nfe = (int *)malloc(sizeof(int) * (nsphere + 1));
    c->rext = (cplx *)malloc(sizeof(cplx) * (nsphere + 1));
    find_hosts(c);
    c->order = (int *)malloc(sizeof(int) * nsphere);
    c->offset = (int *)malloc(sizeof(int) * (nsphere + 1));
    c->mie_offset = (int *)malloc(sizeof(int) * (nsphere + 1));
    c->qext_mie = (double *)malloc(sizeof(double) * nsphere);
    c->qabs_mie = (double *)malloc(sizeof(double) * nsphere);
    /* miecoefcalc (modules:5301-5407): each sphere in the medium around it */
    int nterms = 0, nblk = 0, maxo = 0;
    for (int i = 0; i < nsphere; i++) {
        int nodrn = 0;
        double qe, qs, qa;
        mieoa(c->rad[i], c->ri[i], c->rext[i], &nodrn, mie_eps, &qe, &qs, &qa, NULL, NULL);
        c->order[i] = nodrn;
    }
    for (int i = 0; i < nsphere; i++)
        for (int j = c->host[i]; j >= 0; j = c->host[j]) c->order[j] = imax(c->order[j], c->order[i]);
    for (int i = 0; i < nsphere; i++) {
        c->mie_offset[i] = nterms;
        nterms += 4 * c->order[i];
        c->offset[i] = nblk;
        nblk += 2 * c->order[i] * (c->order[i] + 2) * c->nfe[i];
        maxo = imax(maxo, c->order[i]);
    }
    c->mie_offset[nsphere] = nterms;
    c->offset[nsphere] = nblk;
    c->neqns = nblk;
    c->max_order = maxo;
    c->an = (cplx *)malloc(sizeof(cplx) * (nterms + 1));
    c->an_inv = (cplx *)malloc(sizeof(cplx) * (nterms + 1));
    c->dn = (cplx *)calloc(nterms + 1, sizeof(cplx));
    c->un = (cplx *)calloc(nterms + 1, sizeof(cplx));
    c->vn = (cplx *)calloc(nterms + 1, sizeof(cplx));
    for (int i = 0; i < nsphere; i++) {
        int nodrn = c->order[i];
        mieoa(c->rad[i], c->ri[i], c->rext[i], &nodrn, 0.0, &c->qext_mie[i], NULL, &c->qabs_mie[i],
              c->an + c->mie_offset[i], c->an_inv + c->mie_offset[i]);
        if (c->nfe[i] == 2)
            mieoa_host(c->rad[i], c->ri[i], c->rext[i], nodrn, c->dn + c->mie_offset[i], c->un + c->mie_offset[i],
                       c->vn + c->mie_offset[i]);
    }
    axialtrancoefinit(maxo);
    c->store = store_matrix;
    c->nthreads = nthreads > 0 ? nthreads : 1;
    /* external_to_external_expansion's pairs: i < j in the same host
     * (modules:6466-6469); external_to_internal_expansion's: a host and a
     * sphere it holds (modules:6569-6571) */
    c->npairs = 0;
    c->nhp = 0;
    for (int i = 0; i < nsphere - 1; i++)
        for (int j = i + 1; j < nsphere; j++) {
            if (c->host[i] == c->host[j]) c->npairs++;
            if (c->host[j] == i || c->host[i] == j) c->nhp++;
        }
    c->pi_ = (int *)malloc(sizeof(int) * (c->npairs + 1));
    c->pj_ = (int *)malloc(sizeof(int) * (c->npairs + 1));
    c->hpi = (int *)malloc(sizeof(int) * (c->nhp + 1));
    c->hpj = (int *)malloc(sizeof(int) * (c->nhp + 1));
    int t = 0, h = 0;
    for (int i = 0; i < nsphere - 1; i++)
        for (int j = i + 1; j < nsphere; j++) {
            if (c->host[i] == c->host[j]) { c->pi_[t] = i; c->pj_[t] = j; t++; }
            if (c->host[j] == i) { c->hpi[h] = i; c->hpj[h] = j; h++; }
            else if (c->host[i] == j) { c->hpi[h] = j; c->hpj[h] = i; h++; }
        }
    return c;
}

void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    if (c->ops) { for (int k = 0; k < c->npairs; k++) pairop_free(&c->ops[k]); free(c->ops); }
    free(c->pos); free(c->rad); free(c->ri); free(c->order); free(c->offset); free(c->mie_offset);
    free(c->an); free(c->an_inv); free(c->qext_mie); free(c->qabs_mie); free(c->pi_); free(c->pj_);
    free(c->snode); free(c->Jsn); free(c->Jns); free(c->joff); free(c->Hc);
    if (c->hops) { for (int k = 0; k < c->nhp; k++) pairop_free(&c->hops[k]); free(c->hops); }
    free(c->host); free(c->nfe); free(c->rext); free(c->dn); free(c->un); free(c->vn); free(c->hpi); free(c->hpj);
    free(c);
}

int orc_neqns(const orc_ctx *c) { return c->neqns; }
/* host[i]: the sphere holding sphere i (-1: none); returns number_host_spheres */
int orc_hosts(const orc_ctx *c, int *host)
{
    if (host) memcpy(host, c->host, sizeof(int) * c->n);
    return c->nhosted;
}
void orc_host_mie_coefs(const orc_ctx *c, cplx *dn, cplx *un, cplx *vn)
{
    int nt = c->mie_offset[c->n];
    if (dn) memcpy(dn, c->dn, sizeof(cplx) * nt);
    if (un) memcpy(un, c->un, sizeof(cplx) * nt);
    if (vn) memcpy(vn, c->vn, sizeof(cplx) * nt);
}
void orc_orders(const orc_ctx *c, int *order, int *offset, int *mie_offset)
{
    if (order) memcpy(order, c->order, sizeof(int) * c->n);
    if (offset) memcpy(offset, c->offset, sizeof(int) * (c->n + 1));
    if (mie_offset) memcpy(mie_offset, c->mie_offset, sizeof(int) * (c->n + 1));
}
void orc_mie_coefs(const orc_ctx *c, cplx *an, cplx *an_inv, double *qext, double *qabs)
{
    int nt = c->mie_offset[c->n];
    if (an) memcpy(an, c->an, sizeof(cplx) * nt);
    if (an_inv) memcpy(an_inv, c->an_inv, sizeof(cplx) * nt);
    if (qext) memcpy(qext, c->qext_mie, sizeof(double) * c->n);
    if (qabs) memcpy(qabs, c->qabs_mie, sizeof(double) * c->n);
}

/* onemiecoeffmult / multmiecoeffmult (modules:5585-5688).
 * idir==1: y = A x ; otherwise y = A^T x.  In-place allowed. */
static void mie_acc(const cplx *an1, int nodr, int idir, const cplx *t, cplx *y)
{
    for (int n = 1; n <= nodr; n++)
        for (int p = 1; p <= 2; p++)
            for (int q = 1; q <= 2; q++) {
                cplx a = (idir == 1) ? an1[(p - 1) + 2 * (q - 1) + 4 * (n - 1)] : an1[(q - 1) + 2 * (p - 1) + 4 * (n - 1)];
                for (int m = 1; m <= n; m++) y[AIDX(n + 1, m, p - 1, nodr)] += a * t[AIDX(n + 1, m, q - 1, nodr)];
                for (int m = 0; m <= n; m++) y[AIDX(m, n, p - 1, nodr)] += a * t[AIDX(m, n, q - 1, nodr)];
            }
}
static void mie_mult_sphere(const cplx *an1, int nodr, int idir, const cplx *x, cplx *y)
{
    int nb = 2 * nodr * (nodr + 2);
    cplx *t = (cplx *)malloc(sizeof(cplx) * nb);
    memcpy(t, x, sizeof(cplx) * nb);
    for (int k = 0; k < nb; k++) y[k] = 0;
    mie_acc(an1, nodr, idir, t, y);
    free(t);
}
/* The host branch of multmiecoeffmult (modules:5690-5747): the sphere's
 * block (g) and the block of the field inside it (b) give
 * idir==1: a = A g + U b, f = D g + V b; otherwise the transpose,
 * a = A^T g + D^T b, f = U^T g + V^T b. */
static void mie_mult_host(const orc_ctx *c, int i, int idir, const cplx *ain, cplx *aout)
{
    int nodr = c->order[i], nb = 2 * nodr * (nodr + 2), mo = c->mie_offset[i];
    const cplx *g = ain + c->offset[i], *b = g + nb;
    cplx *a = aout + c->offset[i], *f = a + nb;
    cplx *tg = (cplx *)malloc(sizeof(cplx) * 2 * nb), *tb = tg + nb;
    memcpy(tg, g, sizeof(cplx) * nb);
    memcpy(tb, b, sizeof(cplx) * nb);
    for (int k = 0; k < nb; k++) { a[k] = 0; f[k] = 0; }
    mie_acc(c->an + mo, nodr, idir, tg, a);
    mie_acc((idir == 1 ? c->un : c->dn) + mo, nodr, idir, tb, a);
    mie_acc((idir == 1 ? c->dn : c->un) + mo, nodr, idir, tg, f);
    mie_acc(c->vn + mo, nodr, idir, tb, f);
    free(tg);
}
static void multmiecoeffmult(const orc_ctx *c, int idir, const cplx *ain, cplx *aout, const cplx *coef)
{
    for (int i = 0; i < c->n; i++) {
        if (c->nfe[i] == 2 && coef == c->an) mie_mult_host(c, i, idir, ain, aout);
        else mie_mult_sphere(coef + c->mie_offset[i], c->order[i], idir, ain + c->offset[i], aout + c->offset[i]);
    }
}

/* external_to_external_expansion (modules:6390-6525).  The pair loop is
 * split over threads with a private output each and a final sum, the
 * single-node analogue of the reference's round-robin MPI task split plus
 * allreduce (scatprops:152-156). */
/* ------------------------------------------------------------------------ */
/* FFT translation (fft_translation-5.f90): spheres binned in cubic cells;    */
/* pairs in neighbouring cells are translated directly, all others through    */
/* regular expansions about the cell nodes and the node-to-node outgoing      */
/* translation, which the reference evaluates as an FFT convolution on the    */
/* zero-padded (2 cell_dim)^3 grid (fft:827-899) with kernels built at every  */
/* node offset outside the neighbour stencil (fft:901-974).  Here the         */
/* convolution is summed directly over node pairs: for offsets inside the     */
/* grid it is the same linear map (the padded grid's wrap-around slots are    */
/* never reached), without the kernels' single-precision rounding.            */
/* ------------------------------------------------------------------------ */

static int checkn235(int n) /* fft:1052-1066 */
{
    int nn = n, ifac = 2;
    for (int ll = 1; ll <= 3; ll++) {
        while (nn % ifac == 0) nn /= ifac;
        ifac += ll;
    }
    return nn == 1;
}
static int correctn235(int n) /* fft:1068-1076; n >= 1 */
{
    int n1 = n < 1 ? 1 : n;
    while (!checkn235(n1)) n1++;
    return n1;
}

/* node_selection (fft:654-825) for free-space external spheres with target
 * box [tmin, tmax] (the sphere-centre extents), and the near-pair list j > i
 * in neighbouring cells; then the dense node translations per sphere and
 * the node-offset kernels.  d_cell > 0 fixes the cell edge (d_cell
 * specified), else cell_volume_fraction (<= 0: from the spheres' volume)
 * sets it; node_order <= 0 means -node_order + ceiling(d_cell)
 * (input:1256-1260).  Returns the node order. */
int orc_fft_setup(orc_ctx *c, double cell_volume_fraction, double d_cell, int node_order, int neighbor_node_model,
                  int *cell_dim_out, double *d_cell_out)
{
    tables_init();
    const int n = c->n;
    double tmin[3] = {1e10, 1e10, 1e10}, tmax[3] = {-1e10, -1e10, -1e10};
    for (int i = 0; i < n; i++)
        for (int m = 0; m < 3; m++) {
            tmin[m] = fmin(tmin[m], c->pos[3 * i + m]);
            tmax[m] = fmax(tmax[m], c->pos[3 * i + m]);
        }
    double amean = 0.0, svol = 0.0;
    for (int i = 0; i < n; i++) { amean += c->rad[i]; svol += c->rad[i] * c->rad[i] * c->rad[i]; }
    svol = pow(svol, 1.0 / 3.0);
    amean = amean / (double)n;
    double tvol = 1.0;
    for (int m = 0; m < 3; m++) tvol *= fmax(tmax[m] - tmin[m], amean);
    double dc = d_cell;
    if (!(d_cell > 0.0)) {
        double fv = cell_volume_fraction;
        if (fv <= 0.0) {
            fv = 4.0 * ORC_REF_PI / 3.0 * svol * svol * svol / tvol;
            fv = fmin(fv, 1.0);
            fv = fmax(fv, 0.02);
        }
        dc = pow(4.0 * ORC_REF_PI / 3.0 / fv / (double)n, 1.0 / 3.0) * svol;
    }
    for (int m = 0; m < 3; m++) c->cd[m] = correctn235((int)ceil((tmax[m] - tmin[m]) / dc));
    dc = 0.0;
    for (int m = 0; m < 3; m++) dc = fmax(dc, (tmax[m] - tmin[m]) / (double)c->cd[m]);
    c->dcell = dc;
    for (int m = 0; m < 3; m++) c->cb[m] = tmin[m];
    c->No = node_order > 0 ? node_order : -node_order + (int)ceil(dc);
    free(c->snode);
    c->snode = (int *)malloc(sizeof(int) * 3 * n);
    for (int i = 0; i < n; i++)
        for (int m = 0; m < 3; m++) {
            int nd = (int)floor((c->pos[3 * i + m] - tmin[m]) / dc) + 1;
            nd = nd < c->cd[m] ? nd : c->cd[m];
            c->snode[3 * i + m] = nd > 1 ? nd : 1;
        }
    c->nnb = 0;
    for (int iz = -1; iz <= 1; iz++)
        for (int iy = -1; iy <= 1; iy++)
            for (int ix = -1; ix <= 1; ix++) {
                int ir = ix * ix + iy * iy + iz * iz;
                if (neighbor_node_model == 0 && ir > 0) continue;
                if (neighbor_node_model == 1 && ir > 1) continue;
                if (neighbor_node_model == 2 && ir > 2) continue;
                c->nb_vec[c->nnb][0] = ix; c->nb_vec[c->nnb][1] = iy; c->nb_vec[c->nnb][2] = iz;
                c->nnb++;
            }
    /* near pairs: for sphere i, cells node(i) - neighbour, members j > i in sphere order */
    int cap = 16, np = 0;
    int *pi = (int *)malloc(sizeof(int) * cap), *pj = (int *)malloc(sizeof(int) * cap);
    for (int i = 0; i < n; i++)
        for (int cell = 0; cell < c->nnb; cell++) {
            int sx = c->snode[3 * i] - c->nb_vec[cell][0], sy = c->snode[3 * i + 1] - c->nb_vec[cell][1], sz = c->snode[3 * i + 2] - c->nb_vec[cell][2];
            if (sx < 1 || sy < 1 || sz < 1 || sx > c->cd[0] || sy > c->cd[1] || sz > c->cd[2]) continue;
            for (int j = i + 1; j < n; j++)
                if (c->snode[3 * j] == sx && c->snode[3 * j + 1] == sy && c->snode[3 * j + 2] == sz) {
                    if (np == cap) { cap *= 2; pi = (int *)realloc(pi, sizeof(int) * cap); pj = (int *)realloc(pj, sizeof(int) * cap); }
                    pi[np] = i; pj[np] = j; np++;
                }
        }
    if (c->ops) { for (int k = 0; k < c->npairs; k++) pairop_free(&c->ops[k]); free(c->ops); c->ops = NULL; }
    c->ops_ready = 0;
    free(c->pi_); free(c->pj_);
    c->pi_ = pi; c->pj_ = pj; c->npairs = np;
    /* dense regular translations sphere <-> node (vswf_type 1); a translation
     * shorter than 1e-3 is the identity on the shared orders, as the
     * reference's zero_translation (r^2 < 1e-6) makes it */
    const int No = c->No, nbN = No * (No + 2);
    free(c->joff); free(c->Jsn); free(c->Jns);
    c->joff = (size_t *)malloc(sizeof(size_t) * (n + 1));
    size_t tot = 0;
    for (int i = 0; i < n; i++) { c->joff[i] = tot; tot += (size_t)2 * nbN * c->order[i] * (c->order[i] + 2); }
    c->joff[n] = tot;
    c->Jsn = (cplx *)calloc(tot, sizeof(cplx));
    c->Jns = (cplx *)calloc(tot, sizeof(cplx));
    for (int i = 0; i < n; i++) {
        double rv[3], r2 = 0.0;
        for (int m = 0; m < 3; m++) {
            rv[m] = dc * ((double)c->snode[3 * i + m] - 0.5) - c->pos[3 * i + m] + c->cb[m];
            r2 += rv[m] * rv[m];
        }
        int L = c->order[i], nb = L * (L + 2);
        if (r2 < 1.0e-6) {
            for (int k = 1; k <= imin(nb, nbN); k++)
                for (int p = 0; p < 2; p++) {
                    c->Jsn[c->joff[i] + (k - 1) + (size_t)nbN * ((k - 1) + (size_t)nb * p)] = 1.0;
                    c->Jns[c->joff[i] + (k - 1) + (size_t)nb * ((k - 1) + (size_t)nbN * p)] = 1.0;
                }
            continue;
        }
        gentranmatrix(L, No, rv, c->rimed, 1, c->Jsn + c->joff[i]);
        double rm[3] = {-rv[0], -rv[1], -rv[2]};
        gentranmatrix(No, L, rm, c->rimed, 1, c->Jns + c->joff[i]);
    }
    /* node-offset kernels H((t - s) d_cell), zero inside the neighbour stencil */
    int ox = 2 * c->cd[0] - 1, oy = 2 * c->cd[1] - 1, oz = 2 * c->cd[2] - 1;
    size_t hsz = (size_t)nbN * nbN * 2;
    free(c->Hc);
    c->Hc = (cplx *)calloc((size_t)ox * oy * oz * hsz, sizeof(cplx));
#pragma omp parallel for schedule(dynamic, 4) num_threads(c->nthreads)
    for (int e = 0; e < ox * oy * oz; e++) {
        int dx = e % ox - (c->cd[0] - 1), dy = (e / ox) % oy - (c->cd[1] - 1), dz = e / (ox * oy) - (c->cd[2] - 1);
        int hole = 0;   /* the stencil is symmetric: offsets equal to a neighbour vector */
        for (int k = 0; k < c->nnb; k++)
            if (dx == c->nb_vec[k][0] && dy == c->nb_vec[k][1] && dz == c->nb_vec[k][2]) hole = 1;
        if (hole) continue;
        double xp[3] = {dc * dx, dc * dy, dc * dz};
        gentranmatrix(No, No, xp, c->rimed, 3, c->Hc + (size_t)e * hsz);
    }
    c->fft = 1;
    if (cell_dim_out) for (int m = 0; m < 3; m++) cell_dim_out[m] = c->cd[m];
    if (d_cell_out) *d_cell_out = dc;
    return No;
}

int orc_fft_near_pairs(const orc_ctx *c, int *pi, int *pj)
{
    if (pi) memcpy(pi, c->pi_, sizeof(int) * c->npairs);
    if (pj) memcpy(pj, c->pj_, sizeof(int) * c->npairs);
    return c->npairs;
}

/* far part of fft_external_to_external_expansion (fft:72-336): with
 * S = shiftcoefficient(-1,-1) for conjugate-transpose columns,
 * g += S Jns conv(Jsn S a). */
static void fft_far_field(orc_ctx *c, int nrhs, const cplx *ain, cplx *gout, const int *contran)
{
    const int n = c->n, No = c->No, nbN = No * (No + 2), neq = c->neqns;
    const int ncell = c->cd[0] * c->cd[1] * c->cd[2];
    const int ox = 2 * c->cd[0] - 1, oy = 2 * c->cd[1] - 1;
    const size_t hsz = (size_t)nbN * nbN * 2;
    cplx *anode = (cplx *)malloc(sizeof(cplx) * (size_t)ncell * nbN * 2);
    cplx *gnode = (cplx *)malloc(sizeof(cplx) * (size_t)ncell * nbN * 2);
    cplx *xt = (cplx *)malloc(sizeof(cplx) * 2 * c->max_order * (c->max_order + 2));
    cplx *yt = (cplx *)malloc(sizeof(cplx) * 2 * c->max_order * (c->max_order + 2));
    for (int r = 0; r < nrhs; r++) {
        const int sv = contran[r] ? -1 : 1;
        for (size_t k = 0; k < (size_t)ncell * nbN * 2; k++) { anode[k] = 0; gnode[k] = 0; }
        for (int i = 0; i < n; i++) {
            int L = c->order[i], nb = L * (L + 2);
            shiftcoefficient(L, sv, sv, ain + (size_t)neq * r + c->offset[i], xt);
            int cell = (c->snode[3 * i] - 1) + c->cd[0] * ((c->snode[3 * i + 1] - 1) + c->cd[1] * (c->snode[3 * i + 2] - 1));
            const cplx *J = c->Jsn + c->joff[i];
            for (int p = 0; p < 2; p++)
                for (int k = 0; k < nbN; k++) {
                    cplx s_ = 0;
                    for (int m = 0; m < nb; m++) s_ += J[k + (size_t)nbN * (m + (size_t)nb * p)] * xt[m + nb * p];
                    anode[(size_t)cell * nbN * 2 + (size_t)nbN * p + k] += s_;
                }
        }
#pragma omp parallel for schedule(static) num_threads(c->nthreads)
        for (int t = 0; t < ncell; t++) {
            int tx = t % c->cd[0], ty = (t / c->cd[0]) % c->cd[1], tz = t / (c->cd[0] * c->cd[1]);
            for (int s_ = 0; s_ < ncell; s_++) {
                int sx = s_ % c->cd[0], sy = (s_ / c->cd[0]) % c->cd[1], sz = s_ / (c->cd[0] * c->cd[1]);
                int e = (tx - sx + c->cd[0] - 1) + ox * ((ty - sy + c->cd[1] - 1) + oy * (tz - sz + c->cd[2] - 1));
                const cplx *H = c->Hc + (size_t)e * hsz;
                for (int p = 0; p < 2; p++)
                    for (int l = 0; l < nbN; l++) {
                        cplx acc = 0;
                        for (int k = 0; k < nbN; k++) acc += H[l + (size_t)nbN * (k + (size_t)nbN * p)] * anode[(size_t)s_ * nbN * 2 + (size_t)nbN * p + k];
                        gnode[(size_t)t * nbN * 2 + (size_t)nbN * p + l] += acc;
                    }
            }
        }
        for (int i = 0; i < n; i++) {
            int L = c->order[i], nb = L * (L + 2);
            int cell = (c->snode[3 * i] - 1) + c->cd[0] * ((c->snode[3 * i + 1] - 1) + c->cd[1] * (c->snode[3 * i + 2] - 1));
            const cplx *J = c->Jns + c->joff[i];
            for (int p = 0; p < 2; p++)
                for (int m = 0; m < nb; m++) {
                    cplx s_ = 0;
                    for (int k = 0; k < nbN; k++) s_ += J[m + (size_t)nb * (k + (size_t)nbN * p)] * gnode[(size_t)cell * nbN * 2 + (size_t)nbN * p + k];
                    yt[m + nb * p] = s_;
                }
            shiftcoefficient(L, sv, sv, yt, xt);
            for (int k = 0; k < 2 * nb; k++) gout[(size_t)neq * r + c->offset[i] + k] += xt[k];
        }
    }
    free(anode); free(gnode); free(xt); free(yt);
}

/* Dense pair translation (coefficient_translation with rot_op false): gen_mat
 * = gentranmatrix(L_j -> L_i, r_i - r_j); j -> i uses gen_mat, i -> j its
 * transpose; shiftcoefficient(-1,-1) on input and output when shift_op
 * differs from tran_op. */
static void dense_pair_apply(const orc_ctx *c, int i, int j, int nrhs, const cplx *ain, cplx *g, const int *contran)
{
    int Li = c->order[i], Lj = c->order[j], nbi = Li * (Li + 2), nbj = Lj * (Lj + 2), neq = c->neqns;
    cplx *H = (cplx *)malloc(sizeof(cplx) * (size_t)nbi * nbj * 2);
    double rv[3] = {c->pos[3 * i] - c->pos[3 * j], c->pos[3 * i + 1] - c->pos[3 * j + 1], c->pos[3 * i + 2] - c->pos[3 * j + 2]};
    gentranmatrix(Lj, Li, rv, c->rext[i], 3, H);
    cplx *a = (cplx *)malloc(sizeof(cplx) * 2 * (nbi > nbj ? nbi : nbj));
    cplx *o = (cplx *)malloc(sizeof(cplx) * 2 * (nbi > nbj ? nbi : nbj));
    for (int r = 0; r < nrhs; r++) {
        int top = contran[r] != 0;
        /* j -> i: shift when tran_op (shift_op false) */
        int sv = top ? -1 : 1;
        shiftcoefficient(Lj, sv, sv, ain + (size_t)neq * r + c->offset[j], a);
        for (int p = 0; p < 2; p++)
            for (int t = 0; t < nbi; t++) {
                cplx acc = 0;
                for (int s_ = 0; s_ < nbj; s_++) acc += H[t + (size_t)nbi * (s_ + (size_t)nbj * p)] * a[s_ + nbj * p];
                o[t + nbi * p] = acc;
            }
        shiftcoefficient(Li, sv, sv, o, o);
        for (int k = 0; k < 2 * nbi; k++) g[(size_t)neq * r + c->offset[i] + k] += o[k];
        /* i -> j: shift when not tran_op (shift_op true) */
        sv = top ? 1 : -1;
        shiftcoefficient(Li, sv, sv, ain + (size_t)neq * r + c->offset[i], a);
        for (int p = 0; p < 2; p++)
            for (int s_ = 0; s_ < nbj; s_++) {
                cplx acc = 0;
                for (int t = 0; t < nbi; t++) acc += a[t + nbi * p] * H[t + (size_t)nbi * (s_ + (size_t)nbj * p)];
                o[s_ + nbj * p] = acc;
            }
        shiftcoefficient(Lj, sv, sv, o, o);
        for (int k = 0; k < 2 * nbj; k++) g[(size_t)neq * r + c->offset[j] + k] += o[k];
    }
    free(H); free(a); free(o);
}

static void external_to_external(orc_ctx *c, int nrhs, const cplx *ain, cplx *gout, const int *contran, int initial_run)
{
    int neq = c->neqns;
    for (size_t k = 0; k < (size_t)neq * nrhs; k++) gout[k] = 0;
    if (c->store && (initial_run || !c->ops_ready)) {
        if (c->ops) { for (int k = 0; k < c->npairs; k++) pairop_free(&c->ops[k]); free(c->ops); }
        c->ops = (pairop_t *)calloc(c->npairs > 0 ? c->npairs : 1, sizeof(pairop_t));
#pragma omp parallel for schedule(dynamic, 16) num_threads(c->nthreads)
        for (int t = 0; t < c->npairs; t++) {
            int i = c->pi_[t], j = c->pj_[t];
            double rv[3] = {c->pos[3 * i] - c->pos[3 * j], c->pos[3 * i + 1] - c->pos[3 * j + 1], c->pos[3 * i + 2] - c->pos[3 * j + 2]};
            pairop_compute(&c->ops[t], c->order[i], c->order[j], rv, 3, c->rext[i]);
        }
        c->ops_ready = 1;
    }
    int nth = c->nthreads;
    cplx *priv = (cplx *)calloc((size_t)neq * nrhs * nth, sizeof(cplx));
#pragma omp parallel num_threads(nth)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        cplx *g = priv + (size_t)neq * nrhs * tid;
#pragma omp for schedule(dynamic, 16)
        for (int t = 0; t < c->npairs; t++) {
            int i = c->pi_[t], j = c->pj_[t];
            int noi = c->order[i], noj = c->order[j];
            pairop_t local;
            const pairop_t *op;
            if (c->store) op = &c->ops[t];
            else {
                double rv[3] = {c->pos[3 * i] - c->pos[3 * j], c->pos[3 * i + 1] - c->pos[3 * j + 1], c->pos[3 * i + 2] - c->pos[3 * j + 2]};
                pairop_compute(&local, noi, noj, rv, 3, c->rext[i]);
                op = &local;
            }
            if (imin(noi, noj) < 3) {
                /* dense branch of coefficient_translation (modules:6751-6780), translation_switch_order 3 */
                dense_pair_apply(c, i, j, nrhs, ain, g, contran);
                if (!c->store) pairop_free(&local);
                continue;
            }
            for (int r = 0; r < nrhs; r++) {
                coefficient_translation(noj, noi, ain + (size_t)neq * r + c->offset[j], g + (size_t)neq * r + c->offset[i], op, 0, contran[r]);
                coefficient_translation(noi, noj, ain + (size_t)neq * r + c->offset[i], g + (size_t)neq * r + c->offset[j], op, 1, contran[r]);
            }
            if (!c->store) pairop_free(&local);
        }
    }
    for (int t = 0; t < nth; t++)
        for (size_t k = 0; k < (size_t)neq * nrhs; k++) gout[k] += priv[(size_t)neq * nrhs * t + k];
    free(priv);
    if (c->fft) fft_far_field(c, nrhs, ain, gout, contran);
}

/* external_to_internal_expansion (modules:6533-6608): for each host and a
 * sphere it holds, the regular translation (vswf_type 1, in the host's
 * index) of the sphere's scattered coefficients into the host's internal
 * block, and of the host's internal block back onto the sphere (shift_op);
 * coincident centres copy the common orders (mtransfer).  bout is zeroed. */
static void external_to_internal(orc_ctx *c, int nrhs, const cplx *ain, cplx *bout, const int *contran)
{
    int neq = c->neqns;
    for (size_t k = 0; k < (size_t)neq * nrhs; k++) bout[k] = 0;
    if (!c->hops) {
        c->hops = (pairop_t *)calloc(c->nhp > 0 ? c->nhp : 1, sizeof(pairop_t));
        for (int t = 0; t < c->nhp; t++) {
            int hi = c->hpi[t], e = c->hpj[t];
            double rv[3] = {c->pos[3 * hi] - c->pos[3 * e], c->pos[3 * hi + 1] - c->pos[3 * e + 1], c->pos[3 * hi + 2] - c->pos[3 * e + 2]};
            pairop_compute(&c->hops[t], c->order[hi], c->order[e], rv, 1, c->ri[hi]);
        }
    }
    for (int t = 0; t < c->nhp; t++) {
        int hi = c->hpi[t], e = c->hpj[t];
        int noint = c->order[hi], noext = c->order[e];
        int ext1 = c->offset[e], int1 = c->offset[hi] + noint * (noint + 2) * 2;
        for (int r = 0; r < nrhs; r++) {
            coefficient_translation(noext, noint, ain + (size_t)neq * r + ext1, bout + (size_t)neq * r + int1, &c->hops[t], 0, contran[r]);
            coefficient_translation(noint, noext, ain + (size_t)neq * r + int1, bout + (size_t)neq * r + ext1, &c->hops[t], 1, contran[r]);
        }
    }
}

/* sphereinteraction (scatprops:25-180) without plane boundaries or periodic
 * lattices; skip_external leaves out external_to_external_expansion */
static void sphereinteraction_ex(orc_ctx *c, int nrhs, const cplx *ain, cplx *aout, const int *con_tran,
                                 const int *mie_mult, int initial_run, int skip_external)
{
    int neq = c->neqns;
    cplx *ain_t = (cplx *)malloc(sizeof(cplx) * neq * nrhs);
    cplx *aout_t = (cplx *)malloc(sizeof(cplx) * neq * nrhs);
    int *ct = (int *)calloc(nrhs, sizeof(int));
    for (int r = 0; r < nrhs; r++) {
        int contran = con_tran ? con_tran[r] : 0;
        int mm = mie_mult ? mie_mult[r] : 1;
        ct[r] = contran;
        const cplx *x = ain + (size_t)neq * r;
        cplx *t = ain_t + (size_t)neq * r;
        if (contran) {
            for (int k = 0; k < neq; k++) t[k] = conj(x[k]);
            if (mm) multmiecoeffmult(c, -1, t, t, c->an);
        } else {
            memcpy(t, x, sizeof(cplx) * neq);
        }
    }
    if (skip_external) {
        for (size_t k = 0; k < (size_t)neq * nrhs; k++) aout_t[k] = 0;
    } else {
        external_to_external(c, nrhs, ain_t, aout_t, ct, initial_run);
    }
    if (c->nhosted > 0) {
        cplx *t2 = (cplx *)malloc(sizeof(cplx) * neq * nrhs);
        external_to_internal(c, nrhs, ain_t, t2, ct);
        for (size_t k = 0; k < (size_t)neq * nrhs; k++) aout_t[k] += t2[k];
        free(t2);
    }
    for (int r = 0; r < nrhs; r++) {
        int mm = mie_mult ? mie_mult[r] : 1;
        cplx *o = aout + (size_t)neq * r;
        cplx *t = aout_t + (size_t)neq * r;
        if (!ct[r]) {
            if (mm) multmiecoeffmult(c, 1, t, o, c->an);
            else memcpy(o, t, sizeof(cplx) * neq);
        } else {
            for (int k = 0; k < neq; k++) o[k] = conj(t[k]);
        }
    }
    free(ain_t); free(aout_t); free(ct);
}
void orc_sphereinteraction(orc_ctx *c, int nrhs, const cplx *ain, cplx *aout, const int *con_tran,
                           const int *mie_mult, int initial_run)
{
    sphereinteraction_ex(c, nrhs, ain, aout, con_tran, mie_mult, initial_run, 0);
}
void orc_sphereinteraction_ex(orc_ctx *c, int nrhs, const cplx *ain, cplx *aout, const int *con_tran,
                              const int *mie_mult, int initial_run, int skip_external)
{
    sphereinteraction_ex(c, nrhs, ain, aout, con_tran, mie_mult, initial_run, skip_external);
}

/* Fortran dot_product for complex: sum(conj(a)*b) */
static cplx dotc(const cplx *a, const cplx *b, int n)
{
    cplx s = 0;
    for (int k = 0; k < n; k++) s += conj(a[k]) * b[k];
    return s;
}

/* cbicg (solver:654-949), single-rank branch; niter>0 only.
 * Returns 0 on normal exit (converged or iteration cap), 2 on zero pivot. */
int orc_cbicg(orc_ctx *c, int niter, double eps, const cplx *pnp, cplx *anp, int initialize, int *iter_o, double *err_o)
{
    int neq = c->neqns;
    *iter_o = 0; *err_o = 0.0;
    if (creal(dotc(pnp, pnp, neq)) == 0.0 && cimag(dotc(pnp, pnp, neq)) == 0.0) return 0;
    cplx *cr = (cplx *)malloc(sizeof(cplx) * neq), *cp = (cplx *)malloc(sizeof(cplx) * neq);
    cplx *cw = (cplx *)malloc(sizeof(cplx) * neq), *cq = (cplx *)malloc(sizeof(cplx) * neq);
    cplx *cap = (cplx *)malloc(sizeof(cplx) * neq), *caw = (cplx *)malloc(sizeof(cplx) * neq);
    cplx *ctin = (cplx *)malloc(sizeof(cplx) * neq * 2), *ctout = (cplx *)malloc(sizeof(cplx) * neq * 2);
    double enorm = creal(dotc(pnp, pnp, neq));   /* normalize_solution_error = T */
    double errmin = 1.0e10, errmax = 0.0;
    int one0 = 0, rc = 0, iter;
    if (niter < 0) {
        /* order-of-scattering iteration (solver:787-822): x += M H p, p = M H p */
        memcpy(cp, anp, sizeof(cplx) * neq);
        for (iter = 1; iter <= -niter; iter++) {
            orc_sphereinteraction(c, 1, cp, cr, &one0, NULL, iter == 1 ? initialize : 0);
            for (int k = 0; k < neq; k++) { anp[k] += cr[k]; cp[k] = cr[k]; }
            double eerr = creal(dotc(cr, cr, neq)) / enorm;
            if (eerr < eps) { errmax = eerr; break; }
        }
        *iter_o = iter;
        *err_o = errmax;
        free(cr); free(cp); free(cw); free(cq); free(cap); free(caw); free(ctin); free(ctout);
        return 0;
    }
    orc_sphereinteraction(c, 1, anp, cr, &one0, NULL, initialize);
    for (int k = 0; k < neq; k++) cr[k] = pnp[k] - anp[k] + cr[k];
    for (int k = 0; k < neq; k++) { cq[k] = conj(cr[k]); cw[k] = cq[k]; cp[k] = cr[k]; }
    cplx csk = 0;
    for (int k = 0; k < neq; k++) csk += cr[k] * cr[k];   /* dot_product(conjg(cr),cr) */
    if (cabs(csk) == 0.0) { iter = 0; goto done; }
    int contran2[2] = {0, 1};
    for (iter = 1; iter <= niter; iter++) {
        memcpy(ctin, cp, sizeof(cplx) * neq);
        memcpy(ctin + neq, cw, sizeof(cplx) * neq);
        orc_sphereinteraction(c, 2, ctin, ctout, contran2, NULL, 0);
        for (int k = 0; k < neq; k++) { cap[k] = cp[k] - ctout[k]; caw[k] = cw[k] - ctout[neq + k]; }
        cplx cak = dotc(cw, cap, neq);
        if (cabs(cak) != 0.0) cak = csk / cak;
        else { rc = 2; break; }
        for (int k = 0; k < neq; k++) anp[k] = anp[k] + cak * cp[k];
        for (int k = 0; k < neq; k++) cr[k] = cr[k] - cak * cap[k];
        for (int k = 0; k < neq; k++) cq[k] = cq[k] - conj(cak) * caw[k];
        cplx csk2 = dotc(cq, cr, neq);
        double eerr = creal(dotc(cr, cr, neq)) / enorm;
        errmax = eerr;
        errmin = errmin < errmax ? errmin : errmax;
        if (eerr < eps || cabs(csk) == 0.0) break;
        cplx cbk = csk2 / csk;
        csk = csk2;
        for (int k = 0; k < neq; k++) cp[k] = cr[k] + cbk * cp[k];
        for (int k = 0; k < neq; k++) cw[k] = cq[k] + conj(cbk) * cw[k];
    }
done:
    *iter_o = iter;
    *err_o = errmax;
    free(cr); free(cp); free(cw); free(cq); free(cap); free(caw); free(ctin); free(ctout);
    return rc;
}

/* genplanewavecoef (modules:1453-1520), LR form, complex cos(beta).
 * pmnp0(0:nodr+1, nodr, 2 modes, 2 polarisations) */
static void genplanewavecoef(double alpha, cplx cb, int nodr, cplx *pmnp0)
{
    int nd = nodr * (nodr + 2) + 1;
    cplx *drot = (cplx *)malloc(sizeof(cplx) * 3 * nd);
    crotcoef(cb, 1, nodr, drot);
#define DR(m, nk) drot[((m) + 1) + 3 * (nk)]
    int nb = 2 * nodr * (nodr + 2);
    cplx *tau = (cplx *)calloc(nb, sizeof(cplx));   /* tau(0:nodr+1,nodr,2) */
    for (int n = 1; n <= nodr; n++) {
        int nn1 = n * (n + 1);
        double fnm = sqrt((double)(n + n + 1) / 2.0) / 4.0;
        for (int m = -n; m <= -1; m++) {
            int mn = nn1 + m;
            tau[AIDX(n + 1, -m, 0, nodr)] = -fnm * (-DR(-1, mn) + DR(1, mn));
            tau[AIDX(n + 1, -m, 1, nodr)] = -fnm * (DR(-1, mn) + DR(1, mn));
        }
        for (int m = 0; m <= n; m++) {
            int mn = nn1 + m;
            tau[AIDX(m, n, 0, nodr)] = -fnm * (-DR(-1, mn) + DR(1, mn));
            tau[AIDX(m, n, 1, nodr)] = -fnm * (DR(-1, mn) + DR(1, mn));
        }
    }
#undef DR
    double ca = cos(alpha), sa = sin(alpha);
    cplx ealpha = ca + CI * sa;
    cplx *ealpham = (cplx *)malloc(sizeof(cplx) * (2 * nodr + 1));
    ephicoef(ealpha, nodr, ealpham);
    int half = nb / 2;
    cplx *taulr = (cplx *)malloc(sizeof(cplx) * nb);
    for (int k = 0; k < half; k++) {
        taulr[k] = (tau[k] + tau[half + k]) * 0.5;
        taulr[half + k] = (tau[k] - tau[half + k]) * 0.5;
    }
    for (int n = 1; n <= nodr; n++) {
        int e = (n + 1) % 4;
        cplx ipow = (e == 0) ? 1.0 : (e == 1 ? CI : (e == 2 ? -1.0 : -CI));
        cplx cin = 4.0 * ipow;
        for (int p = 1; p <= 2; p++) {
            double sp = -pm1(p);
            for (int m = -n; m <= -1; m++) {
                int a = AIDX(n + 1, -m, p - 1, nodr);
                pmnp0[a] = -cin * taulr[a] * ealpham[nodr - m];
                pmnp0[nb + a] = sp * CI * cin * taulr[a] * ealpham[nodr - m];
            }
            for (int m = 0; m <= n; m++) {
                int a = AIDX(m, n, p - 1, nodr);
                pmnp0[a] = -cin * taulr[a] * ealpham[nodr - m];
                pmnp0[nb + a] = sp * CI * cin * taulr[a] * ealpham[nodr - m];
            }
        }
    }
    free(drot); free(tau); free(ealpham); free(taulr);
}

/* sphereplanewavecoef (scatprops:217-284) -> layerplanewavecoef
 * (modules:3901-3965) with no plane boundaries: medium index 1, source plane
 * z=0, field scale 1.  pmnp(neqns, 2) column-major. */
void orc_planewave(const orc_ctx *c, double alpha, double sinc, int dir, cplx *pmnp)
{
    int neq = c->neqns;
    cplx riinc = c->rimed;
    cplx cbinc = csqrt((1.0 - sinc / riinc) * (1.0 + sinc / riinc)) * (double)(3 - 2 * dir);
    double ca = cos(alpha), sa = sin(alpha);
    cplx s = sinc;
    for (size_t k = 0; k < (size_t)neq * 2; k++) pmnp[k] = 0;
    for (int i = 0; i < c->n; i++) {
        if (c->host[i] >= 0) continue;   /* spheres inside others see no incident wave (scatprops:268) */
        int L = c->order[i], nb = 2 * L * (L + 2);
        cplx *pw = (cplx *)malloc(sizeof(cplx) * nb * 2);
        genplanewavecoef(alpha, cbinc, L, pw);
        const double *rp = c->pos + 3 * i;
        cplx phz = cexp(CI * riinc * cbinc * (rp[2] - 0.0));
        cplx phl = cexp(CI * s * (ca * rp[0] + sa * rp[1]));
        for (int p = 0; p < 2; p++)
            for (int k = 0; k < nb; k++)
                pmnp[(size_t)neq * p + c->offset[i] + k] = (pw[nb * p + k] * phz) * phl / 1.0;
        free(pw);
    }
}

/* lrsphereqeff (scatprops:676-776), npol=2 */
static void lrsphereqeff(cplx ri0, int nodr, double xsp, const cplx *anp /*(nb,2)*/, int lda,
                         const cplx *gnpinc, const cplx *gnp, double *qe, double *qs, double *qa)
{
    int npol = 2;
    double qi[3] = {0, 0, 0};
    for (int k = 0; k < 3; k++) { qe[k] = 0; qa[k] = 0; qs[k] = 0; }
    cplx xri = xsp * ri0;   /* both helicities equal */
    cplx rib = 2.0 / (1.0 / ri0 + 1.0 / ri0);
    cplx *psi = (cplx *)malloc(sizeof(cplx) * (nodr + 1));
    cplx *xi = (cplx *)malloc(sizeof(cplx) * (nodr + 1));
    cricbessel(nodr, xri, psi);
    crichankel(nodr, xri, xi);
    for (int n = 1; n <= nodr; n++) {
        cplx psip = psi[n - 1] - (double)n * psi[n] / xri;
        cplx xip = xi[n - 1] - (double)n * xi[n] / xri;
        cplx aamat[4], ggmat[4], agmat[4];
        for (int s = 1; s <= 2; s++) {
            double ss = pm1(s);
            for (int t = 1; t <= 2; t++) {
                double st = pm1(t);
                cplx cterm = CI * conj(1.0 / ri0) / ri0;
                M2(aamat, s, t) = cterm * (xip * conj(xi[n]) - ss * st * xi[n] * conj(xip));
                M2(ggmat, s, t) = cterm * (psip * conj(psi[n]) - ss * st * psi[n] * conj(psip));
                M2(agmat, s, t) = cterm * (xip * conj(psi[n]) - ss * st * xi[n] * conj(psip));
            }
        }
        for (int m = -n; m <= n; m++) {
            int ma, na;
            if (m <= -1) { ma = n + 1; na = -m; } else { ma = m; na = n; }
            for (int p1 = 1; p1 <= npol; p1++)
                for (int p2 = 1; p2 <= npol; p2++) {
                    int k; double cst;
                    if (p1 == 1 && p2 == 1) { k = 0; cst = 1.0; }
                    else if (p1 == 2 && p2 == 2) { k = 1; cst = 1.0; }
                    else { k = 2; cst = 0.5; }
                    for (int s = 1; s <= 2; s++)
                        for (int t = 1; t <= 2; t++) {
                            cplx as1 = anp[AIDX(ma, na, s - 1, nodr) + (size_t)lda * (p1 - 1)];
                            cplx at2 = anp[AIDX(ma, na, t - 1, nodr) + (size_t)lda * (p2 - 1)];
                            cplx gs1 = gnp[AIDX(ma, na, s - 1, nodr) + (size_t)lda * (p1 - 1)];
                            cplx gt2 = gnp[AIDX(ma, na, t - 1, nodr) + (size_t)lda * (p2 - 1)];
                            cplx fs1 = gnpinc[AIDX(ma, na, s - 1, nodr) + (size_t)lda * (p1 - 1)];
                            cplx ft2 = gnpinc[AIDX(ma, na, t - 1, nodr) + (size_t)lda * (p2 - 1)];
                            double sgn = pm1(s + t);
                            qi[k] = qi[k] + creal(cst * M2(ggmat, s, t) * fs1 * conj(rib * ft2));
                            qa[k] = qa[k] + creal(cst * (M2(aamat, s, t) * as1 * conj(rib * at2)
                                                         + M2(ggmat, s, t) * gs1 * conj(rib * gt2)
                                                         + M2(agmat, s, t) * as1 * conj(gt2) * (conj(rib) + sgn * rib)));
                            qs[k] = qs[k] - creal(cst * M2(aamat, s, t) * as1 * conj(rib * at2));
                            qe[k] = qe[k] + creal(cst * (M2(agmat, s, t) * as1 * conj(ft2) * (conj(rib) + sgn * rib)));
                        }
                }
        }
    }
    for (int k = 0; k < 2 * npol - 1; k++) {
        qi[k] = qi[k] * 2.0 / xsp / xsp;
        qe[k] = qe[k] * 2.0 / xsp / xsp;
        qa[k] = qa[k] * 2.0 / xsp / xsp;
        qs[k] = qi[k];
    }
    free(psi); free(xi);
}

/* qefficiencyfactors (scatprops:782-870), npol=2.
 * qeff(3,3,N) column-major: qeff[q + 3*(pol + 3*i)], q: ext,abs,sca(inc).
 * Without host spheres the exciting field is A^{-1} a; with them it is the
 * interaction without the Mie multiply plus the incident field. */
static void qefficiencyfactors(orc_ctx *c, const cplx *amnp, const cplx *gmnp0, double *qeff)
{
    int neq = c->neqns;
    cplx *gmnp = (cplx *)calloc((size_t)neq * 2, sizeof(cplx));
    if (c->nhosted == 0) {
        for (int p = 0; p < 2; p++)
            for (int i = 0; i < c->n; i++)
                mie_mult_sphere(c->an_inv + c->mie_offset[i], c->order[i], 1, amnp + (size_t)neq * p + c->offset[i],
                                gmnp + (size_t)neq * p + c->offset[i]);
    } else {
        int zero = 0;
        for (int p = 0; p < 2; p++) {
            sphereinteraction_ex(c, 1, amnp + (size_t)neq * p, gmnp + (size_t)neq * p, &zero, &zero, 0, 0);
            for (int k = 0; k < neq; k++) gmnp[(size_t)neq * p + k] += gmnp0[(size_t)neq * p + k];
        }
    }
    for (int i = 0; i < c->n; i++) {
        double qe[3], qs[3], qa[3];
        int off = c->offset[i];
        lrsphereqeff(c->rext[i], c->order[i], c->rad[i], amnp + off, neq, gmnp0 + off, gmnp + off, qe, qs, qa);
        double qeffi[3][3];  /* [q][k] */
        for (int k = 0; k < 3; k++) { qeffi[0][k] = qe[k]; qeffi[2][k] = qs[k]; qeffi[1][k] = qa[k]; }
        for (int q = 0; q < 3; q++) {
            qeff[q + 3 * (0 + 3 * i)] = 0.5 * (qeffi[q][0] + qeffi[q][1]);
            qeff[q + 3 * (1 + 3 * i)] = qeffi[q][0];
            qeff[q + 3 * (2 + 3 * i)] = qeffi[q][1];
        }
    }
    free(gmnp);
}

/* vol_radius as main_calling_program forms it, over the spheres outside
 * every other: (sum r^3)**.333333 where .333333 is a default-real (single
 * precision) literal (input:1218-1225). */
double orc_vol_radius(const orc_ctx *c)
{
    double v = 0.0;
    for (int i = 0; i < c->n; i++)
        if (c->host[i] < 0) v = v + c->rad[i] * c->rad[i] * c->rad[i];
    return pow(v, (double)0.333333f);
}

/* qtotcalc (scatprops:872-912); qtot(3,3) column-major.  A host's absorption
 * net of the spheres it holds (qabsvol), then the holds' added back, each
 * scaled by the area ratio; qeff's absorption rows are rewritten as the
 * reference does.  The totals sum the spheres outside every other. */
void orc_qtotcalc(const orc_ctx *c, double *qeff, double *qtot)
{
    int n = c->n;
    double xg = orc_vol_radius(c);
    if (c->nhosted > 0) {
        double *qv = (double *)malloc(sizeof(double) * 3 * n);
        for (int i = 0; i < n; i++)
            for (int p = 0; p < 3; p++) {
                double v = qeff[1 + 3 * (p + 3 * i)];
                for (int j = 0; j < n; j++)
                    if (c->host[j] == i) v = v - qeff[1 + 3 * (p + 3 * j)] * c->rad[j] * c->rad[j] / (c->rad[i] * c->rad[i]);
                qv[p + 3 * i] = v;
            }
        for (int i = 0; i < n; i++)
            for (int p = 0; p < 3; p++) {
                double v = qv[p + 3 * i];
                for (int j = 0; j < n; j++)
                    if (c->host[j] == i) v = v + qv[p + 3 * j] * c->rad[j] * c->rad[j] / (c->rad[i] * c->rad[i]);
                qeff[1 + 3 * (p + 3 * i)] = v;
            }
        free(qv);
    }
    for (int k = 0; k < 9; k++) qtot[k] = 0.0;
    for (int i = 0; i < n; i++)
        if (c->host[i] < 0)
            for (int k = 0; k < 9; k++) qtot[k] = qtot[k] + qeff[k + 9 * i] * c->rad[i] * c->rad[i] / (xg * xg);
    for (int pol = 0; pol < 3; pol++) qtot[2 + 3 * pol] = qtot[0 + 3 * pol] + qtot[2 + 3 * pol] - qtot[1 + 3 * pol];
}

/* dense (I - Mie H) from gentranmatrix (modules:5854-5985) + LU with three
 * refinement steps (solver:571-642, 951-1052). */
static void lu_decomposition(cplx *a, int n, int *indx)
{
#define A_(i, j) a[((i) - 1) + (size_t)n * ((j) - 1)]
    double *vv = (double *)malloc(sizeof(double) * (n + 1));
    const double tiny = 1.0e-20;
    for (int i = 1; i <= n; i++) {
        double aamax = 0.0;
        for (int j = 1; j <= n; j++) if (cabs(A_(i, j)) > aamax) aamax = cabs(A_(i, j));
        vv[i] = 1.0 / aamax;
    }
    for (int j = 1; j <= n; j++) {
        for (int i = 1; i <= j - 1; i++) {
            cplx sum = A_(i, j);
            for (int k = 1; k <= i - 1; k++) sum -= A_(i, k) * A_(k, j);
            A_(i, j) = sum;
        }
        double aamax = 0.0;
        int imx = j;
        for (int i = j; i <= n; i++) {
            cplx sum = A_(i, j);
            for (int k = 1; k <= j - 1; k++) sum -= A_(i, k) * A_(k, j);
            A_(i, j) = sum;
            double dum = vv[i] * cabs(sum);
            if (dum >= aamax) { imx = i; aamax = dum; }
        }
        if (j != imx) {
            for (int k = 1; k <= n; k++) { cplx d = A_(imx, k); A_(imx, k) = A_(j, k); A_(j, k) = d; }
            vv[imx] = vv[j];
        }
        indx[j - 1] = imx;
        if (j != n) {
            if (cabs(A_(j, j)) == 0.0) A_(j, j) = tiny;
            cplx cd = 1.0 / A_(j, j);
            for (int i = j + 1; i <= n; i++) A_(i, j) = A_(i, j) * cd;
        }
    }
    if (cabs(A_(n, n)) == 0.0) A_(n, n) = tiny;
    free(vv);
}
static void lu_backsubstitution(const cplx *a, int n, const int *indx, cplx *b)
{
    int ii = 0;
    for (int i = 1; i <= n; i++) {
        int ll = indx[i - 1];
        cplx sum = b[ll - 1];
        b[ll - 1] = b[i - 1];
        if (ii != 0) { for (int j = ii; j <= i - 1; j++) sum -= A_(i, j) * b[j - 1]; }
        else if (cabs(sum) != 0.0) ii = i;
        b[i - 1] = sum;
    }
    for (int i = n; i >= 1; i--) {
        cplx sum = b[i - 1];
        for (int j = i + 1; j <= n; j++) sum -= A_(i, j) * b[j - 1];
        b[i - 1] = sum / A_(i, i);
    }
#undef A_
}

static void direct_solve(orc_ctx *c, const cplx *pnp, cplx *anp)
{
    int neq = c->neqns;
    cplx *amat = (cplx *)calloc((size_t)neq * neq, sizeof(cplx));
    cplx *col = NULL;
    if (c->nhosted > 0) {
        /* with host spheres: column k of I - M H is e_k minus the interaction
         * of e_k (the same linear map general_interaction_matrix assembles
         * block by block, modules:5854-5985) */
        cplx *e = (cplx *)calloc(neq, sizeof(cplx));
        int zero = 0;
        for (int k = 0; k < neq; k++) {
            e[k] = 1.0;
            sphereinteraction_ex(c, 1, e, amat + (size_t)neq * k, &zero, NULL, 0, 0);
            e[k] = 0.0;
            for (int r = 0; r < neq; r++) amat[(size_t)neq * k + r] = -amat[(size_t)neq * k + r];
            amat[(size_t)neq * k + k] += 1.0;
        }
        free(e);
        goto factor;
    }
    for (int i = 0; i < c->n; i++) {
        int nbi = c->order[i] * (c->order[i] + 2);
        for (int j = 0; j < c->n; j++) {
            int nbj = c->order[j] * (c->order[j] + 2);
            double rp[3] = {c->pos[3 * i] - c->pos[3 * j], c->pos[3 * i + 1] - c->pos[3 * j + 1], c->pos[3 * i + 2] - c->pos[3 * j + 2]};
            cplx *fs = (cplx *)malloc(sizeof(cplx) * nbi * nbj * 2);
            gentranmatrix(c->order[j], c->order[i], rp, c->rimed, 3, fs);
            for (int p = 0; p < 2; p++)
                for (int cc = 0; cc < nbj; cc++)
                    for (int rr = 0; rr < nbi; rr++)
                        amat[(size_t)(c->offset[i] + p * nbi + rr) + (size_t)neq * (c->offset[j] + p * nbj + cc)] = fs[rr + (size_t)nbi * (cc + (size_t)nbj * p)];
            free(fs);
        }
    }
    col = (cplx *)malloc(sizeof(cplx) * neq);
    for (int j = 0; j < neq; j++) {
        cplx *mj = amat + (size_t)neq * j;
        int nz = 0;
        for (int k = 0; k < neq; k++) if (cabs(mj[k]) != 0.0) { nz = 1; break; }
        if (nz) {
            multmiecoeffmult(c, 1, mj, col, c->an);
            for (int k = 0; k < neq; k++) mj[k] = -col[k];
        }
        mj[j] += 1.0;
    }
factor:;
    cplx *lu = (cplx *)malloc(sizeof(cplx) * (size_t)neq * neq);
    memcpy(lu, amat, sizeof(cplx) * (size_t)neq * neq);
    int *indx = (int *)malloc(sizeof(int) * neq);
    lu_decomposition(lu, neq, indx);
    memcpy(anp, pnp, sizeof(cplx) * neq);
    lu_backsubstitution(lu, neq, indx, anp);
    cplx *rnp = (cplx *)malloc(sizeof(cplx) * neq);
    for (int it = 1; it <= 3; it++) {
        for (int i = 0; i < neq; i++) {
            cplx s = 0;
            for (int j = 0; j < neq; j++) s += amat[i + (size_t)neq * j] * anp[j];
            rnp[i] = s - pnp[i];
        }
        lu_backsubstitution(lu, neq, indx, rnp);
        for (int i = 0; i < neq; i++) anp[i] -= rnp[i];
    }
    free(amat); free(col); free(lu); free(indx); free(rnp);
}

/* fixedorsoln (solver:350-569), single rank.  amnp(neqns,2); qeff(3,3,N).
 * direct != 0 uses the dense LU path (solution_method='d'). */
int orc_fixedorsoln(orc_ctx *c, double alpha, double sinc, int dir, double eps, int niter,
                    cplx *amnp, double *qeff, double *maxerr, int *maxiter, int direct)
{
    int neq = c->neqns;
    cplx *pmnp0 = (cplx *)malloc(sizeof(cplx) * neq * 2);
    cplx *pmnpan = (cplx *)malloc(sizeof(cplx) * neq);
    orc_planewave(c, alpha, sinc, dir, pmnp0);
    int istat = 0, initialize = 1;
    *maxiter = 0; *maxerr = 0.0;
    for (int p = 0; p < 2; p++) {
        istat = 0;
        *maxiter = 0;
        *maxerr = 0.0;
        multmiecoeffmult(c, 1, pmnp0 + (size_t)neq * p, pmnpan, c->an);
        memcpy(amnp + (size_t)neq * p, pmnpan, sizeof(cplx) * neq);
        int iter = 0; double serr = 0.0;
        if (niter != 0) {
            if (direct) direct_solve(c, pmnpan, amnp + (size_t)neq * p);
            else orc_cbicg(c, niter, eps, pmnpan, amnp + (size_t)neq * p, initialize, &iter, &serr);
        } else if (c->nhosted > 0) {
            /* the coupling of the spheres inside hosts alone (solver:509-518) */
            int zero = 0;
            cplx *t = (cplx *)calloc(neq, sizeof(cplx));
            sphereinteraction_ex(c, 1, amnp + (size_t)neq * p, t, &zero, NULL, initialize, 1);
            sphereinteraction_ex(c, 1, t, t, &zero, NULL, 0, 1);
            for (int k = 0; k < neq; k++) amnp[(size_t)neq * p + k] += t[k];
            free(t);
        }
        initialize = 0;
        c->last_iter[p] = iter;
        *maxiter = imax(iter, *maxiter);
        *maxerr = serr > *maxerr ? serr : *maxerr;
        if (iter > niter || serr > eps) istat = 1;
    }
    qefficiencyfactors(c, amnp, pmnp0, qeff);
    free(pmnp0); free(pmnpan);
    return istat;
}

/* Iteration counts of both polarisations of the last orc_fixedorsoln (the
 * reference reports only the second one, solver:524-531). */
void orc_last_iterations(const orc_ctx *c, int *iters2) { iters2[0] = c->last_iter[0]; iters2[1] = c->last_iter[1]; }

/* ---- low-level exports used by the unit tests ---- */
void orc_x_rotcoef(double cbe, int kmax, int nmax, double *dc) { tables_init(); rotcoef(cbe, kmax, nmax, dc); }
void orc_x_vcfunc(int m, int n, int k, int l, double *vcn) { tables_init(); vcfunc(m, n, k, l, vcn); }
int orc_x_atcdim(int n, int l) { return atcdim(n, l); }
int orc_x_moffset(int m, int n, int l) { return moffset(m, n, l); }
void orc_x_axial(int itype, double r, double rire, double riim, int nmax, int lmax, cplx *ac)
{
    tables_init();
    axialtrancoefinit(imax(nmax, lmax));
    axialtrancoefrecurrence(itype, r, rire + CI * riim, nmax, lmax, ac);
}
void orc_x_mieoa(double x, double rire, double riim, double qeps, int *nodr, double *qext, double *qsca,
                 double *qabs, cplx *anp, cplx *anpinv)
{
    tables_init();
    mieoa(x, rire + CI * riim, 1.0, nodr, qeps, qext, qsca, qabs, anp, anpinv);
}
/* One translation by the rotation path and by the dense matrix, for the
 * equivalence test: source order ns, target order nt, vector rvec (t - s). */
void orc_x_translate_rot(int ns, int nt, const double *rvec, int vtype, const cplx *a, cplx *g, int sop, int top)
{
    tables_init();
    axialtrancoefinit(imax(ns, nt));
    pairop_t op;
    if (!sop) { pairop_compute(&op, nt, ns, rvec, vtype, 1.0); coefficient_translation(ns, nt, a, g, &op, 0, top); }
    else {
        double rneg[3] = {-rvec[0], -rvec[1], -rvec[2]};
        pairop_compute(&op, ns, nt, rneg, vtype, 1.0);
        coefficient_translation(ns, nt, a, g, &op, 1, top);
    }
    pairop_free(&op);
}
void orc_x_gentranmatrix(int ns, int nt, const double *rvec, int vtype, cplx *ac)
{
    tables_init();
    gentranmatrix(ns, nt, rvec, 1.0, vtype, ac);
}
void orc_x_cspherebessel(int n, double zr, double zi, cplx *csj, cplx *csy) { cspherebessel(n, zr + CI * zi, csj, csy); }
void orc_x_crichankel(int n, double zr, double zi, cplx *xi) { crichankel(n, zr + CI * zi, xi); }
void orc_x_direct_solve(orc_ctx *c, const cplx *pnp, cplx *anp) { direct_solve(c, pnp, anp); }
void orc_x_multmie(orc_ctx *c, int idir, const cplx *ain, cplx *aout) { multmiecoeffmult(c, idir, ain, aout, c->an); }
void orc_x_qeff(orc_ctx *c, const cplx *amnp, const cplx *pmnp0, double *qeff) { qefficiencyfactors(c, amnp, pmnp0, qeff); }

/* ======================================================================== */
/* Post-processing: common-origin expansion, GSF expansion, scattering matrix */
/* ======================================================================== */
static cplx ipow(int k) /* i**k for any integer k */
{
    int e = ((k % 4) + 4) % 4;
    return (e == 0) ? 1.0 : (e == 1 ? CI : (e == 2 ? -1.0 : -CI));
}

/* tranordertest (modules:1896-1942): order needed to translate a sphere of
 * order lmax over distance r with regular functions to accuracy eps. */
int orc_tranordertest(double r, double ri_re, int lmax, double eps)
{
    tables_init();
    const int nlim = 200;
    if (r == 0.0) return lmax;
    cplx z = r * ri_re;
    double sum = 0.0;
    cplx *xi = (cplx *)malloc(sizeof(cplx) * (nlim + lmax + 2));
    double *vc1 = (double *)malloc(sizeof(double) * (nlim + lmax + 2));
    int n;
    for (n = 1; n <= nlim; n++) {
        cricbessel(n + lmax, z, xi);
        for (int l = 0; l <= n + lmax; l++) xi[l] = xi[l] / z * ipow(l);
        int n21 = n + n + 1, l = lmax;
        cplx c = FNR(n21) * FNR(l + l + 1) * ipow(n - l);
        vcfunc(-1, n, 1, l, vc1);
        int wmin = iabs_(n - l), wmax = n + l;
        cplx a = 0, b = 0;
        for (int w = wmin; w <= wmax; w++) {
            double alnw = vc1[w] * vc1[w];
            if ((n + l + w) % 2 == 0) a = a + alnw * xi[w];
            else b = b + alnw * xi[w];
        }
        a = c * a;
        b = c * b;
        sum = creal(sum + a * conj(a) + b * conj(b));
        if (fabs(1.0 - sum) < eps) break;
    }
    free(xi); free(vc1);
    int nmax = n < nlim ? n : nlim;
    return nmax > lmax ? nmax : lmax;
}

/* cluster origin, translation orders and t_matrix_order as main_calling_program
 * sets them (input:1159-1197): origin = mean external position, orders from
 * tranordertest with translation_epsilon, capped at max_t_matrix_order. */
int orc_t_matrix_order(const orc_ctx *c, double trans_eps, int maxt, double *origin, int *trans_order)
{
    /* the cluster origin and the translation orders over the spheres outside
     * every other (input:1166-1197); a held sphere keeps its own order */
    double r0[3] = {0, 0, 0};
    int nout = 0;
    for (int i = 0; i < c->n; i++) {
        if (c->host[i] >= 0) continue;
        nout++;
        for (int k = 0; k < 3; k++) r0[k] = r0[k] + c->pos[3 * i + k];
    }
    for (int k = 0; k < 3; k++) r0[k] = r0[k] / (double)nout;
    int tmo = imin(c->max_order, maxt);
    for (int i = 0; i < c->n; i++) {
        if (c->host[i] >= 0) { trans_order[i] = c->order[i]; continue; }
        double d2 = 0.0;
        for (int k = 0; k < 3; k++) d2 += (c->pos[3 * i + k] - r0[k]) * (c->pos[3 * i + k] - r0[k]);
        int to = orc_tranordertest(sqrt(d2), creal(c->rimed), c->order[i], trans_eps);
        to = imin(to, maxt);
        trans_order[i] = to;
        tmo = imax(tmo, to);
    }
    for (int k = 0; k < 3; k++) origin[k] = r0[k];
    return tmo;
}

/* merge_to_common_origin (scatprops:447-559), one right-hand side: regular (J)
 * translation of each sphere's expansion to r0, converted LR -> TE/TM.
 * amnp0 is the nodrt block a(0:nodrt+1,1:nodrt,1:2). */
void orc_merge_to_common_origin(const orc_ctx *c, int nodrt, const cplx *amnp, const double *r0, const int *trans_order,
                                cplx *amnp0)
{
    int nb0 = 2 * nodrt * (nodrt + 2);
    for (int k = 0; k < nb0; k++) amnp0[k] = 0;
    axialtrancoefinit(imax(nodrt, c->max_order));
    for (int i = 0; i < c->n; i++) {
        if (c->host[i] >= 0) continue;   /* origin_host 0: the spheres outside every other (scatprops:631) */
        int noi = c->order[i];
        int ntrani = imin(nodrt, trans_order[i]);
        int nbt = 2 * ntrani * (ntrani + 2);
        cplx *amnpt = (cplx *)calloc(nbt, sizeof(cplx));
        double rv[3] = {r0[0] - c->pos[3 * i], r0[1] - c->pos[3 * i + 1], r0[2] - c->pos[3 * i + 2]};
        pairop_t op;
        pairop_compute(&op, ntrani, noi, rv, 1, c->rimed);
        coefficient_translation(noi, ntrani, amnp + c->offset[i], amnpt, &op, 0, 0);
        pairop_free(&op);
        for (int n = 1; n <= ntrani; n++)
            for (int m = 0; m <= ntrani + 1; m++) {
                cplx t1 = amnpt[m + (ntrani + 2) * (n - 1)];
                cplx t2 = amnpt[m + (ntrani + 2) * (n - 1) + (ntrani + 2) * ntrani];
                amnp0[m + (nodrt + 2) * (n - 1)] = amnp0[m + (nodrt + 2) * (n - 1)] + t1 + t2;
                amnp0[m + (nodrt + 2) * (n - 1) + (nodrt + 2) * nodrt] = amnp0[m + (nodrt + 2) * (n - 1) + (nodrt + 2) * nodrt] + t1 - t2;
            }
        free(amnpt);
    }
}

/* distribute_from_common_origin (scatprops:561-669), one right-hand side,
 * regular (J, vswf_type=1) functions: amnp (neqns) = translation of the
 * nodrt common-origin block amnp0 (LR basis) from r0 to every sphere. */
void orc_distribute_from_common_origin(const orc_ctx *c, int nodrt, const cplx *amnp0, const double *r0, cplx *amnp)
{
    for (int k = 0; k < c->neqns; k++) amnp[k] = 0;
    axialtrancoefinit(imax(nodrt, c->max_order));
    for (int i = 0; i < c->n; i++) {
        if (c->host[i] >= 0) continue;   /* origin_host 0: the spheres outside every other (scatprops:631) */
        int noi = c->order[i];
        double rv[3] = {c->pos[3 * i] - r0[0], c->pos[3 * i + 1] - r0[1], c->pos[3 * i + 2] - r0[2]};
        pairop_t op;
        pairop_compute(&op, noi, nodrt, rv, 1, c->rimed);
        coefficient_translation(nodrt, noi, amnp0, amnp + c->offset[i], &op, 0, 0);
        pairop_free(&op);
    }
}

/* tmatrix_solution (solver:22-332) on one process with the iterative solver:
 * for l = 1..tmo and the 2(2l+1) columns (k, q) of order l, the unit
 * common-origin field of degree k, order l and TE (q=1) / TM (q=2) mode is
 * distributed to the spheres, multiplied by the Mie coefficients, solved by
 * cbicg (initial guess = right-hand side), merged back to the origin, and
 * stored as T-matrix column 2(l(l+1)+k-1)+q-1 (rows 2(n(n+1)+m-1)+p-1, n <= l;
 * tmat is nblkt x nblkt column-major, nblkt = 2 tmo (tmo+2)).  The per-sphere
 * efficiencies of every column (qefficiencyfactors with npol=1) are summed in
 * sphere_qeff(3,N); the order loop stops after the order at which the
 * summed extinction changes by less than conveps (qeff(1) - qeffold(1), signed).
 * With host spheres the excitation reaches the spheres outside every other
 * only, and the sum runs over every sphere (exlist all true, solver:266-271).
 * Returns istat; *order_used = the T-matrix order kept (t_matrix_order). */
int orc_tmatrix_solution(orc_ctx *c, int tmo, const int *trans_order, const double *r0, double solneps, double conveps,
                         int niter, cplx *tmat, double *sphere_qeff, int *order_used, int *maxiter_o, double *maxerr_o)
{
    int neq = c->neqns, nblkt = 2 * tmo * (tmo + 2), istat = 0, initialize = 1, maxiter = 0;
    double maxerr = 0.0, qeffold = 0.0, xv = orc_vol_radius(c);
    for (size_t k = 0; k < (size_t)nblkt * nblkt; k++) tmat[k] = 0;
    for (int k = 0; k < 3 * c->n; k++) sphere_qeff[k] = 0.0;
    cplx *pmnpkq = (cplx *)malloc(sizeof(cplx) * neq), *pmnpan = (cplx *)malloc(sizeof(cplx) * neq);
    cplx *amnpkq = (cplx *)malloc(sizeof(cplx) * neq), *gmnp = (cplx *)malloc(sizeof(cplx) * neq);
    int l;
    for (l = 1; l <= tmo; l++) {
        int nb = 2 * l * (l + 2);
        cplx *pmnp0 = (cplx *)malloc(sizeof(cplx) * nb), *amnp0 = (cplx *)malloc(sizeof(cplx) * nb);
        for (int kq = 1; kq <= 2 * (2 * l + 1); kq++) {
            int k = -l + (kq - 1) / 2, q = (kq - 1) % 2 + 1;
            for (int e = 0; e < nb; e++) pmnp0[e] = 0;
            /* the T matrix is TE-TM based: unit TE / TM field in the LR basis */
            pmnp0[AIDX(k < 0 ? l + 1 : k, k < 0 ? -k : l, 0, l)] = 0.5;
            pmnp0[AIDX(k < 0 ? l + 1 : k, k < 0 ? -k : l, 1, l)] = -0.5 * pm1(q);
            orc_distribute_from_common_origin(c, l, pmnp0, r0, pmnpkq);
            multmiecoeffmult(c, 1, pmnpkq, pmnpan, c->an);
            memcpy(amnpkq, pmnpan, sizeof(cplx) * neq);
            if (niter != 0) {
                int iter = 0;
                double serr = 0.0;
                orc_cbicg(c, niter, solneps, pmnpan, amnpkq, initialize, &iter, &serr);
                maxiter = imax(iter, maxiter);
                maxerr = serr > maxerr ? serr : maxerr;
                if (iter > niter || serr > solneps) istat = 1;
            }
            initialize = 0;
            /* qefficiencyfactors(npol=1): the first-polarisation terms of
             * lrsphereqeff; with host spheres the exciting field is the
             * interaction without the Mie multiply plus the incident field */
            if (c->nhosted == 0) {
                for (int i = 0; i < c->n; i++)
                    mie_mult_sphere(c->an_inv + c->mie_offset[i], c->order[i], 1, amnpkq + c->offset[i], gmnp + c->offset[i]);
            } else {
                int zero = 0;
                sphereinteraction_ex(c, 1, amnpkq, gmnp, &zero, &zero, 0, 0);
                for (int e = 0; e < neq; e++) gmnp[e] += pmnpkq[e];
            }
            for (int i = 0; i < c->n; i++) {
                double qe[3], qs[3], qa[3];
                int off = c->offset[i];
                lrsphereqeff(c->rext[i], c->order[i], c->rad[i], amnpkq + off, 0, pmnpkq + off, gmnp + off, qe, qs, qa);
                sphere_qeff[3 * i] += qe[0];
                sphere_qeff[3 * i + 1] += qa[0];
                sphere_qeff[3 * i + 2] += qs[0];
            }
            orc_merge_to_common_origin(c, l, amnpkq, r0, trans_order, amnp0);
            int col = 2 * (l * (l + 1) + k - 1) + q - 1;
            for (int n = 1; n <= l; n++)
                for (int m = -n; m <= n; m++)
                    for (int p = 0; p < 2; p++)
                        tmat[(size_t)(2 * (n * (n + 1) + m - 1) + p) + (size_t)nblkt * col] =
                            amnp0[AIDX(m < 0 ? n + 1 : m, m < 0 ? -m : n, p, l)];
        }
        free(pmnp0);
        free(amnp0);
        double qext = 0.0;
        for (int i = 0; i < c->n; i++) qext = qext + sphere_qeff[3 * i] * c->rad[i] * c->rad[i] / (xv * xv);
        double converr = qext - qeffold;
        qeffold = qext;
        if (conveps > 0.0 && converr < conveps) break;
    }
    *order_used = l < tmo ? l : tmo;
    *maxiter_o = maxiter;
    *maxerr_o = maxerr;
    free(pmnpkq); free(pmnpan); free(amnpkq); free(gmnp);
    return istat;
}

/* The T matrix as ranorientscatmatrix holds it after reading the file
 * (scatprops:2031-2075): complex(4) storage tc(2,nblk,2,nblk) with the
 * computed entries (rows of order n <= l in the column of order l) and the
 * rest from the symmetry tc(q,l(l+1)-k,p,n(n+1)-m) = (-1)^(m+k) tc(p,n(n+1)+m,q,l(l+1)+k)
 * for n < l.  tmat: nblkt x nblkt column-major as orc_tmatrix_solution
 * writes it; tc: the same layout in single precision. */
void orc_tmatrix_symmetrize(int tmo, const cplx *tmat, float _Complex *tc)
{
    int nblkt = 2 * tmo * (tmo + 2);
    for (size_t k = 0; k < (size_t)nblkt * nblkt; k++) tc[k] = 0;
#define TIX(p, mn, q, kl) ((size_t)(2 * ((mn) - 1) + (p) - 1) + (size_t)nblkt * (size_t)(2 * ((kl) - 1) + (q) - 1))
    for (int l = 1; l <= tmo; l++)
        for (int k = -l; k <= l; k++) {
            int kl = l * (l + 1) + k, klm = l * (l + 1) - k;
            for (int q = 1; q <= 2; q++)
                for (int n = 1; n <= l; n++)
                    for (int m = -n; m <= n; m++) {
                        int mn = n * (n + 1) + m, mnm = n * (n + 1) - m;
                        for (int p = 1; p <= 2; p++) {
                            cplx t = tmat[TIX(p, mn, q, kl)];
                            tc[TIX(p, mn, q, kl)] = (float)creal(t) + I * (float)cimag(t);
                        }
                        if (n < l) {
                            float ikm = (float)pm1(m + k);
                            for (int p = 1; p <= 2; p++) tc[TIX(q, klm, p, mnm)] = tc[TIX(p, mn, q, kl)] * ikm;
                        }
                    }
        }
#undef TIX
}

/* Orientation-averaged extinction and scattering efficiencies from the T
 * matrix (ranorientscatmatrix, scatprops:2103-2122), summed over the
 * single-precision symmetrised matrix; xv = cross_section_radius. */
void orc_tmatrix_qext_qsca(int tmo, const cplx *tmat, double xv, double *qext, double *qsca)
{
    int nblkt = 2 * tmo * (tmo + 2);
    float _Complex *tc = (float _Complex *)malloc(sizeof(float _Complex) * (size_t)nblkt * nblkt);
    orc_tmatrix_symmetrize(tmo, tmat, tc);
    double qe = 0.0, qs = 0.0;
    for (int col = 0; col < nblkt; col++) {
        for (int row = 0; row < nblkt; row++) {
            float a = cabsf(tc[(size_t)row + (size_t)nblkt * col]);
            qs = qs + (double)(a * a);
        }
        qe = qe - (double)crealf(tc[(size_t)col + (size_t)nblkt * col]);
    }
    free(tc);
    *qext = qe * 2.0 / (xv * xv);
    *qsca = qs * 2.0 / (xv * xv);
}

/* ranorientscatmatrix (scatprops:1963-2530), beam_width 0, one process:
 * GSF expansion coefficients sm(4,4,0:2nodr) and smcf (the coherent part)
 * of the orientation-averaged scattering matrix from the T matrix of order
 * nodr (tmat as orc_tmatrix_solution stores it; read into complex(4) and
 * symmetrised exactly as the reference's file reader does), divided by
 * 2 Re(medium index).  sm, smcf: 16 * (2 nodr + 1), Fortran (4,4,0:2nodr). */
void orc_ranorientscatmatrix(int nodr, const cplx *tmat, double rimed_re, double *sm, double *smcf)
{
    tables_init();
    const int nodr2 = 2 * nodr, nodrw = nodr2, nblk = nodr * (nodr + 2), nblkt = 2 * nblk;
    float _Complex *tc = (float _Complex *)malloc(sizeof(float _Complex) * (size_t)nblkt * nblkt);
    orc_tmatrix_symmetrize(nodr, tmat, tc);
#define TC(p, mn, q, kl) tc[(size_t)(2 * ((mn) - 1) + (p) - 1) + (size_t)nblkt * (size_t)(2 * ((kl) - 1) + (q) - 1)]
    /* the GB-modified T matrix (no beam: gbn = 1), stored back in single precision */
    for (int n = 1; n <= nodr; n++)
        for (int m = -n; m <= n; m++) {
            int mn = n * (n + 1) + m;
            for (int p = 1; p <= 2; p++)
                for (int l = 1; l <= nodr; l++) {
                    cplx pp11 = -0.5 * ipow(l + 1) * FNR(l + l + 1);
                    cplx pp21 = -pp11, pp12 = -pp11, pp22 = pp21;
                    for (int k = -l; k <= l; k++) {
                        int kl = l * (l + 1) + k;
                        cplx a = TC(p, mn, 1, kl);
                        cplx t1 = (cplx)TC(p, mn, 1, kl) * pp11 + (cplx)TC(p, mn, 2, kl) * pp12;
                        TC(p, mn, 1, kl) = (float)creal(t1) + I * (float)cimag(t1);
                        cplx t2 = a * pp21 + (cplx)TC(p, mn, 2, kl) * pp22;
                        TC(p, mn, 2, kl) = (float)creal(t2) + I * (float)cimag(t2);
                    }
                }
        }
    const int U = nodr + 1, ldu = 2 * U + 1;
    size_t dmsz = (size_t)ldu * 3 * nodr * 2 * nodr * 2;
    cplx *dm = (cplx *)calloc(dmsz, sizeof(cplx)), *dmcf = (cplx *)calloc(dmsz, sizeof(cplx));
#define DM(arr, u, ku, n, p, n1, p1) arr[((u) + U) + (size_t)ldu * ((ku) - 1 + 3 * (((n) - 1) + nodr * (((p) - 1) + 2 * (((n1) - 1) + nodr * ((p1) - 1)))))]
    cplx *bm = (cplx *)malloc(sizeof(cplx) * 2 * nblk * 2), *bmcf = (cplx *)malloc(sizeof(cplx) * 2 * nblk * 2);
    cplx *am = (cplx *)malloc(sizeof(cplx) * 2 * (nodr + 1) * 2), *amcf = (cplx *)malloc(sizeof(cplx) * 2 * (nodr + 1) * 2);
#define BM(arr, k, mn, p) arr[((k) - 1) + 2 * (((mn) - 1) + nblk * ((p) - 1))]
#define AM(arr, k, l, p) arr[((k) - 1) + 2 * (((l) - 1) + (nodr + 1) * ((p) - 1))]
    double *vc = (double *)malloc(sizeof(double) * (4 * nodr + 3));
    for (int w = 0; w <= nodr2; w++)
        for (int v = -w; v <= w; v++) {
            for (size_t e = 0; e < (size_t)2 * nblk * 2; e++) { bm[e] = 0; bmcf[e] = 0; }
            for (int n = 1; n <= nodr; n++) {
                int nn1 = n * (n + 1);
                for (int l = imax(1, iabs_(w - n)); l <= imin(nodr, w + n); l++)
                    for (int k = 1; k <= 2; k++)
                        for (int p = 1; p <= 2; p++) { AM(am, k, l, p) = 0; AM(amcf, k, l, p) = 0; }
                for (int t = -n; t <= n; t++) {
                    int tn = nn1 + t, lmax = imin(nodr, w + n);
                    vcfunc(v, w, -t, n, vc);
                    for (int l = imax(imax(1, iabs_(v - t)), iabs_(n - w)); l <= lmax; l++) {
                        int tvl = l * (l + 1) + t - v;
                        for (int k = 1; k <= 2; k++)
                            for (int p = 1; p <= 2; p++) {
                                AM(am, k, l, p) += vc[l] * (cplx)TC(p, tn, k, tvl);
                                if (l == n && v == 0) {
                                    cplx tct = 0;
                                    for (int kt = -n; kt <= n; kt++) tct += (cplx)TC(p, nn1 + kt, k, nn1 + kt);
                                    AM(amcf, k, l, p) += vc[l] * tct / (double)(n + n + 1);
                                }
                            }
                    }
                }
                for (int m = -n; m <= n; m++) {
                    int mn = nn1 + m;
                    for (int k = 1; k <= 2; k++) {
                        int u = m - (-3 + 2 * k);
                        if (iabs_(u) > w) continue;
                        int lmax = imin(nodr, w + n);
                        vcfunc(-u, w, m, n, vc);
                        for (int l = imax(1, iabs_(w - n)); l <= lmax; l++) {
                            double fl = -pm1(l) * vc[l] / (double)(l + l + 1);
                            for (int p = 1; p <= 2; p++) {
                                BM(bm, k, mn, p) += AM(am, k, l, p) * fl;
                                if (v == 0) BM(bmcf, k, mn, p) += AM(amcf, k, l, p) * fl;
                            }
                        }
                    }
                }
            }
            int umax = imin(w, nodr + 1);
            for (int u = -umax; u <= umax; u++)
                for (int ku = 1; ku <= 3; ku++) {
                    int k = (ku == 1) ? -1 : 1, k1 = (ku == 2) ? 1 : -1;
                    int m = u + k, m1 = u + k1, ns = imax(1, iabs_(m));
                    int ik = (k + 1) / 2 + 1, ik1 = (k1 + 1) / 2 + 1;
                    for (int n = ns; n <= nodr; n++) {
                        int nu = n * (n + 1) + m;
                        int n1s = imax(imax(1, iabs_(m1)), n - nodrw), n1e = imin(nodr, n + nodrw);
                        for (int n1 = n1s; n1 <= n1e; n1++) {
                            cplx cin = ipow(n - n1);
                            int nu1 = n1 * (n1 + 1) + m1;
                            double fl = -FNR(n + n + 1) * FNR(n1 + n1 + 1) * (double)(w + w + 1);
                            for (int p = 1; p <= 2; p++)
                                for (int p1 = 1; p1 <= 2; p1++) {
                                    DM(dm, u, ku, n, p, n1, p1) += BM(bm, ik, nu, p) * cin * fl * conj(BM(bm, ik1, nu1, p1));
                                    if (v == 0) DM(dmcf, u, ku, n, p, n1, p1) += BM(bmcf, ik, nu, p) * cin * fl * conj(BM(bmcf, ik1, nu1, p1));
                                }
                        }
                    }
                }
        }
    /* expansion coefficients */
    cplx *aw = (cplx *)calloc(3 * 3 * (nodrw + 1), sizeof(cplx)), *bw = (cplx *)calloc(3 * 3 * (nodrw + 1), sizeof(cplx));
    cplx *awcf = (cplx *)calloc(3 * 3 * (nodrw + 1), sizeof(cplx)), *bwcf = (cplx *)calloc(3 * 3 * (nodrw + 1), sizeof(cplx));
    cplx *cw = (cplx *)calloc(nodrw + 1, sizeof(cplx)), *dw = (cplx *)calloc(nodrw + 1, sizeof(cplx));
    cplx *cwcf = (cplx *)calloc(nodrw + 1, sizeof(cplx)), *dwcf = (cplx *)calloc(nodrw + 1, sizeof(cplx));
#define AW(arr, i, k, w) arr[(i) + 3 * (((k) + 1) + 3 * (w))]
    cplx *fm = (cplx *)malloc(sizeof(cplx) * 3 * nodr * 2 * nodr * 2), *fmcf = (cplx *)malloc(sizeof(cplx) * 3 * nodr * 2 * nodr * 2);
#define FM(arr, k, n, p, n1, p1) arr[((k) - 1) + 3 * (((n) - 1) + nodr * (((p) - 1) + 2 * (((n1) - 1) + nodr * ((p1) - 1))))]
    for (int w = 0; w <= nodrw; w++) {
        for (size_t e = 0; e < (size_t)3 * nodr * 2 * nodr * 2; e++) { fm[e] = 0; fmcf[e] = 0; }
        for (int u = -nodr - 1; u <= nodr + 1; u++) {
            for (int k = -1; k <= 1; k += 2) {
                int m = u + k, ik = (k + 1) / 2 + 1, ns = imax(1, iabs_(m));
                for (int n = ns; n <= nodr; n++) {
                    vcfunc(m, n, 0, w, vc);
                    for (int n1 = ns; n1 <= nodr; n1++) {
                        if (n + n1 < w || iabs_(n - n1) > w) continue;
                        double fl = -pm1(n) * vc[n1] * FNR(w + w + 1) / FNR(n1 + n1 + 1);
                        for (int p = 1; p <= 2; p++)
                            for (int p1 = 1; p1 <= 2; p1++) {
                                FM(fm, ik, n, p, n1, p1) += DM(dm, u, ik, n, p, n1, p1) * fl;
                                FM(fmcf, ik, n, p, n1, p1) += DM(dmcf, u, ik, n, p, n1, p1) * fl;
                            }
                    }
                }
            }
            if (w < 2) continue;
            int m = u + 1, m1 = u - 1, ns = imax(1, iabs_(m)), n1s = imax(1, iabs_(m1));
            for (int n = ns; n <= nodr; n++) {
                vcfunc(m, n, -2, w, vc);
                for (int n1 = n1s; n1 <= nodr; n1++) {
                    if (n + n1 < w || iabs_(n - n1) > w) continue;
                    double fl = -pm1(n) * vc[n1] * FNR(w + w + 1) / FNR(n1 + n1 + 1);
                    for (int p = 1; p <= 2; p++)
                        for (int p1 = 1; p1 <= 2; p1++) {
                            FM(fm, 3, n, p, n1, p1) += DM(dm, u, 3, n, p, n1, p1) * fl;
                            FM(fmcf, 3, n, p, n1, p1) += DM(dmcf, u, 3, n, p, n1, p1) * fl;
                        }
                }
            }
        }
        for (int n = 1; n <= nodr; n++) {
            int n1s = imax(1, iabs_(n - w)), n1e = imin(nodr, n + w);
            double in = pm1(n);
            vcfunc(1, n, 0, w, vc);
            for (int n1 = n1s; n1 <= n1e; n1++) {
                double fl = 2.0 * in * vc[n1] * FNR(w + w + 1) / FNR(n1 + n1 + 1);
                int i = (n + n1 - w) % 2 + 1;
                for (int p = 1; p <= 2; p++) {
                    int p1 = (2 - i) * p + (i - 1) * (3 - p);
                    for (int k = -1; k <= 1; k += 2) {
                        int ik = (k + 1) / 2 + 1;
                        AW(aw, 0, k, w) += FM(fm, ik, n, p, n1, p1) * fl;
                        AW(bw, 0, k, w) += FM(fm, ik, n, p, n1, 3 - p1) * fl;
                        AW(awcf, 0, k, w) += FM(fmcf, ik, n, p, n1, p1) * fl;
                        AW(bwcf, 0, k, w) += FM(fmcf, ik, n, p, n1, 3 - p1) * fl;
                    }
                    AW(bw, 2, 0, w) += FM(fm, 3, n, p, n1, 3 - p1) * fl;
                    AW(aw, 2, 0, w) += FM(fm, 3, n, p, n1, p1) * fl;
                    AW(bwcf, 2, 0, w) += FM(fmcf, 3, n, p, n1, 3 - p1) * fl;
                    AW(awcf, 2, 0, w) += FM(fmcf, 3, n, p, n1, p1) * fl;
                }
            }
            if (w < 2) continue;
            vcfunc(1, n, -2, w, vc);
            for (int n1 = n1s; n1 <= n1e; n1++) {
                double fl = 2.0 * in * vc[n1] * FNR(w + w + 1) / FNR(n1 + n1 + 1);
                int i = (n + n1 - w) % 2 + 1;
                for (int p = 1; p <= 2; p++) {
                    int p1 = (2 - i) * p + (i - 1) * (3 - p);
                    for (int k = -1; k <= 1; k += 2) {
                        int ik = (k + 1) / 2 + 1;
                        AW(aw, 2, k, w) += FM(fm, ik, n, p, n1, p1) * fl * pm1(p1);
                        AW(bw, 2, k, w) += FM(fm, ik, n, p, n1, 3 - p1) * fl * pm1(3 - p1);
                        AW(awcf, 2, k, w) += FM(fmcf, ik, n, p, n1, p1) * fl * pm1(p1);
                        AW(bwcf, 2, k, w) += FM(fmcf, ik, n, p, n1, 3 - p1) * fl * pm1(3 - p1);
                    }
                }
                double fl2 = 2.0 * pm1(n1 + w) * vc[n1] * FNR(w + w + 1) / FNR(n1 + n1 + 1);
                for (int p = 1; p <= 2; p++)
                    for (int p1 = 1; p1 <= 2; p1++) {
                        cw[w] += FM(fm, 3, n, p, n1, p1) * fl * pm1(p1);
                        dw[w] += FM(fm, 3, n, p, n1, p1) * fl2 * pm1(p);
                        cwcf[w] += FM(fmcf, 3, n, p, n1, p1) * fl * pm1(p1);
                        dwcf[w] += FM(fmcf, 3, n, p, n1, p1) * fl2 * pm1(p);
                    }
            }
        }
    }
#define SMX(arr, i, j, n) arr[((i) - 1) + 4 * ((j) - 1) + 16 * (n)]
    for (int k = 0; k < 16 * (nodrw + 1); k++) { sm[k] = 0.0; smcf[k] = 0.0; }
    for (int pass = 0; pass < 2; pass++) {
        double *o = pass ? smcf : sm;
        cplx *A = pass ? awcf : aw, *B = pass ? bwcf : bw, *Cc = pass ? cwcf : cw, *D = pass ? dwcf : dw;
        for (int n = 0; n <= nodrw; n++) {
            SMX(o, 1, 1, n) = creal(AW(A, 0, -1, n) + AW(A, 0, 1, n));
            SMX(o, 1, 2, n) = creal(AW(A, 2, -1, n) + AW(A, 2, 1, n));
            SMX(o, 1, 3, n) = 2.0 * cimag(AW(A, 2, 0, n));
            SMX(o, 1, 4, n) = creal(AW(A, 0, 1, n) - AW(A, 0, -1, n));
            SMX(o, 2, 2, n) = creal(D[n]);
            SMX(o, 2, 3, n) = cimag(D[n]);
            SMX(o, 2, 4, n) = creal(AW(A, 2, 1, n) - AW(A, 2, -1, n));
            SMX(o, 3, 1, n) = -cimag(AW(B, 2, -1, n) + AW(B, 2, 1, n));
            SMX(o, 3, 2, n) = cimag(Cc[n]);
            SMX(o, 3, 3, n) = creal(Cc[n]);
            SMX(o, 3, 4, n) = cimag(AW(B, 2, -1, n) - AW(B, 2, 1, n));
            SMX(o, 4, 1, n) = creal(AW(B, 0, -1, n) + AW(B, 0, 1, n));
            SMX(o, 4, 2, n) = 2.0 * creal(AW(B, 2, 0, n));
            SMX(o, 4, 4, n) = creal(AW(B, 0, 1, n) - AW(B, 0, -1, n));
        }
        for (int k = 0; k < 16 * (nodrw + 1); k++) o[k] = o[k] / rimed_re / 2.0;
    }
#undef TC
#undef DM
#undef BM
#undef AM
#undef AW
#undef FM
    free(tc); free(dm); free(dmcf); free(bm); free(bmcf); free(am); free(amcf); free(vc);
    free(aw); free(bw); free(awcf); free(bwcf); free(cw); free(dw); free(cwcf); free(dwcf); free(fm); free(fmcf);
}

/* ranorienscatmatrixcalc (scatprops:2538-2592): the 16 elements at cos(theta)
 * = ct from the expansion smc(4,4,0:nodrexp); the reference's assignment
 * sm(3,1) = sm(1,3) + ... is kept as written. */
void orc_ranorienscatmatrixcalc(double ct, const double *smc, int nodrexp, double *smo)
{
    tables_init();
    double *dc = (double *)malloc(sizeof(double) * 5 * (nodrexp * (nodrexp + 2) + 1));
    rotcoef(ct, 2, nodrexp, dc);
#define DCX(k, nm) dc[((k) + 2) + 5 * (nm)]
#define SC(i, j, n) smc[((i) - 1) + 4 * ((j) - 1) + 16 * (n)]
#define SO(i, j) smo[((i) - 1) + 4 * ((j) - 1)]
    for (int k = 0; k < 16; k++) smo[k] = 0.0;
    for (int n = 0; n <= nodrexp; n++) {
        int nn0 = n * (n + 1), nnp2 = nn0 + 2, nnm2 = nn0 - 2;
        SO(1, 1) = SO(1, 1) + DCX(0, nn0) * SC(1, 1, n);
        SO(1, 4) = SO(1, 4) + DCX(0, nn0) * SC(1, 4, n);
        SO(4, 1) = SO(4, 1) + DCX(0, nn0) * SC(4, 1, n);
        SO(4, 4) = SO(4, 4) + DCX(0, nn0) * SC(4, 4, n);
        if (n >= 2) {
            SO(1, 2) = SO(1, 2) + DCX(2, nn0) * SC(1, 2, n);
            SO(2, 4) = SO(2, 4) + DCX(2, nn0) * SC(2, 4, n);
            SO(3, 4) = SO(3, 4) + DCX(2, nn0) * SC(3, 4, n);
            SO(1, 3) = SO(1, 3) + DCX(2, nn0) * SC(1, 3, n);
            SO(3, 1) = SO(1, 3) + DCX(2, nn0) * SC(3, 1, n);
            SO(4, 2) = SO(4, 2) + DCX(2, nn0) * SC(4, 2, n);
            SO(2, 2) = SO(2, 2) + DCX(2, nnm2) * SC(2, 2, n) + DCX(2, nnp2) * SC(3, 3, n);
            SO(2, 3) = SO(2, 3) + DCX(2, nnp2) * SC(2, 3, n) + DCX(2, nnp2) * SC(3, 2, n);
            SO(3, 3) = SO(3, 3) - DCX(2, nnm2) * SC(2, 2, n) + DCX(2, nnp2) * SC(3, 3, n);
            SO(3, 2) = SO(3, 2) + DCX(2, nnp2) * SC(2, 3, n) - DCX(2, nnp2) * SC(3, 2, n);
        }
    }
    SO(2, 1) = SO(1, 2);
    SO(4, 3) = -SO(3, 4);
#undef DCX
#undef SC
#undef SO
    free(dc);
}

/* fosmexpansion (scatprops:1820-1951): GSF expansion coefficients of the
 * azimuth-averaged scattering matrix.  amnp0: (nb(ntot), 2 polarisations).
 * s00..sm22: 16*(2ntot+1) each, Fortran (4,4,0:2ntot) order. */
void orc_fosmexpansion(int ntot, const cplx *amnp0, double *s00, double *s02, double *sp22, double *sm22)
{
    tables_init();
    int nb = 2 * ntot * (ntot + 2);
    int W = 2 * ntot + 1;
    int ldm = 2 * ntot + 5;   /* m from -ntot-2..ntot+2 */
    cplx *a1 = (cplx *)calloc((size_t)ldm * ntot * 2, sizeof(cplx));
    cplx *a2 = (cplx *)calloc((size_t)ldm * ntot * 2, sizeof(cplx));
#define AA(arr, m, n, p) arr[((m) + ntot + 2) + ldm * (((n) - 1) + ntot * (p))]
    for (int n = 1; n <= ntot; n++)
        for (int p = 0; p < 2; p++)
            for (int m = -n; m <= n; m++) {
                int s = (m < 0) ? ((n + 1) + (ntot + 2) * (-m - 1)) : (m + (ntot + 2) * (n - 1));
                AA(a1, m, n, p) = amnp0[s + (ntot + 2) * ntot * p];
                AA(a2, m, n, p) = amnp0[nb + s + (ntot + 2) * ntot * p];
            }
    for (int k = 0; k < 16 * W; k++) { s00[k] = 0; s02[k] = 0; sp22[k] = 0; sm22[k] = 0; }
#define SS(arr, i, j, w) arr[((i) - 1) + 4 * ((j) - 1) + 16 * (w)]
    double *cm1p1 = (double *)malloc(sizeof(double) * (2 * ntot + 2));
    double *cm1m1 = (double *)malloc(sizeof(double) * (2 * ntot + 2));
    double *cmmpm = (double *)malloc(sizeof(double) * (2 * ntot + 2));
    double *cmmm2pm = (double *)malloc(sizeof(double) * (2 * ntot + 2));
    double *cmmp2pm = (double *)malloc(sizeof(double) * (2 * ntot + 2));
    for (int n = 1; n <= ntot; n++)
        for (int l = 1; l <= ntot; l++) {
            int wmin = iabs_(n - l), wmax = n + l;
            cplx fnl = sqrt((double)((n + n + 1) * (l + l + 1))) * ipow(l - n);
            vcfunc(-1, n, 1, l, cm1p1);
            vcfunc(-1, n, -1, l, cm1m1);
            int mm = imin(n, l + 2);
            for (int m = -mm; m <= mm; m++) {
                double m1m = pm1(m);
                if (iabs_(m) <= l) vcfunc(-m, n, m, l, cmmpm);
                else for (int w = 0; w <= n + l; w++) cmmpm[w] = 0.0;
                if (iabs_(-2 + m) <= l) vcfunc(-m, n, -2 + m, l, cmmm2pm);
                else for (int w = 0; w <= n + l; w++) cmmm2pm[w] = 0.0;
                if (iabs_(2 + m) <= l) vcfunc(-m, n, 2 + m, l, cmmp2pm);
                else for (int w = 0; w <= n + l; w++) cmmp2pm[w] = 0.0;
                for (int p = 1; p <= 2; p++)
                    for (int q = 1; q <= 2; q++) {
                        double m1mq = pm1(m + q);
                        double m1mnpl = pm1(m + n + p + l);
                        cplx a1122 = AA(a1, m, n, p - 1) * conj(AA(a1, m, l, q - 1)) + AA(a2, m, n, p - 1) * conj(AA(a2, m, l, q - 1));
                        cplx a2112 = AA(a2, m, n, p - 1) * conj(AA(a1, m, l, q - 1)) - AA(a1, m, n, p - 1) * conj(AA(a2, m, l, q - 1));
                        cplx a1p2 = (AA(a1, m, n, p - 1) + CI * AA(a2, m, n, p - 1)) * conj(AA(a1, m - 2, l, q - 1) - CI * AA(a2, m - 2, l, q - 1));
                        cplx a1m2 = (AA(a1, m, n, p - 1) - CI * AA(a2, m, n, p - 1)) * conj(AA(a1, m + 2, l, q - 1) + CI * AA(a2, m + 2, l, q - 1));
                        for (int w = wmin; w <= wmax; w++) {
                            double m1w = pm1(w);
                            int ev = ((n + l + w + p + q) % 2 == 0);
                            if (ev) SS(s00, 1, 1, w) = SS(s00, 1, 1, w) - creal(m1m * fnl * a1122 * cm1p1[w] * cmmpm[w]) / 2.0;
                            else SS(s00, 4, 4, w) = SS(s00, 4, 4, w) + creal(CI / 2.0 * m1m * fnl * a2112 * cm1p1[w] * cmmpm[w]);
                            if (w < 2) continue;
                            if (ev) {
                                SS(s02, 2, 1, w) = SS(s02, 2, 1, w) - creal(m1mq * a1122 * fnl * cm1m1[w] * cmmpm[w]) / 2.0;
                                SS(s02, 1, 2, w) = SS(s02, 1, 2, w) - creal(m1m * a1p2 * fnl * cm1p1[w] * cmmm2pm[w]) / 4.0;
                                SS(s02, 1, 2, w) = SS(s02, 1, 2, w) - creal(m1m * a1m2 * fnl * cm1p1[w] * cmmp2pm[w]) / 4.0;
                            } else {
                                SS(s02, 3, 4, w) = SS(s02, 3, 4, w) + cimag(-CI / 2.0 * m1mq * a2112 * fnl * cm1m1[w] * cmmpm[w]);
                                SS(s02, 4, 3, w) = SS(s02, 4, 3, w) + cimag(m1m * a1p2 * fnl * cm1p1[w] * cmmm2pm[w]) / 4.0;
                                SS(s02, 4, 3, w) = SS(s02, 4, 3, w) - cimag(m1m * a1m2 * fnl * cm1p1[w] * cmmp2pm[w]) / 4.0;
                            }
                            SS(sm22, 2, 2, w) = SS(sm22, 2, 2, w) - creal(m1mnpl * m1w * a1p2 * fnl * cm1m1[w] * cmmm2pm[w]) / 8.0;
                            SS(sp22, 2, 2, w) = SS(sp22, 2, 2, w) - creal(m1mq * a1p2 * fnl * cm1m1[w] * cmmm2pm[w]) / 8.0;
                            SS(sm22, 2, 2, w) = SS(sm22, 2, 2, w) - creal(m1mq * a1m2 * fnl * cm1m1[w] * cmmp2pm[w]) / 8.0;
                            SS(sp22, 2, 2, w) = SS(sp22, 2, 2, w) - creal(m1mnpl * m1w * a1m2 * fnl * cm1m1[w] * cmmp2pm[w]) / 8.0;
                        }
                    }
            }
        }
    for (int i = 3; i <= 4; i++)
        for (int j = 1; j <= i; j++)
            for (int w = 0; w < W; w++) {
                SS(s00, j, i, w) = -SS(s00, j, i, w);
                SS(s02, j, i, w) = -SS(s02, j, i, w);
                SS(sm22, j, i, w) = -SS(sm22, j, i, w);
                SS(sp22, j, i, w) = -SS(sp22, j, i, w);
            }
    for (int w = 0; w < W; w++) {
        SS(sm22, 3, 3, w) = -SS(sm22, 2, 2, w);
        SS(sp22, 3, 3, w) = SS(sp22, 2, 2, w);
    }
    for (int k = 0; k < 16 * W; k++) {
        s00[k] = 0.5 * s00[k] / 1.0;
        s02[k] = 0.5 * s02[k] / 1.0;
        sm22[k] = 0.5 * sm22[k] / 1.0;
        sp22[k] = 0.5 * sp22[k] / 1.0;
    }
#undef AA
#undef SS
    free(a1); free(a2); free(cm1p1); free(cm1m1); free(cmmpm); free(cmmm2pm); free(cmmp2pm);
}

/* fosmcalc (scatprops:1750-1810), normalize_s11 = .false.: sm(4,4) Fortran order. */
void orc_fosmcalc(int ntot, const double *s00, const double *s02, const double *sp22, const double *sm22, double ct, double *sm)
{
    tables_init();
    int kmax = 2, nmax = 2 * ntot;
    double *dc = (double *)malloc(sizeof(double) * 5 * (nmax * (nmax + 2) + 1));
    rotcoef(ct, kmax, nmax, dc);
#define DC(m, nk) dc[((m) + 2) + 5 * (nk)]
    for (int k = 0; k < 16; k++) sm[k] = 0.0;
    for (int w = 0; w <= 2 * ntot; w++) {
        int ww1 = w * (w + 1);
        for (int k = 0; k < 16; k++) {
            double v = s00[k + 16 * w] * DC(0, ww1);
            v = v + s02[k + 16 * w] * DC(0, ww1 + 2) + sp22[k + 16 * w] * DC(2, ww1 + 2) + sm22[k + 16 * w] * DC(-2, ww1 + 2);
            sm[k] = sm[k] + v;
        }
    }
#undef DC
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
    free(dc);
}

/* ------------------------------------------------------------------------ */
/* Scattering matrix at one direction from the common-origin expansion,     */
/* not azimuth-averaged: scatteringmatrix (scatprops:1498-1573) with        */
/* normalize_s11 = .false., its tau functions (taufunc, modules:1324-1344)  */
/* and amplitude_to_scattering_matrix (scatprops:1410-1436).                */
/* amn0: 2*nodrt*(nodrt+2) x 2 (TE/TM, index model 2, two polarizations).   */
/* ------------------------------------------------------------------------ */
static void amplitude_to_sm(const cplx *sa, double *sm)
{
    cplx sp[4][4];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) sp[i][j] = sa[i] * conj(sa[j]);
#define SP(i, j) sp[(i) - 1][(j) - 1]
#define SM(i, j) sm[((i) - 1) + 4 * ((j) - 1)]
    SM(1, 1) = creal(SP(1, 1) + SP(2, 2) + SP(3, 3) + SP(4, 4));
    SM(1, 2) = creal(-SP(1, 1) + SP(2, 2) - SP(3, 3) + SP(4, 4));
    SM(2, 1) = creal(-SP(1, 1) + SP(2, 2) + SP(3, 3) - SP(4, 4));
    SM(2, 2) = creal(SP(1, 1) + SP(2, 2) - SP(3, 3) - SP(4, 4));
    SM(3, 3) = 2.0 * creal(SP(1, 2) + SP(3, 4));
    SM(3, 4) = 2.0 * cimag(SP(2, 1) + SP(4, 3));
    SM(4, 3) = 2.0 * cimag(SP(1, 2) - SP(3, 4));
    SM(4, 4) = 2.0 * creal(SP(1, 2) - SP(3, 4));
    SM(1, 3) = 2.0 * creal(SP(2, 3) + SP(1, 4));
    SM(3, 1) = 2.0 * creal(SP(2, 4) + SP(1, 3));
    SM(1, 4) = -2.0 * cimag(SP(2, 3) - SP(1, 4));
    SM(4, 1) = -2.0 * cimag(SP(4, 2) + SP(1, 3));
    SM(2, 3) = -2.0 * creal(SP(2, 3) - SP(1, 4));
    SM(3, 2) = -2.0 * creal(SP(2, 4) - SP(1, 3));
    SM(2, 4) = -2.0 * cimag(SP(2, 3) + SP(1, 4));
    SM(4, 2) = -2.0 * cimag(SP(4, 2) - SP(1, 3));
#undef SP
#undef SM
}

void orc_scatteringmatrix(int nodrt, const cplx *amn0, double ct, double phi, int rotate, double rimed_re, cplx *sa, double *sm)
{
    tables_init();
    const int nb = nodrt * (nodrt + 2);
    const int ld = 2 * nb;
    double *dc = (double *)malloc(sizeof(double) * 3 * (nb + 1));
    rotcoef(ct, 1, nodrt, dc);
#define DC(k, mn) dc[((k) + 1) + 3 * (mn)]
    double cphi = cos(phi), sphi = sin(phi);
    cplx *ephim = (cplx *)malloc(sizeof(cplx) * (2 * nodrt + 1));
    ephicoef(cphi + CI * sphi, nodrt, ephim);
    for (int k = 0; k < 4; k++) sa[k] = 0.0;
    cplx cin = 1.0;
    for (int n = 1; n <= nodrt; n++) {
        cin = cin * (-CI);
        double fnm = sqrt((double)(n + n + 1) / 2.0) / 4.0;
        for (int m = -n; m <= n; m++) {
            int mn = n * (n + 1) + m;
            double tau[2] = {-fnm * (-DC(-1, mn) + DC(1, mn)), -fnm * (DC(-1, mn) + DC(1, mn))};
            int m1 = (m <= -1) ? n + 1 : m, n1 = (m <= -1) ? -m : n;
            cplx e = ephim[m + nodrt];
            for (int p = 1; p <= 2; p++) {
                int ia = AIDX(m1, n1, p - 1, nodrt);
                cplx a1 = amn0[ia], a2 = amn0[ia + ld], a, b;
                if (rotate) {
                    a = a1 * cphi + a2 * sphi;
                    b = a1 * sphi - a2 * cphi;
                } else {
                    a = a1;
                    b = -a2;
                }
                sa[0] += cin * tau[2 - p] * b * e;
                sa[1] += CI * cin * tau[p - 1] * a * e;
                sa[2] += CI * cin * tau[p - 1] * b * e;
                sa[3] += cin * tau[2 - p] * a * e;
            }
        }
    }
#undef DC
    double qsca = 1.0 / ORC_REF_PI;
    for (int k = 0; k < 4; k++) sa[k] = sa[k] * 4.0 / sqrt(2.0 * qsca);
    amplitude_to_sm(sa, sm);
    for (int k = 0; k < 16; k++) sm[k] = sm[k] / (4.0 * ORC_REF_PI) / rimed_re;
    free(dc);
    free(ephim);
}

/* The angle loop of scattering_matrix_calculation (input:3038-3061) for a
 * single-origin expansion without azimuthal averaging: i = ldim..udim,
 * theta_i = amin + (amax - amin)(i - ldim)/(udim - ldim) degrees, cos theta
 * kept off +-1, azimuth alpha + pi for i < 0 and alpha otherwise.
 * sm: 16 x (udim - ldim + 1). */
void orc_incident_plane_scattering(int nodrt, const cplx *amn0, int ldim, int udim, double amin, double amax, double alpha,
                                   int rotate, double rimed_re, double *sm)
{
    cplx sa[4];
    for (int i = ldim; i <= udim; i++) {
        double ct = cos(ORC_REF_PI / 180.0 * (amin + (amax - amin) * (double)(i - ldim) / (double)(udim - ldim)));
        if (ct == 1.0) ct = 0.9999999;
        if (ct == -1.0) ct = -0.9999999;
        double phi = (i < 0) ? alpha + ORC_REF_PI : alpha;
        orc_scatteringmatrix(nodrt, amn0, ct, phi, rotate, rimed_re, sa, sm + 16 * (size_t)(i - ldim));
    }
}
