// special.cuh -- FP64 special functions used on the device for coefficient
// generation: Riccati-Bessel/Hankel functions of complex argument (Jin's
// backward recurrence), vector-coupling-free Mie coefficients, Wigner-d.
//
// Each routine restates the MSTM Fortran routine it cites; the arithmetic is
// FP64 throughout, with CUDA's own sin/cos/exp/log10.
#pragma once
#include "common.cuh"

// envj (december2023/mstm-modules-33.f90:936-942).  The reference overwrites
// its integer argument with max(1,|n|); callers rely on that, so it is kept.
__host__ __device__ inline double mstm_envj(int* n, double x)
{
    int v = *n < 0 ? -*n : *n;
    if (v < 1) v = 1;
    *n = v;
    return 0.5 * log10(6.28 * v) - v * log10(1.36 * x / v);
}

// msta1 (modules:873-893)
__host__ __device__ inline int mstm_msta1(double x, int mp)
{
    double a0 = fabs(x);
    int n0 = (int)(1.1 * a0) + 1;
    double f0 = mstm_envj(&n0, a0) - mp;
    int n1 = n0 + 5;
    double f1 = mstm_envj(&n1, a0) - mp;
    int nn = n1;
    for (int it = 1; it <= 20; it++) {
        nn = (int)(n1 - (n1 - n0) / (1.0 - f0 / f1));
        double f = mstm_envj(&nn, a0) - mp;
        int d = nn - n1;
        if ((d < 0 ? -d : d) < 1) break;
        n0 = n1; f0 = f1; n1 = nn; f1 = f;
    }
    return nn;
}

// msta2 (modules:907-934)
__host__ __device__ inline int mstm_msta2(double x, int n, int mp)
{
    double a0 = fabs(x);
    double hmp = 0.5 * (double)mp;
    int nt = n;
    double ejn = mstm_envj(&nt, a0);
    double obj;
    int n0;
    if (ejn <= hmp) { obj = mp; n0 = (int)(1.1 * a0); }
    else { obj = hmp + ejn; n0 = n; }
    double f0 = mstm_envj(&n0, a0) - obj;
    int n1 = n0 + 5;
    double f1 = mstm_envj(&n1, a0) - obj;
    int nn = n1;
    for (int it = 1; it <= 20; it++) {
        nn = (int)(n1 - (n1 - n0) / (1.0 - f0 / f1));
        double f = mstm_envj(&nn, a0) - obj;
        int d = nn - n1;
        if ((d < 0 ? -d : d) < 1) break;
        n0 = n1; f0 = f1; n1 = nn; f1 = f;
    }
    return nn + 10;
}

// cspherebessel: spherical Bessel j_n(z), y_n(z), complex z, n <= nmaxarr
// (modules:322-371; algorithm of J.-M. Jin as vendored there).
__host__ __device__ inline void mstm_cspherebessel(int n, zd z, zd* csj, zd* csy)
{
    double a0 = cabsd(z);
    int nm = n;
    if (a0 < 1.0e-60) {
        for (int k = 0; k <= n; k++) { csj[k] = mk(0.0, 0.0); csy[k] = mk(-1.0e300, 0.0); }
        csy[0] = mk(1.0, 0.0);
        return;
    }
    for (int k = 0; k <= n; k++) csj[k] = mk(0.0, 0.0);
    csj[0] = cdiv(csind(z), z);
    if (n >= 1) csj[1] = cdiv(csj[0] - ccosd(z), z);
    if (n >= 2) {
        zd csa = csj[0], csb = csj[1], cs = mk(0.0, 0.0), cf0, cf1, cf = mk(0.0, 0.0);
        int m = mstm_msta1(a0, 200);
        if (m < n) nm = m;
        else m = mstm_msta2(a0, n, 15);
        cf0 = mk(0.0, 0.0);
        cf1 = mk(1.0 - 100, 0.0);   // the reference writes 1.0d0-100
        for (int k = m; k >= 0; k--) {
            cf = cdiv((2.0 * k + 3.0) * cf1, z) - cf0;
            if (k <= nm) csj[k] = cf;
            cf0 = cf1;
            cf1 = cf;
        }
        if (cabsd(csa) > cabsd(csb)) cs = cdiv(csa, cf);
        if (cabsd(csa) <= cabsd(csb)) cs = cdiv(csb, cf0);
        int kk = nm < n ? nm : n;
        for (int k = 0; k <= kk; k++) csj[k] = cs * csj[k];
    }
    for (int k = 0; k <= n; k++) csy[k] = mk(1.0e200, 0.0);
    csy[0] = -cdiv(ccosd(z), z);
    if (n >= 1) csy[1] = cdiv(csy[0] - csind(z), z);
    int kk = nm < n ? nm : n;
    zd z2 = z * z, z3 = z * z * z;
    for (int k = 2; k <= kk; k++) {
        if (cabsd(csj[k - 1]) > cabsd(csj[k - 2]))
            csy[k] = cdiv(csj[k] * csy[k - 1] - cdivr(1.0, z2), csj[k - 1]);
        else
            csy[k] = cdiv(csj[k] * csy[k - 2] - cdivr(2.0 * k - 1.0, z3), csj[k - 2]);
    }
}

// cricbessel (modules:262-271): psi_n(z) = z j_n(z); scratch holds n+1 values.
__host__ __device__ inline void mstm_cricbessel(int n, zd ds, zd* psi, zd* scratch)
{
    mstm_cspherebessel(n, ds, psi, scratch);
    for (int i = 0; i <= n; i++) psi[i] = psi[i] * ds;
}

// crichankel (modules:281-300); scratch holds 2(n+1) values.
__host__ __device__ inline void mstm_crichankel(int n, zd ds, zd* xi, zd* scratch)
{
    zd ci = mk(0.0, 1.0);
    xi[0] = -(ci * cexpd(ci * ds));
    zd psi0 = csind(ds);
    if (cabsd(xi[0]) / cabsd(psi0) < 1.0e-6) {
        if (n >= 1) xi[1] = cdiv(-(cexpd(ci * ds) * (ci + ds)), ds);
        for (int i = 2; i <= n; i++) xi[i] = cdiv(mk((double)(i + i + 1), 0.0), ds) * xi[i - 1] - xi[i - 2];
    } else {
        zd* psi = scratch;
        zd* chi = scratch + (n + 1);
        mstm_cspherebessel(n, ds, psi, chi);
        for (int i = 1; i <= n; i++) xi[i] = (psi[i] + ci * chi[i]) * ds;
    }
}

// 2x2 complex matrices stored column-major: m[(s-1)+2(t-1)]
__host__ __device__ inline void mstm_inv22(const zd* mat, zd* imat)
{
    zd det = mat[0] * mat[3] - mat[1] * mat[2];
    zd t[4] = {mat[0], mat[1], mat[2], mat[3]};
    // imat(s,t) = (-1)^s (-1)^t mat(3-t,3-s) / det
    imat[0] = cdiv(t[3], det);          // (1,1) <- (2,2)
    imat[1] = -cdiv(t[1], det);         // (2,1) <- (2,1) with sign -
    imat[2] = -cdiv(t[2], det);         // (1,2) <- (1,2) with sign -
    imat[3] = cdiv(t[0], det);          // (2,2) <- (1,1)
}
