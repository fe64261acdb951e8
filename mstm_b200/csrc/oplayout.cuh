// oplayout.cuh -- offsets inside one pair operator record (see opgen.cu for
// the layout).  Shared by the generator and the translation kernel.
#pragma once

__host__ __device__ constexpr int op_rot_size(int nmax, int nmin)
{
    int s = 0;
    for (int n = 1; n <= nmax; n++) {
        int kk = n < nmin ? n : nmin;
        s += (kk + 1) * (n + 1) + kk * n;
    }
    return s;
}
__host__ __device__ constexpr int op_rot_offset(int n, int nmin)   // offset of E_n from the start of the rot section
{
    int s = 0;
    for (int q = 1; q < n; q++) {
        int kk = q < nmin ? q : nmin;
        s += (kk + 1) * (q + 1) + kk * q;
    }
    return s;
}
__host__ __device__ constexpr int op_z_offset(int m, int nt, int ns)  // complex offset of block Z_m (mode 0)
{
    int s = 0;
    for (int q = 0; q < m; q++) {
        int m1 = q < 1 ? 1 : q;
        s += (q == 0 ? 1 : 2) * (nt - m1 + 1) * (ns - m1 + 1);
    }
    return s;
}
__host__ __device__ constexpr int op_record_units(int nt, int ns)
{
    int nmin = nt < ns ? nt : ns, nmax = nt > ns ? nt : ns;
    int units = 2 + op_rot_size(nmax, nmin) + 2 * op_z_offset(nmin + 1, nt, ns);
    return (units + 3) & ~3;
}

