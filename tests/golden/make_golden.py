"""Generate the committed golden fixtures under tests/golden/.

mie_bh.npz: Lorenz-Mie coefficients a_n, b_n and Qext, Qsca for the size
parameters and indices of the workloads, computed with the textbook
Bohren-Huffman formulas on scipy's spherical Bessel functions -- an
implementation independent of MSTM's mieoa (mstm-modules-33.f90:5438-5578).
MSTM's LR-basis 2x2 Mie matrix maps to the TE/TM basis as diag(-a_n, -b_n).

Run:  python tests/golden/make_golden.py
"""
import os

import numpy as np
from scipy.special import spherical_jn, spherical_yn

HERE = os.path.dirname(os.path.abspath(__file__))


def bohren_huffman(x, m, N):
    n = np.arange(1, N + 1)

    def psi(z):
        return z * spherical_jn(n, z)

    def dpsi(z):
        return spherical_jn(n, z) + z * spherical_jn(n, z, derivative=True)

    def xi(z):
        return z * (spherical_jn(n, z) + 1j * spherical_yn(n, z))

    def dxi(z):
        return (spherical_jn(n, z) + 1j * spherical_yn(n, z)) + z * (
            spherical_jn(n, z, derivative=True) + 1j * spherical_yn(n, z, derivative=True))

    mx = m * x
    a = (m * psi(mx) * dpsi(x) - psi(x) * dpsi(mx)) / (m * psi(mx) * dxi(x) - xi(x) * dpsi(mx))
    b = (psi(mx) * dpsi(x) - m * psi(x) * dpsi(mx)) / (psi(mx) * dxi(x) - m * xi(x) * dpsi(mx))
    qe = 2 / x ** 2 * np.sum((2 * n + 1) * (a + b).real)
    qs = 2 / x ** 2 * np.sum((2 * n + 1) * (abs(a) ** 2 + abs(b) ** 2))
    return a, b, qe, qs


def main():
    cases = [(1.0, 1.5 + 0.01j, 7), (2.0, 1.6 + 0.05j, 9), (1.5, 1.6 + 0.005j, 8), (0.5, 1.31 + 0.0j, 6),
             (1.0, 1.31 + 0.0j, 7), (3.0, 1.45 + 0.1j, 12)]
    Lmax = max(c[2] for c in cases)
    A = np.zeros((len(cases), Lmax), complex)
    B = np.zeros((len(cases), Lmax), complex)
    qe = np.zeros(len(cases))
    qs = np.zeros(len(cases))
    for k, (x, m, L) in enumerate(cases):
        a, b, e, s = bohren_huffman(x, m, L)
        A[k, :L], B[k, :L], qe[k], qs[k] = a, b, e, s
    np.savez(os.path.join(HERE, "mie_bh.npz"), x=np.array([c[0] for c in cases]), m=np.array([c[1] for c in cases]),
             L=np.array([c[2] for c in cases]), a=A, b=B, qext=qe, qsca=qs)


if __name__ == "__main__":
    main()
