"""The reference's T-matrix text file, both directions.

Writer: tmatrix_solution (mstm-solver-8.f90:125-130 header, :243-257 columns,
:321-327 header rewrite when the order loop stops early): a first record
'(2i4)' with the order twice, then for l = 1..T, for the 2(2l+1) columns
(k = -l..l, q = 1, 2 in the kq order of the solve), the entries of rows
n = 1..l, m = -n..n, p = 1, 2, one '(' e18.10 ',' e18.10 ')' per line.

Reader: ranorientscatmatrix (mstm-scatprops-26.f90:2031-2075) reads the order
pair and, for a symmetric file, the same entries back.
"""
import numpy as np


def _e18_10(x):
    """Fortran E18.10: sign, '0.', ten digits, exponent 'E+dd'; right-justified in 18."""
    if x == 0.0:
        return "  0.0000000000E+00"
    m, e = f"{abs(x):.9e}".split("e")
    d = m.replace(".", "")              # ten significant digits d0 d1 ... d9
    exp = int(e) + 1                    # 0.d0d1... x 10^(e+1)
    s = ("-" if x < 0 else "") + "0." + d + "E" + ("+" if exp >= 0 else "-") + f"{abs(exp):02d}"
    return s.rjust(18)


def _index(n, m, p):
    return 2 * (n * (n + 1) + m - 1) + p - 1


def write_tmatrix_file(path, tmat, t_matrix_order, order_used=None):
    """tmat: (nblkt, nblkt) as mstmg_tmatrix returns it; only the columns of orders
    l <= order_used are written, and the header holds order_used twice."""
    T = int(t_matrix_order)
    used = T if order_used is None else int(order_used)
    with open(path, "w") as f:
        f.write(f"{used:4d}{used:4d}\n")
        for l in range(1, used + 1):
            for kq in range(1, 2 * (2 * l + 1) + 1):
                k, q = -l + (kq - 1) // 2, (kq - 1) % 2 + 1
                col = _index(l, k, q)
                for n in range(1, l + 1):
                    for m in range(-n, n + 1):
                        for p in (1, 2):
                            z = tmat[_index(n, m, p), col]
                            f.write("(" + _e18_10(z.real) + "," + _e18_10(z.imag) + ")\n")


def read_tmatrix_file(path):
    """Returns (order, tmat) with tmat (nblkt, nblkt) complex128 holding the file's
    entries (rows of order n <= l in the column of order l; the rest zero)."""
    with open(path) as f:
        head = f.readline()
        T = int(head[0:4])
        vals = []
        for line in f:
            line = line.strip()
            if not line:
                continue
            re_, im_ = line.strip("()").split(",")
            vals.append(complex(float(re_.replace("D", "E")), float(im_.replace("D", "E"))))
    nb = 2 * T * (T + 2)
    tm = np.zeros((nb, nb), np.complex128, order="F")
    it = iter(vals)
    for l in range(1, T + 1):
        for kq in range(1, 2 * (2 * l + 1) + 1):
            k, q = -l + (kq - 1) // 2, (kq - 1) % 2 + 1
            col = _index(l, k, q)
            for n in range(1, l + 1):
                for m in range(-n, n + 1):
                    for p in (1, 2):
                        tm[_index(n, m, p), col] = next(it)
    return T, tm
