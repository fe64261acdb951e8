"""Seeded sphere-cluster generators and position-file I/O.

MSTM's own generator (random_configuration-10.f90:43-364, 479-540) draws from an
unseeded ``random_seed()``; these generators are seeded so every workload is
reproducible.  Positions are in size-parameter units (k = 1), so a sphere's
radius is its size parameter x, as in MSTM (input:2886-2923).

* ``rsa_sphere`` / ``rsa_cylinder``: random sequential addition inside a
  bounding sphere or an upright cylinder, sampling as ``sample_position``
  (random_configuration-10.f90:327-364) does, rejecting overlaps as
  ``add_sphere_to_cluster`` (random_configuration-10.f90:479-540) does.
* ``pca_aggregate``: tunable particle-cluster aggregation with fractal
  dimension Df and prefactor kf (N = kf (Rg/a)^Df at every step).  The
  reference ships no such generator (only the example file
  examples/frac_agg.pos).
"""
import math

import numpy as np


def truncation_order(x):
    """L = round(x + 4 x^(1/3) + 2), the order the workloads force with mie_epsilon=-L."""
    return int(round(x + 4.0 * x ** (1.0 / 3.0) + 2.0))


class _Grid:
    def __init__(self, cell):
        self.cell = cell
        self.cells = {}

    def key(self, p):
        return tuple(int(math.floor(v / self.cell)) for v in p)

    def add(self, idx, p):
        self.cells.setdefault(self.key(p), []).append(idx)

    def near(self, p):
        k = self.key(p)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    yield from self.cells.get((k[0] + dx, k[1] + dy, k[2] + dz), ())


def _rsa(n, radius, sampler, rng, gap=0.0, max_tries=2000000):
    pos = np.zeros((n, 3))
    grid = _Grid(2.0 * radius + gap)
    placed = 0
    tries = 0
    while placed < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("random sequential addition failed to place %d spheres" % n)
        p = sampler(rng)
        ok = True
        for j in grid.near(p):
            if np.sum((p - pos[j]) ** 2) < (2.0 * radius + gap) ** 2:
                ok = False
                break
        if ok:
            pos[placed] = p
            grid.add(placed, p)
            placed += 1
    return pos


def rsa_sphere(n, radius, volume_fraction, seed):
    """n equal spheres by random sequential addition in a bounding sphere.

    The bounding radius R satisfies n radius^3 / R^3 = volume_fraction.
    """
    rng = np.random.default_rng(seed)
    R = radius * (n / volume_fraction) ** (1.0 / 3.0)

    def sampler(g):
        u = g.random(3)
        r = (R - radius) * u[0] ** (1.0 / 3.0)
        phi = 2.0 * math.pi * u[1]
        ct = -1.0 + 2.0 * u[2]
        st = math.sqrt(max(0.0, 1.0 - ct * ct))
        return np.array([r * st * math.cos(phi), r * st * math.sin(phi), r * ct])

    return _rsa(n, radius, sampler, rng), R


def rsa_sphere_batched(n, radius, volume_fraction, seed, batch=None):
    """Random sequential addition in a bounding sphere, candidates drawn in
    batches: each batch of uniform points in the sphere is screened against
    the spheres already placed and, in draw order, against the earlier
    candidates it keeps (a k-d tree finds the pairs closer than a diameter),
    so the accepted set is what adding the candidates one at a time would
    give.  Same process and bounding radius as rsa_sphere, another random
    stream; for drawing many configurations quickly (the warm-start study)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    R = radius * (n / volume_fraction) ** (1.0 / 3.0)
    d2 = 2.0 * radius
    placed = np.zeros((0, 3))
    batch = batch or max(64, 2 * n)
    while len(placed) < n:
        u = rng.random((batch, 3))
        r = (R - radius) * u[:, 0] ** (1.0 / 3.0)
        phi = 2.0 * math.pi * u[:, 1]
        ct = -1.0 + 2.0 * u[:, 2]
        st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
        cand = np.stack([r * st * np.cos(phi), r * st * np.sin(phi), r * ct], axis=1)
        ok = np.ones(batch, bool)
        if len(placed):
            dist, _ = cKDTree(placed).query(cand, k=1)
            ok &= dist >= d2
        idx = np.nonzero(ok)[0]
        pairs = cKDTree(cand[idx]).query_pairs(d2, output_type="ndarray") if len(idx) > 1 else np.zeros((0, 2), int)
        conflicts = [[] for _ in range(len(idx))]
        for a_, b_ in pairs:
            lo, hi = (a_, b_) if a_ < b_ else (b_, a_)
            conflicts[hi].append(lo)
        keep = np.zeros(len(idx), bool)
        need = n - len(placed)
        for q in range(len(idx)):
            if need == 0:
                break
            if not any(keep[p_] for p_ in conflicts[q]):
                keep[q] = True
                need -= 1
        placed = np.concatenate([placed, cand[idx[keep]]])
    return placed[:n], R


def rsa_cylinder(n, radius, volume_fraction, aspect, seed):
    """n equal spheres by random sequential addition in a cylinder (axis z).

    aspect = length / diameter; n (4/3 pi radius^3) / (pi Rc^2 H) = volume_fraction.
    """
    rng = np.random.default_rng(seed)
    vol = n * 4.0 / 3.0 * math.pi * radius ** 3 / volume_fraction
    Rc = (vol / (2.0 * math.pi * aspect)) ** (1.0 / 3.0)
    H = 2.0 * aspect * Rc

    def sampler(g):
        u = g.random(3)
        r = (Rc - radius) * math.sqrt(u[0])
        phi = 2.0 * math.pi * u[1]
        z = -0.5 * H + radius + (H - 2.0 * radius) * u[2]
        return np.array([r * math.cos(phi), r * math.sin(phi), z])

    return _rsa(n, radius, sampler, rng), (Rc, H)


def pca_aggregate(n, radius, df, kf, seed, max_tries=400):
    """Touching monomers by tunable particle-cluster aggregation.

    Monomer k+1 is placed in contact with a randomly chosen monomer at the
    distance Gamma from the centre of mass that keeps N Rg_N^2 on the target
    N = kf (Rg/a)^Df:  Gamma^2 = N/(N-1) (N Rg_N^2 - (N-1) Rg_{N-1}^2).
    """
    rng = np.random.default_rng(seed)
    a = radius
    pos = np.zeros((n, 3))
    if n == 1:
        return pos
    d = rng.normal(size=3)
    pos[1] = 2.0 * a * d / np.linalg.norm(d)

    def rg2(N):
        return (a * (N / kf) ** (1.0 / df)) ** 2

    grid = _Grid(2.0 * a)
    grid.add(0, pos[0])
    grid.add(1, pos[1])
    for k in range(2, n):
        N = k + 1
        c = pos[:k].mean(axis=0)
        g2 = N / (N - 1.0) * (N * rg2(N) - (N - 1.0) * rg2(N - 1))
        gam = math.sqrt(max(g2, (2.0 * a) ** 2 * 0.25))
        dist = np.linalg.norm(pos[:k] - c, axis=1)
        placed = False
        for attempt in range(max_tries):
            # candidates whose contact sphere (radius 2a) meets the sphere of radius gamma about c
            band = 2.0 * a + attempt * 0.01 * a
            cand = np.nonzero(np.abs(dist - gam) <= band)[0]
            if len(cand) == 0:
                cand = np.array([int(np.argmin(np.abs(dist - gam)))])
            j = int(cand[rng.integers(len(cand))])
            pj = pos[j]
            v = pj - c
            dj = np.linalg.norm(v)
            if dj < 1e-12:
                v = rng.normal(size=3)
                dj = np.linalg.norm(v)
            u = v / dj
            # intersection circle of |p-c|=gam and |p-pj|=2a (clamped to a valid cosine)
            cosang = (gam * gam + dj * dj - 4.0 * a * a) / (2.0 * gam * dj) if dj > 0 else 1.0
            cosang = min(1.0, max(-1.0, cosang))
            sinang = math.sqrt(1.0 - cosang * cosang)
            t = rng.normal(size=3)
            t -= t.dot(u) * u
            t /= np.linalg.norm(t)
            w = np.cross(u, t)
            phi = 2.0 * math.pi * rng.random()
            dirv = cosang * u + sinang * (math.cos(phi) * t + math.sin(phi) * w)
            p = c + gam * dirv
            # put the new monomer exactly in contact with j
            dv = p - pj
            p = pj + 2.0 * a * dv / np.linalg.norm(dv)
            ok = True
            for i in grid.near(p):
                if i != j and np.sum((p - pos[i]) ** 2) < (2.0 * a) ** 2 * (1.0 - 1e-12):
                    ok = False
                    break
            if ok:
                pos[k] = p
                grid.add(k, p)
                placed = True
                break
        if not placed:
            raise RuntimeError("aggregation failed at monomer %d" % k)
    return pos - pos.mean(axis=0)


def radius_of_gyration(pos):
    c = pos.mean(axis=0)
    return math.sqrt(np.mean(np.sum((pos - c) ** 2, axis=1)))


def write_position_file(path, pos, radius, ref_index=None):
    """x y z r [Re(m) Im(m)] lines, readable by read_sphere_data_input_file (input:2886-2923)."""
    with open(path, "w") as f:
        for i, p in enumerate(pos):
            r = radius[i] if np.ndim(radius) else radius
            if ref_index is None:
                f.write("%.10e %.10e %.10e %.10e\n" % (p[0], p[1], p[2], r))
            else:
                m = ref_index[i] if np.ndim(ref_index) else ref_index
                f.write("%.10e %.10e %.10e %.10e %.10e %.10e\n" % (p[0], p[1], p[2], r, m.real, m.imag))


def read_position_file(path):
    rows = [list(map(float, line.split())) for line in open(path) if line.strip()]
    a = np.array([r[:4] for r in rows])
    return a[:, :3], a[:, 3]


# ---------------------------------------------------------------------------
# The named workloads (sizes and seeds fixed here so tests and bench agree).
# ---------------------------------------------------------------------------
def host_inclusions(n, radius, volume_fraction, seed, host_index=1.33 + 0.0j, inclusion_index=1.6 + 0.05j):
    """A host sphere holding n equal inclusions placed by random sequential
    addition (rsa_sphere: inclusion volume fraction `volume_fraction` of the
    host).  Returns dict(pos, radius, ref_index) with the host first, at the
    origin, its radius the RSA bounding radius so every inclusion lies inside."""
    inner, R = rsa_sphere(n, radius, volume_fraction, seed)
    pos = np.vstack([np.zeros((1, 3)), inner])
    rad = np.r_[R, np.full(n, radius)]
    ri = np.r_[complex(host_index), np.full(n, complex(inclusion_index))]
    return dict(pos=pos, radius=rad, ref_index=ri.astype(np.complex128))


def workload(name):
    """Return dict(pos, radius, ref_index, order) for a named workload."""
    if name == "cluster20":
        x, m = 1.0, 1.5 + 0.01j
        pos, _ = rsa_sphere(20, x, 0.10, seed=1)
    elif name == "fractal500":
        x, m = 2.0, 1.6 + 0.05j
        pos = pca_aggregate(500, x, 1.8, 1.3, seed=2)
    elif name.startswith("fractal"):
        n = int(name[len("fractal"):])
        x, m = 2.0, 1.6 + 0.05j
        pos = pca_aggregate(n, x, 1.8, 1.3, seed=2)
    elif name.startswith("cluster"):
        n = int(name[len("cluster"):])
        x, m = 1.0, 1.5 + 0.01j
        pos, _ = rsa_sphere(n, x, 0.10, seed=1)
    else:
        raise KeyError(name)
    n = len(pos)
    return dict(pos=pos, radius=np.full(n, x), ref_index=np.full(n, m, dtype=np.complex128),
                order=truncation_order(x), x=x, m=m)
