"""Seeded synthetic structures for the benchmark and parity workloads.

All generators return ``(Z, xyz_angstrom)`` with ``Z`` an int32 array and
``xyz_angstrom`` a float64 (n_atoms, 3) array.  They draw from numpy's PCG64
(``numpy.random.default_rng(seed)``) so that the oracle and the GPU engine see
identical inputs.

* water clusters (H2O)_n: waters on a grid with 3.0 Angstrom spacing, every
  oxygen jittered by +-0.3 Angstrom (uniform per axis), O-H 0.96 Angstrom,
  H-O-H 104.5 degrees, each water in a uniformly random orientation;
* saturated hydrocarbons C_nH_{2n+2}: all-trans zig-zag backbone, C-C 1.54 and
  C-H 1.09 Angstrom, tetrahedral angles, every C-C-C-C torsion perturbed by a
  uniform +-15 degrees, then a random rigid rotation;
* linear polyenes C_{2k}H_{2k+2}: alternating C=C 1.34 / C-C 1.46 Angstrom,
  C-H 1.09 Angstrom, 120 degree angles, torsions perturbed by +-10 degrees.
"""
import math

import numpy as np

ANGSTROM_TO_BOHR = 1.0 / 0.52917721067
TETRAHEDRAL = math.degrees(math.acos(-1.0 / 3.0))  # 109.47 degrees


def random_rotation(rng):
    """Uniform random rotation matrix from a random unit quaternion."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def grid_shape(n):
    """Near-cubic grid holding n points; 32 -> (4, 4, 2)."""
    if n == 32:
        return (4, 4, 2)
    a = int(round(n ** (1.0 / 3.0)))
    best = None
    for nx in range(max(1, a - 2), a + 3):
        for ny in range(max(1, a - 2), a + 3):
            nz = -(-n // (nx * ny))
            waste = nx * ny * nz - n
            spread = max(nx, ny, nz) - min(nx, ny, nz)
            key = (waste, spread)
            if best is None or key < best[0]:
                best = (key, (nx, ny, nz))
    return best[1]


def water_cluster(n, seed=0, spacing=3.0, jitter=0.3):
    rng = np.random.default_rng(seed)
    nx, ny, nz = grid_shape(n)
    half = math.radians(104.5) / 2
    local = np.array([[0.0, 0.0, 0.0],
                      [0.96 * math.sin(half), 0.0, 0.96 * math.cos(half)],
                      [-0.96 * math.sin(half), 0.0, 0.96 * math.cos(half)]])
    Z, X = [], []
    k = 0
    for ix in range(nx):
        for iy in range(ny):
            for iz in range(nz):
                if k == n:
                    break
                o = np.array([ix, iy, iz], dtype=float) * spacing + rng.uniform(-jitter, jitter, size=3)
                R = random_rotation(rng)
                X.extend(o + local @ R.T)
                Z.extend([8, 1, 1])
                k += 1
    return np.array(Z, dtype=np.int32), np.array(X)


def _place(a, b, c, bond, angle_deg, torsion_deg):
    """Position of atom d with |cd| = bond, angle(b, c, d), dihedral(a, b, c, d)."""
    ang, tor = math.radians(angle_deg), math.radians(torsion_deg)
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    d2 = np.array([-bond * math.cos(ang), bond * math.sin(ang) * math.cos(tor), bond * math.sin(ang) * math.sin(tor)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def _tetrahedral_h(center, neighbors, n_h, dist=1.09, phase=0.0):
    """Hydrogen positions completing a tetrahedron around center."""
    c = np.asarray(center)
    if len(neighbors) == 2:
        u = (c - neighbors[0]) / np.linalg.norm(c - neighbors[0]) + (c - neighbors[1]) / np.linalg.norm(
            c - neighbors[1])
        u /= np.linalg.norm(u)
        v = np.cross(neighbors[0] - c, neighbors[1] - c)
        v /= np.linalg.norm(v)
        h = math.radians(TETRAHEDRAL) / 2
        return [c + dist * (u * math.cos(h) + s * v * math.sin(h)) for s in (1.0, -1.0)]
    if len(neighbors) == 1:
        w = (c - neighbors[0]) / np.linalg.norm(c - neighbors[0])
        ref = np.array([1.0, 0.0, 0.0]) if abs(w[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        p1 = np.cross(w, ref)
        p1 /= np.linalg.norm(p1)
        p2 = np.cross(w, p1)
        t = math.radians(180.0 - TETRAHEDRAL)
        out = []
        for i in range(n_h):
            phi = phase + 2 * math.pi * i / 3
            out.append(c + dist * (w * math.cos(t) + math.sin(t) * (math.cos(phi) * p1 + math.sin(phi) * p2)))
        return out
    # methane
    dirs = np.array([[1, 1, 1], [-1, -1, 1], [-1, 1, -1], [1, -1, -1]], dtype=float) / math.sqrt(3)
    return [c + dist * d for d in dirs[:n_h]]


def alkane(n, rng):
    """C_nH_{2n+2} as (Z, xyz) using the given numpy Generator."""
    cc, ch = 1.54, 1.09
    C = [np.zeros(3)]
    if n >= 2:
        C.append(np.array([cc, 0.0, 0.0]))
    if n >= 3:
        ang = math.radians(180.0 - TETRAHEDRAL)
        C.append(C[1] + cc * np.array([math.cos(ang), math.sin(ang), 0.0]))
    for k in range(3, n):
        tor = 180.0 + rng.uniform(-15.0, 15.0)
        C.append(_place(C[k - 3], C[k - 2], C[k - 1], cc, TETRAHEDRAL, tor))
    Z = [6] * n
    X = list(C)
    for k in range(n):
        nb = []
        if k > 0:
            nb.append(C[k - 1])
        if k < n - 1:
            nb.append(C[k + 1])
        if n == 1:
            hs = _tetrahedral_h(C[0], [], 4, ch)
        elif len(nb) == 1:
            hs = _tetrahedral_h(C[k], nb, 3, ch, phase=math.pi / 3)
        else:
            hs = _tetrahedral_h(C[k], nb, 2, ch)
        X.extend(hs)
        Z.extend([1] * len(hs))
    X = np.array(X)
    X -= X.mean(axis=0)
    X = X @ random_rotation(rng).T
    return np.array(Z, dtype=np.int32), X


def alkane_batch(count, seed=1, n_min=2, n_max=30):
    """`count` hydrocarbons with n uniform in [n_min, n_max]."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_min, n_max + 1, size=count)
    return [alkane(int(n), rng) for n in ns]


def polyene(k, rng):
    """C_{2k}H_{2k+2}, all-trans with +-10 degree torsion noise."""
    nC = 2 * k
    C = [np.zeros(3), np.array([1.34, 0.0, 0.0])]
    if nC >= 3:
        ang = math.radians(60.0)
        C.append(C[1] + 1.46 * np.array([math.cos(ang), math.sin(ang), 0.0]))
    for i in range(3, nC):
        bond = 1.34 if i % 2 == 1 else 1.46
        tor = 180.0 + rng.uniform(-10.0, 10.0)
        C.append(_place(C[i - 3], C[i - 2], C[i - 1], bond, 120.0, tor))
    Z = [6] * nC
    X = list(C)
    for i in range(nC):
        if i == 0 or i == nC - 1:
            nb = C[1] if i == 0 else C[nC - 2]
            prev = C[2] if i == 0 else C[nC - 3]
            for tor in (0.0, 180.0):
                X.append(_place(prev, nb, C[i], 1.09, 120.0, tor))
                Z.append(1)
        else:
            a, b = C[i - 1], C[i + 1]
            u = (C[i] - a) / np.linalg.norm(C[i] - a) + (C[i] - b) / np.linalg.norm(C[i] - b)
            u /= np.linalg.norm(u)
            X.append(C[i] + 1.09 * u)
            Z.append(1)
    X = np.array(X)
    X -= X.mean(axis=0)
    X = X @ random_rotation(rng).T
    return np.array(Z, dtype=np.int32), X


def polyene_batch(count, seed=6, k_min=5, k_max=40):
    rng = np.random.default_rng(seed)
    ks = rng.integers(k_min, k_max + 1, size=count)
    return [polyene(int(k), rng) for k in ks]


def to_bohr(xyz_angstrom):
    return np.asarray(xyz_angstrom, dtype=np.float64) * ANGSTROM_TO_BOHR
