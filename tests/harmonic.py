"""Harmonic frequencies from a Cartesian Hessian (test infrastructure).

Mass-weighting with standard atomic weights, projection of the rigid
translations and rotations about the centre of mass, and conversion of the
eigenvalues (Hartree / (bohr^2 u)) to wavenumbers, negative for imaginary
modes; the 3n - 6 (3n - 5 when linear) vibrational frequencies in ascending
order, as the reference's app lists them.
"""
import numpy as np

MASS = {1: 1.00794, 6: 12.0107, 7: 14.0067, 8: 15.9994}
HARTREE_J = 4.359744650e-18
BOHR_M = 0.52917721067e-10
AMU_KG = 1.660539040e-27
C_CM_S = 2.99792458e10


def frequencies(Z, xyz_bohr, H):
    Z = list(Z)
    x = np.asarray(xyz_bohr, dtype=float).reshape(-1, 3)
    m = np.array([MASS[z] for z in Z])
    sm = np.sqrt(m)
    m3 = np.repeat(m, 3)
    Hm = np.asarray(H) / np.sqrt(np.outer(m3, m3))
    r = x - (x * m[:, None]).sum(0) / m.sum()
    rigid = []
    for a in range(3):
        v = np.zeros_like(x)
        v[:, a] = sm
        rigid.append(v.reshape(-1))
    for a in range(3):
        e = np.zeros(3)
        e[a] = 1.0
        rigid.append((np.cross(e, r) * sm[:, None]).reshape(-1))
    U, s, _ = np.linalg.svd(np.array(rigid).T, full_matrices=False)
    Q = U[:, s > 1e-6 * s.max()]
    P = np.eye(len(m3)) - Q @ Q.T
    w, _ = np.linalg.eigh(P @ Hm @ P)
    # drop the rigid-motion null space: the eigenvalues closest to zero
    keep = np.sort(np.argsort(np.abs(w))[Q.shape[1]:])
    w = w[keep]
    f = np.sqrt(np.abs(w) * HARTREE_J / (BOHR_M ** 2 * AMU_KG)) / (2 * np.pi * C_CM_S)
    return np.sort(np.sign(w) * f)
