"""Invariances of the GPU results, after the reference's tests
(src/Sparrow/Tests/MethodsTests/Pm6/PM6Test.cpp:237-258: the energy does not
depend on the atom order, 1e-10; the same holds for rigid motions).

One batch holds a molecule in several atom orders and rigid rotations /
translations: energies agree to 1e-9 Hartree, gradients (permuted back,
rotated back) to 1e-8 Hartree/bohr; restricted PM6, DFTB2, DFTB3 and an
unrestricted PM6 radical.  The DFTB3 gradient is checked under rigid motion
only: the reference's third-order pair term (Dftb/Utils/ThirdOrderFock.cpp,
kept for parity) treats the two atoms of a pair asymmetrically, so its
gradient moves by ~1e-4 Hartree/bohr when the atoms are renumbered (the
oracle shows the same), while the energy does not.
"""
import numpy as np
import pytest

import sparrow_b200
from sparrow_b200 import geometry

pytestmark = pytest.mark.gpu


def _rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def _variants(Z, x, rng, n=4, permute=True):
    """(Z', x', permutation, rotation) with x' = (x[perm] @ R^T) + t."""
    out = [(np.asarray(Z), x, np.arange(len(Z)), np.eye(3))]
    for _ in range(n):
        perm = rng.permutation(len(Z)) if permute else np.arange(len(Z))
        R = _rotation(rng)
        t = rng.normal(size=3) * 3.0
        out.append((np.asarray(Z)[perm], x[perm] @ R.T + t, perm, R))
    return out


@pytest.mark.parametrize("method,mult", [("PM6", 1), ("DFTB2", 1), ("DFTB3", 1), ("PM6", 2), ("DFTB2", 2)])
def test_atom_order_and_rigid_motion(method, mult):
    rng = np.random.default_rng(17)
    z, xa = geometry.alkane(7, rng)
    Z, x = np.asarray(z), geometry.to_bohr(xa)
    if mult == 2:  # heptyl radical
        Z, x = Z[:-1], x[:-1]
    var = _variants(Z, x, rng)
    if method == "DFTB3":  # energies under renumbering; gradients under rigid motion
        b = sparrow_b200.Batch(method, [(v[0], v[1]) for v in var], scc=1e-11, rmsd=1e-10, max_iter=300)
        b.run()
        e = b.results()[0]
        assert np.max(np.abs(e - e[0])) < 1e-9
        var = _variants(Z, x, rng, permute=False)
    b = sparrow_b200.Batch(method, [(v[0], v[1]) for v in var], scc=1e-11, rmsd=1e-10, max_iter=300,
                           multiplicities=[mult] * len(var))
    b.run(gradients=True)
    e, g, _, conv = b.results()
    assert conv.all()
    assert np.max(np.abs(e - e[0])) < 1e-9
    for (Zv, xv, perm, R), gv in zip(var, g):
        back = np.empty_like(gv)
        back[perm] = gv @ R  # undo the rotation (g' = g R^T), then the permutation
        assert np.max(np.abs(back - g[0])) < 1e-8
