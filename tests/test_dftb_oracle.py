"""Pin the DFTB2 / DFTB3 CPU oracle against the reference's DFTB+ known answers
(tests/golden/dftb_known_answers.json, extracted from the reference's
DFTB2Test.cpp / DFTB3Test.cpp) and check its internal consistency."""
import json
import os

import numpy as np
import pytest

from tests import oracle_lib as O

HERE = os.path.dirname(os.path.abspath(__file__))
KA = json.load(open(os.path.join(HERE, "golden", "dftb_known_answers.json")))["tests"]
EMBEDDED = {"mio-1-1", "3ob-3-1", "3ob-2-1"}
ELEMENTS = {"H", "C", "N", "O"}


def _cases():
    out = []
    for t in KA:
        if t["parameters"] in EMBEDDED and set(t["elements"]) <= ELEMENTS:
            out.append(pytest.param(t, id="%s-dftb%d" % (t["name"], t["order"])))
    return out


def _bohr(t):
    return np.array(t["xyz_angstrom"]) * O.bohr_per_angstrom()


@pytest.mark.parametrize("t", _cases())
def test_dftb_known_answers(t):
    Z = [O.SYMBOLS[e] for e in t["elements"]]
    r = O.dftb_scf(t["order"], Z, _bohr(t), parameters=t["parameters"], scc=1e-10, rmsd=1e-9)
    assert r["converged"]
    assert abs(r["energy"] - t["energy"]) < t["energy_tol"]
    if "charges" in t:
        q = r["charges"][:len(t["charges"])]
        assert np.max(np.abs(q - np.array(t["charges"]))) < t["charges_tol"]
    if "orbital_energies" in t:
        eps = r["eps"][:len(t["orbital_energies"])]
        assert np.max(np.abs(eps - np.array(t["orbital_energies"]))) < t["orbital_energies_tol"]
    if "forces" in t:
        f = np.array(t["forces"])
        g = r["gradient"][:len(f)]
        assert np.max(np.linalg.norm(-g - f, axis=1)) < max(t["forces_tol"], 1e-10)


def _water_dimer():
    x = np.array([[0.0, 0.0, 0.0], [0.96, 0.0, 0.0], [-0.24, 0.93, 0.0],
                  [2.9, 0.1, 0.2], [3.4, 0.8, -0.3], [3.3, -0.7, 0.1]]) * O.bohr_per_angstrom()
    return [8, 1, 1, 8, 1, 1], x


@pytest.mark.parametrize("order,params", [(2, "mio-1-1"), (3, "3ob-3-1")])
def test_dftb_atom_order_invariance(order, params):
    Z, x = _water_dimer()
    perm = [3, 1, 5, 0, 4, 2]
    a = O.dftb_scf(order, Z, x, parameters=params, scc=1e-10, rmsd=1e-9)
    b = O.dftb_scf(order, [Z[i] for i in perm], x[perm], parameters=params, scc=1e-10, rmsd=1e-9)
    assert abs(a["energy"] - b["energy"]) < 1e-9
    if order == 2:
        # DFTB3 gradients follow the reference's pair term, whose Gamma_ba part
        # depends on which atom of a pair comes first (see dftb_oracle.cpp)
        assert np.max(np.abs(a["gradient"][perm] - b["gradient"])) < 1e-7


def test_dftb2_gradient_matches_finite_difference():
    Z, x = _water_dimer()
    r = O.dftb_scf(2, Z, x, scc=1e-11, rmsd=1e-10)
    h = 1e-4
    for a, k in [(0, 0), (2, 1), (4, 2), (3, 0)]:
        xp, xm = x.copy(), x.copy()
        xp[a, k] += h
        xm[a, k] -= h
        ep = O.dftb_scf(2, Z, xp, scc=1e-12, rmsd=1e-10, gradient=False)["energy"]
        em = O.dftb_scf(2, Z, xm, scc=1e-12, rmsd=1e-10, gradient=False)["energy"]
        assert abs((ep - em) / (2 * h) - r["gradient"][a, k]) < 2e-6


def test_dftb3_gradient_gamma_terms_as_in_the_reference():
    # the reference's DFTB3 pair term differs from the energy derivative only
    # through the Gamma_ba sign (see dftb_oracle.cpp); on a neutral, nearly
    # charge-free dimer both agree to the size of (2/3) q_a q_b^2 Gamma_ba'
    Z, x = _water_dimer()
    r = O.dftb_scf(3, Z, x, scc=1e-11, rmsd=1e-10)
    h = 1e-4
    xp, xm = x.copy(), x.copy()
    xp[0, 0] += h
    xm[0, 0] -= h
    ep = O.dftb_scf(3, Z, xp, scc=1e-12, rmsd=1e-10, gradient=False)["energy"]
    em = O.dftb_scf(3, Z, xm, scc=1e-12, rmsd=1e-10, gradient=False)["energy"]
    assert abs((ep - em) / (2 * h) - r["gradient"][0, 0]) < 5e-3


def test_dftb_matrices_are_symmetric_and_bookkept():
    Z, x = _water_dimer()
    H0, S, gam, Gam = O.dftb_matrices(3, Z, x)
    assert H0.shape == (12, 12)
    assert np.allclose(H0, H0.T) and np.allclose(S, S.T)
    assert np.allclose(np.diag(S), 1.0)
    assert np.allclose(gam, gam.T)
    assert np.all(np.linalg.eigvalsh(S) > 0)
