"""The TD-DFTB oracle against the reference's known answers
(src/Sparrow/Tests/TimeDependent/TDDFTBTest.cpp, extracted into
tests/golden/tddftb_known_answers.json): the ten lowest singlet and triplet
excitation energies of a distorted methane with mio-1-1 DFTB2 at the
reference's 1e-3 eV, and the DFTB+ gamma matrix of the same molecule at 1e-4.
"""
import json
import os

import numpy as np
import pytest

from tests import oracle_lib as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "tddftb_known_answers.json")))
SYM = {"H": 1, "C": 6, "N": 7, "O": 8}


def _case(name):
    rec = next(t for t in GOLD["tests"] if t["name"] == name)
    Z = [SYM[e] for e in rec["elements"]]
    x = np.array(rec["xyz_angstrom"]) * O.bohr_per_angstrom()
    return rec, Z, x


@pytest.mark.parametrize("name", ["CanPerformRestrictedSingletTDDFTCalculation",
                                  "CanPerformRestrictedTripletTDDFTCalculation"])
def test_excitation_energies_match_reference(name):
    rec, Z, x = _case(name)
    n = len(rec["energies_ev"])
    r = O.dftb_tddftb(2, Z, x, nroots=n, triplet=rec["spin"] == "triplet", parameters=rec["parameters"])
    got = r["omega"] * O.ev_per_hartree()
    assert np.max(np.abs(got - np.array(rec["energies_ev"]))) < rec["tolerance_ev"]


def test_gamma_matrix_matches_dftbplus():
    rec, Z, x = _case("TDDFTBDataRecordsRightConstants")
    n = rec["gamma_n"]
    ref = np.array(rec["gamma_lower_rowmajor"]).reshape(n, n)
    ref = np.tril(ref) + np.tril(ref, -1).T
    _, _, gam, _ = O.dftb_matrices(2, Z, x, parameters=rec["parameters"])
    assert np.max(np.abs(gam - ref)) < rec["gamma_tolerance"]


def test_excitations_invariant_under_translation():
    # transition charges sum to zero over the atoms, so the transition dipoles
    # do not depend on the origin
    rec, Z, x = _case("CanPerformRestrictedSingletTDDFTCalculation")
    a = O.dftb_tddftb(2, Z, x, nroots=6)
    b = O.dftb_tddftb(2, Z, x + np.array([3.0, -2.0, 1.5]), nroots=6)
    assert np.max(np.abs(a["omega"] - b["omega"])) < 1e-9
    for i in range(6):
        s = 1.0 if np.dot(a["dipoles"][i], b["dipoles"][i]) >= 0 else -1.0
        assert np.max(np.abs(a["dipoles"][i] - s * b["dipoles"][i])) < 1e-7


def test_davidson_path_matches_dense_diagonalisation():
    # the oracle's matrix-free Davidson iteration (used above 2000
    # transitions) against its dense diagonalisation on the same polyene and
    # on the reference's methane: energies and transition dipoles
    from sparrow_b200 import geometry
    rng = np.random.default_rng(4)
    Z, xa = geometry.polyene(6, rng)
    cases = [(3, Z, geometry.to_bohr(xa), None), (2,) + _case("CanPerformRestrictedSingletTDDFTCalculation")[1:] +
             ("mio-1-1",)]
    try:
        for order, Zc, xc, params in cases:
            O.set_dense_casida_limit(100000)
            dense = O.dftb_tddftb(order, Zc, xc, nroots=8, parameters=params)
            O.set_dense_casida_limit(0)
            dav = O.dftb_tddftb(order, Zc, xc, nroots=8, parameters=params)
            assert np.max(np.abs(dense["omega"] - dav["omega"])) < 1e-10
            for i in range(len(dense["omega"])):
                s = 1.0 if np.dot(dense["dipoles"][i], dav["dipoles"][i]) >= 0 else -1.0
                assert np.max(np.abs(dense["dipoles"][i] - s * dav["dipoles"][i])) < 1e-7
    finally:
        O.set_dense_casida_limit(2000)
