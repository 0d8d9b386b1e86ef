"""Dipole moment against the reference's known answers (tests/golden/dipole_known_answers.json).

CPU: the dipole formulas applied to the oracle's converged state reproduce
the reference's MOPAC PM6 values (NDDO approximation about the centre of
mass, 0.001 D) and its DFTB+ DFTB2 vector (1e-6 e bohr).  GPU: the
Calculator's SG_PROP_DIPOLE matches the same values and the oracle's
dipole within 1e-8 e bohr.
"""
import json
import os

import numpy as np
import pytest

import sparrow_b200
from tests import oracle_lib as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "dipole_known_answers.json")))
SYM = {"H": 1, "C": 6, "N": 7, "O": 8, "F": 9}
MASS = {1: 1.00794, 6: 12.0107, 7: 14.0067, 8: 15.9994, 9: 18.9984032}


def structure(name):
    s = GOLD["structures"][name]
    return [SYM[e] for e in s["elements"]], np.array(s["xyz_angstrom"]) * O.bohr_per_angstrom()


def oracle_nddo_dipole(method, Z, x, charge=0):
    r = O.scf(method, Z, x, charge=charge, scc=1e-11, rmsd=1e-10, want_density=True)
    P = r["P"]
    m = np.array([MASS[z] for z in Z])
    xr = x - (x * m[:, None]).sum(0) / m.sum()
    mu, k = np.zeros(3), 0
    for a, z in enumerate(Z):
        ep = O.element_params(method, z)
        nao, core, D = int(ep[0]), ep[1], ep[7]
        mu += (core - np.trace(P[k:k + nao, k:k + nao])) * xr[a]
        if nao == 4:
            mu -= 2 * D * P[k, k + 1:k + 4]
        k += nao
    return mu


def oracle_dftb_dipole(Z, x):
    r = O.dftb_scf(2, Z, x, scc=1e-11, rmsd=1e-10)
    return (r["charges"][:, None] * x).sum(0)


@pytest.mark.parametrize("case", GOLD["pm6_norm_debye"], ids=lambda c: c["structure"])
def test_oracle_pm6_dipole_matches_mopac(case):
    Z, x = structure(case["structure"])
    mu = oracle_nddo_dipole("PM6", Z, x)
    assert abs(np.linalg.norm(mu) * GOLD["debye_per_e_bohr"] - case["value"]) < case["tolerance"]


def test_oracle_dftb2_dipole_matches_dftbplus():
    case = GOLD["dftb2_vector_e_bohr"]
    Z, x = structure(case["structure"])
    assert np.max(np.abs(oracle_dftb_dipole(Z, x) - case["value"])) < case["tolerance"]


def _engine_dipole(method, Z, x, charge=0):
    c = sparrow_b200.get_calculator(method)
    c.set_structure(Z, x)
    c.settings["molecular_charge"] = charge
    c.settings["self_consistence_criterion"] = 1e-11
    c.settings["density_rmsd_criterion"] = 1e-10
    c.set_required_properties(["energy", "dipole"])
    r = c.calculate()
    assert r.successful_calculation
    return r.dipole


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLD["pm6_norm_debye"], ids=lambda c: c["structure"])
def test_gpu_pm6_dipole(case):
    Z, x = structure(case["structure"])
    mu = _engine_dipole("PM6", Z, x)
    assert abs(np.linalg.norm(mu) * GOLD["debye_per_e_bohr"] - case["value"]) < case["tolerance"]
    assert np.max(np.abs(mu - oracle_nddo_dipole("PM6", Z, x))) < 1e-8


@pytest.mark.gpu
def test_gpu_dftb2_dipole():
    case = GOLD["dftb2_vector_e_bohr"]
    Z, x = structure(case["structure"])
    mu = _engine_dipole("DFTB2", Z, x)
    assert np.max(np.abs(mu - case["value"])) < case["tolerance"]
    assert np.max(np.abs(mu - oracle_dftb_dipole(Z, x))) < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["AM1", "MNDO"])
def test_gpu_nddo_dipole_of_an_ion_matches_oracle(method):
    # a cation: its dipole depends on the origin, here the centre of mass
    Z = [7, 1, 1, 1, 1]
    x = np.array([[0, 0, 0], [0.6, 0.6, 0.6], [-0.6, -0.6, 0.6], [-0.6, 0.6, -0.6], [0.7, -0.5, -0.6]]) * 1.8 + 0.7
    mu = _engine_dipole(method, Z, x, charge=1)
    assert np.max(np.abs(mu - oracle_nddo_dipole(method, Z, x, charge=1))) < 1e-8
