"""Atomic charges (the AtomicCharges result) on the GPU.

DFTB: the reference's DFTB+ known answers at its 1e-6 (CH4,
src/Sparrow/Tests/MethodsTests/Dftb/DFTB2Test.cpp:97-126 with mio-1-1 and
DFTB3Test.cpp:94-123 with 3ob-2-1; the spin-polarised CH3 doublets of the
same files).  NDDO: core charge minus the atom's diagonal density of the
oracle's converged density, 1e-6; the charges sum to the molecular charge.
"""
import numpy as np
import pytest

import sparrow_b200
from sparrow_b200 import geometry
from tests import oracle_lib as O
from tests.test_sdftb_oracle import CH3, KNOWN

pytestmark = pytest.mark.gpu

CH4 = np.array([[0, 0, 0], [0.6287, 0.6287, 0.6287], [-0.6287, -0.6287, 0.6287], [-0.6287, 0.6287, -0.6287],
                [0.6287, -0.6287, -0.6287]])


def _charges(method, Z, x, params=None, mult=1, charge=0):
    c = sparrow_b200.get_calculator(method)
    c.set_structure(Z, x)
    if params:
        c.settings["method_parameters"] = params
    c.settings["spin_multiplicity"] = mult
    c.settings["molecular_charge"] = charge
    c.settings["self_consistence_criterion"] = 1e-11
    c.settings["density_rmsd_criterion"] = 1e-10
    c.settings["max_scf_iterations"] = 500
    c.set_required_properties(["energy", "atomic_charges"])
    r = c.calculate()
    assert r.successful_calculation
    return r.atomic_charges


@pytest.mark.parametrize("method,params,expected", [
    ("DFTB2", "mio-1-1", [-0.30575605, 0.07643901, 0.07643901, 0.07643901, 0.07643901]),
    ("DFTB3", "3ob-2-1", [-0.41128058, 0.10282014, 0.10282014, 0.10282014, 0.10282014]),
])
def test_dftb_ch4_matches_dftbplus(method, params, expected):
    q = _charges(method, [6, 1, 1, 1, 1], CH4 * O.bohr_per_angstrom(), params)
    assert np.max(np.abs(q - expected)) < 1e-6


@pytest.mark.parametrize("order", [2, 3])
def test_spin_polarised_ch3_matches_dftbplus(order):
    k = KNOWN[order]
    q = _charges("DFTB%d" % order, [6, 1, 1, 1], CH3 * O.bohr_per_angstrom(), k["parameters"], mult=2)
    assert np.max(np.abs(q - k["charges"])) < 1e-6


@pytest.mark.parametrize("method", ["PM6", "AM1", "MNDO"])
def test_nddo_charges_match_oracle(method):
    Z, xa = geometry.water_cluster(3, seed=4)
    Z = list(Z) + [7, 1, 1, 1, 1]  # with an NH4+ ion
    nh4 = np.array([[0, 0, 0], [0.6, 0.6, 0.6], [-0.6, -0.6, 0.6], [-0.6, 0.6, -0.6], [0.6, -0.6, -0.6]]) + [6.0, 0, 0]
    x = geometry.to_bohr(np.vstack([xa, nh4]))
    q = _charges(method, Z, x, charge=1)
    ref = O.scf(method, Z, x, charge=1, scc=1e-11, rmsd=1e-10, want_density=True)
    core = {1: 1.0, 7: 5.0, 8: 6.0}
    nao = {1: 1, 7: 4, 8: 4}
    expected, k = [], 0
    for z in Z:
        expected.append(core[z] - np.trace(ref["P"][k:k + nao[z], k:k + nao[z]]))
        k += nao[z]
    assert np.max(np.abs(q - expected)) < 1e-6
    assert abs(q.sum() - 1.0) < 1e-9
