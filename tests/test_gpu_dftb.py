"""DFTB2 / DFTB3 on the GPU against the CPU oracle and the reference's DFTB+
known answers (energies 1e-6 Eh, gradients 1e-5 Eh/bohr)."""
import json
import os

import numpy as np
import pytest

import sparrow_b200
from sparrow_b200 import geometry
from tests import oracle_lib as O

pytestmark = pytest.mark.gpu

E_TOL = 1e-6   # Hartree
G_TOL = 1e-5   # Hartree / bohr
HERE = os.path.dirname(os.path.abspath(__file__))
KA = {(t["name"], t["order"]): t
      for t in json.load(open(os.path.join(HERE, "golden", "dftb_known_answers.json")))["tests"]}


def _ka(name, order):
    t = KA[(name, order)]
    return t, [O.SYMBOLS[e] for e in t["elements"]], np.array(t["xyz_angstrom"]) * O.bohr_per_angstrom()


@pytest.mark.parametrize("order", [2, 3])
def test_ch4_known_answer_through_the_calculator(order):
    t, Z, x = _ka("GetsSameResultAsDFTBPlusForCH4", order)
    c = sparrow_b200.get_calculator("DFTB%d" % order)
    c.settings["method_parameters"] = t["parameters"]
    c.settings["density_rmsd_criterion"] = 1e-9
    c.settings["self_consistence_criterion"] = 1e-10
    c.set_structure(Z, x)
    c.set_required_properties(["energy", "gradients"])
    r = c.calculate()
    assert r.successful_calculation
    assert abs(r.energy - t["energy"]) < max(t["energy_tol"], 1e-8)
    f = np.array(t["forces"])
    assert np.max(np.linalg.norm(-r.gradients - f, axis=1)) < t["forces_tol"]
    ref = O.dftb_scf(order, Z, x, parameters=t["parameters"], scc=1e-10, rmsd=1e-9)
    assert abs(r.energy - ref["energy"]) < E_TOL
    assert np.max(np.abs(r.gradients - ref["gradient"])) < G_TOL


@pytest.mark.parametrize("order", [2, 3])
def test_carbon_atom(order):
    t, Z, x = _ka("GetsSameResultAsDFTBPlusForC", order)
    e, g, it, conv = sparrow_b200.batch_calculate("DFTB%d:%s" % (order, t["parameters"]), [(Z, x)], gradients=True)
    assert abs(e[0] - t["energy"]) < t["energy_tol"]
    assert np.max(np.abs(g[0])) < 1e-12


@pytest.mark.parametrize("order", [2, 3])
def test_water_cluster_and_alkanes_against_oracle(order):
    Zw, xw = geometry.water_cluster(8, seed=4)
    mols = [(np.asarray(Zw), geometry.to_bohr(xw))]
    rng = np.random.default_rng(7)
    for n in (1, 4, 9):
        z, x = geometry.alkane(n, rng)
        mols.append((np.asarray(z), geometry.to_bohr(x)))
    e, g, it, conv = sparrow_b200.batch_calculate("DFTB%d" % order, mols, scc=1e-9, rmsd=1e-8, gradients=True)
    assert conv.all()
    for i, (z, x) in enumerate(mols):
        ref = O.dftb_scf(order, z, x, scc=1e-10, rmsd=1e-9)
        assert abs(e[i] - ref["energy"]) < E_TOL
        assert np.max(np.abs(g[i] - ref["gradient"])) < G_TOL


def test_dftb3_polyenes_against_oracle():
    mols = [(np.asarray(z), geometry.to_bohr(x)) for z, x in geometry.polyene_batch(3, seed=6, k_max=20)]
    e, g, it, conv = sparrow_b200.batch_calculate("DFTB3", mols, scc=1e-9, rmsd=1e-8, gradients=True)
    assert conv.all()
    for i, (z, x) in enumerate(mols):
        ref = O.dftb_scf(3, z, x, scc=1e-10, rmsd=1e-9)
        assert abs(e[i] - ref["energy"]) < E_TOL
        assert np.max(np.abs(g[i] - ref["gradient"])) < G_TOL


def test_dftb_errors_and_warm_start():
    c = sparrow_b200.get_calculator("DFTB2")
    c.set_structure([17, 17], np.array([[0, 0, 0], [3.8, 0, 0.0]]))
    with pytest.raises(sparrow_b200.SparrowError) as ei:   # Cl is not embedded (d shell)
        c.calculate()
    assert ei.value.code == 3
    Z, x = geometry.water_cluster(3, seed=5)
    c.set_structure(Z, geometry.to_bohr(x))
    c.settings["method_parameters"] = "no-such-set"  # neither an embedded set nor a directory
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        c.calculate()
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS
    c.settings["method_parameters"] = ""
    r1 = c.calculate()
    P = c.density()
    c.set_density(P)
    r2 = c.calculate()
    assert r2.iterations <= 3 and abs(r1.energy - r2.energy) < 1e-8
