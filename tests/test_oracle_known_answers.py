"""Pin the CPU oracle against the reference's own known-answer tests.

Every vector comes from tests/golden/nddo_known_answers.json, extracted from
the reference's test sources (file:line stored per record).  Tolerances are
the ones the reference asserts.  Structures whose elements need a d shell in
the method (and therefore fall outside the s/p engine) are skipped.
"""
import json
import math
import os

import numpy as np
import pytest

from tests import oracle_lib as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "nddo_known_answers.json")))
KCAL_PER_HARTREE = 627.5094740631  # hartree_per_kCalPerMol of the reference's constants (CODATA 2014)


def _records(method, key):
    out = []
    for r in GOLD["methods"][method]:
        if key in r and not r["name"].startswith("DISABLED"):
            out.append(pytest.param(r, id=r["name"]))
    return out


def _supported(method, r):
    for el in r["elements"]:
        try:
            p = O.element_params(method, O.SYMBOLS[el])
        except RuntimeError:
            return False
        if p[0] not in (1, 4):
            return False
    return True


def _geometry(r):
    Z = [O.SYMBOLS[e] for e in r["elements"]]
    x = np.array(r["xyz_angstrom"]) * O.bohr_per_angstrom()
    return Z, x


def _closed_shell_charge(method, Z, charge):
    nel = sum(O.element_params(method, z)[1] for z in Z) - charge
    return charge + (int(round(nel)) % 2)


def test_python_binding_h2_energy_and_gradient():
    r = GOLD["python_h2"]
    res = O.scf("PM6", [1, 1], r["xyz_bohr"], rmsd=1e-10, scc=1e-10)
    assert abs(res["energy"] - r["energy_hartree"]) < 0.5 * 10 ** (-r["places"])
    # measured agreement is ~5e-11 Eh: it pins E_h = 27.21138602 eV (CODATA 2014)
    assert abs(res["energy"] - r["energy_hartree"]) < 1e-9
    assert abs(res["gradient"][0, 0] - r["gradient_x_atom0"]) < 1e-9
    assert abs(res["gradient"][1, 0] + r["gradient_x_atom0"]) < 1e-9


def test_local_CO_integral_block():
    r = GOLD["local_CO"]
    kc, ko = r["klopman"]["C"], r["klopman"]["O"]
    c_in, o_in = r["charge_separation_inputs"]["C"], r["charge_separation_inputs"]["O"]
    DC = O.charge_separations(*c_in)
    DO = O.charge_separations(*o_in)
    rhoC = [kc["ss0"], kc["sp1"], kc["pp0"], kc["pp2"]]
    rhoO = [ko["ss0"], ko["sp1"], ko["pp0"], ko["pp2"]]
    L = O.local_block(r["R_bohr"], rhoC, DC, rhoO, DO) * O.ev_per_hartree()
    exp = np.array(r["expected_ev"]).reshape(10, 10)
    assert np.max(np.abs(L - exp)) < r["tol_ev"]


def test_multipole_parameters():
    r = GOLD["multipole_parameters"]
    for c in r["charge_separation"]:
        D = O.charge_separations(c["ns"], c["np"], c["zs"], c["zp"])
        assert abs(D[0] - c["sp1"]) < 1e-8
        assert abs(D[1] - c["pp2_times_sqrt2"] / math.sqrt(2)) < 1e-8
    for k in r["klopman_PM6"]:
        p = O.element_params("PM6", k["Z"])
        assert abs(p[9] - k["ss0"]) < r["tol"]
        if "sp1" in k:
            assert abs(p[10] - k["sp1"]) < r["tol"]
            assert abs(p[11] - k["pp0"]) < r["tol"]
            assert abs(p[12] - k["pp2"]) < r["tol"]


@pytest.mark.parametrize("method", ["PM6", "AM1"])
def test_one_electron_matrices(method):
    ev = O.ev_per_hartree()
    ran = 0
    for r in GOLD["methods"][method]:
        if not _supported(method, r):
            continue
        Z, x = _geometry(r)
        if "one_electron_00_ev" in r:
            H, _ = O.one_electron(method, Z, x)
            v, tol = r["one_electron_00_ev"]
            assert abs(H[0, 0] * ev - v) < tol, r["name"]
            ran += 1
        if "one_electron_ev" in r:
            H, _ = O.one_electron(method, Z, x)
            n = H.shape[0]
            exp = np.array(r["one_electron_ev"]).reshape(n, n)
            # the reference fills the lower triangle only; compare that part
            Hl = np.tril(H) * ev
            El = np.tril(exp)
            # Eigen isApprox: ||a-b|| <= prec * min(||a||, ||b||)
            assert np.linalg.norm(Hl - El) <= r["one_electron_rel_tol"] * min(np.linalg.norm(Hl), np.linalg.norm(El)), \
                r["name"]
            ran += 1
    assert ran >= 4


@pytest.mark.parametrize("method", ["PM6", "AM1"])
def test_energies_against_mopac(method):
    ev = O.ev_per_hartree()
    ran = 0
    for r in GOLD["methods"][method]:
        if r["name"].startswith("DISABLED") or not _supported(method, r):
            continue
        if not any(k in r for k in ("repulsion_ev", "electronic_ev", "total_ev")):
            continue
        Z, x = _geometry(r)
        charge = _closed_shell_charge(method, Z, r["charge"])
        res = O.scf(method, Z, x, charge=charge, gradient=False)
        if "repulsion_ev" in r:
            v, tol = r["repulsion_ev"]
            assert abs(res["e_rep"] * ev - v) < tol, r["name"]
        if charge != r["charge"]:
            continue  # open-shell in the reference: only the repulsion energy is comparable
        assert res["converged"], r["name"]
        if "electronic_ev" in r:
            v, tol = r["electronic_ev"]
            assert abs(res["e_el"] * ev - v) < tol, r["name"]
        if "total_ev" in r:
            v, tol = r["total_ev"]
            assert abs(res["energy"] * ev - v) < tol, r["name"]
        ran += 1
    assert ran >= 5


@pytest.mark.parametrize("method", ["PM6", "AM1"])
def test_methane_gradients_against_mopac(method):
    for r in GOLD["methods"][method]:
        if "gradient_kcal_per_mol_angstrom" not in r:
            continue
        Z, x = _geometry(r)
        res = O.scf(method, Z, x)
        conv = 1.0 / (KCAL_PER_HARTREE * O.bohr_per_angstrom())  # kcal/mol/Angstrom -> Eh/bohr
        exp = np.array(r["gradient_kcal_per_mol_angstrom"]) * conv
        tol = r["gradient_row_norm_tol_hartree_per_bohr"]
        for i in range(len(Z)):
            assert np.linalg.norm(res["gradient"][i] - exp[i]) < tol, (r["name"], i)


@pytest.mark.parametrize("method", ["PM6", "AM1"])
def test_optimised_methane_has_zero_gradient(method):
    for r in GOLD["methods"][method]:
        if "zero_gradient_row_norm_tol" not in r:
            continue
        Z, x = _geometry(r)
        res = O.scf(method, Z, x)
        assert np.all(np.linalg.norm(res["gradient"], axis=1) < r["zero_gradient_row_norm_tol"])


@pytest.mark.parametrize("method", ["PM6", "AM1", "MNDO"])
def test_atom_order_invariance(method):
    # PM6Test.cpp:237-258: water, two atom orders, electronic energy equal to 1e-10
    b = O.bohr_per_angstrom()
    w1 = np.array([[0, 0, 0], [0.4005871485, 0.3100978455, 0], [-0.4005871485, 0.3100978455, 0]]) * b
    r1 = O.scf(method, [8, 1, 1], w1, gradient=False, scc=1e-12, rmsd=1e-11)
    r2 = O.scf(method, [1, 1, 8], w1[[1, 2, 0]], gradient=False, scc=1e-12, rmsd=1e-11)
    assert abs(r1["e_el"] - r2["e_el"]) < 1e-10


@pytest.mark.parametrize("method", ["PM6", "AM1", "MNDO"])
def test_gradient_matches_finite_difference(method):
    # analytic gradient of the converged energy vs central differences (formaldehyde + H2)
    b = O.bohr_per_angstrom()
    Z = [6, 8, 1, 1, 1, 1]
    x = np.array([[0, 0, 0], [0.05, -0.3, 1.2], [-0.53, 0.9, -0.5], [0.9, -0.5, -0.4], [2.5, 1.0, 0.3],
                  [3.1, 1.2, 0.6]]) * b
    res = O.scf(method, Z, x, scc=1e-12, rmsd=1e-11)
    h = 1e-4
    for (i, d) in [(0, 0), (1, 2), (2, 1), (4, 0), (5, 2)]:
        xp = x.copy()
        xm = x.copy()
        xp[i, d] += h
        xm[i, d] -= h
        ep = O.scf(method, Z, xp, gradient=False, scc=1e-12, rmsd=1e-11)["energy"]
        em = O.scf(method, Z, xm, gradient=False, scc=1e-12, rmsd=1e-11)["energy"]
        fd = (ep - em) / (2 * h)
        assert abs(fd - res["gradient"][i, d]) < 1e-6, (i, d, fd, res["gradient"][i, d])


def test_integer_bookkeeping():
    # AO counts and electron counts (PrincipalQuantumNumbers.cpp, NDDOInitializer.cpp:69-81)
    assert O.element_params("PM6", 1)[0] == 1
    assert O.element_params("PM6", 6)[0] == 4
    with pytest.raises(RuntimeError):  # Cl carries d orbitals in PM6: outside the s/p scope
        O.element_params("PM6", 17)
    assert O.element_params("AM1", 17)[0] == 4
    assert O.element_params("PM6", 54)[1] == 6  # rare-gas core charge rule
    res = O.scf("PM6", [8, 1, 1], np.array([[0, 0, 0], [1.8, 0, 0], [-0.45, 1.75, 0]]), gradient=False)
    assert (res["nao"], res["nel"], res["nocc"]) == (6, 8, 4)
