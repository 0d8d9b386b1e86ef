"""The oracle's unrestricted (UHF) NDDO SCF against the reference's known answers.

Known answers (MOPAC values asserted by the reference's own tests):
- PM6 boron doublet: energy and alpha / beta eigenvalues at 1e-5 eV
  (src/Sparrow/Tests/MethodsTests/Pm6/PM6Test.cpp:211-234);
- AM1 lithium doublet (Tests/MethodsTests/Am1/AM1Test.cpp:193-216);
- MNDO boron doublet (Tests/MethodsTests/Mndo/MNDOTest.cpp:187-210);
- the CH radical's repulsion energy, 1e-4 eV (PM6Test.cpp:349-361,
  AM1Test.cpp:282-295, MNDOTest.cpp:277-290).
Plus two properties: UHF of a closed-shell singlet is the restricted result,
and the UHF gradient is the derivative of the UHF energy (central differences).
"""
import numpy as np
import pytest

from tests import oracle_lib as O

ATOM = np.array([[-0.1058354421, 0.1058354421, -0.1587531632]])


@pytest.mark.parametrize("method,Z,energy,alpha,beta", [
    ("PM6", 5, -49.53668, [-11.74716, -5.78067, -0.09376, -0.09376], [-10.49432, 0.62041, 0.62041, 2.04873]),
    ("AM1", 3, -4.93844, [-4.93844, 5.45631, 5.45631, 5.45631], [0.46149, 5.85628, 5.85628, 5.85628]),
    ("MNDO", 5, -64.31595, [-16.20713, -5.81169, 1.54831, 1.54831], [-14.39713, 2.04831, 2.04831, 3.04831]),
])
def test_doublet_atoms_match_mopac(method, Z, energy, alpha, beta):
    ev = O.ev_per_hartree()
    r = O.scf_uhf(method, [Z], ATOM * O.bohr_per_angstrom(), 2)
    assert r["converged"] and r["n_alpha"] - r["n_beta"] == 1
    assert abs(r["energy"] * ev - energy) < 1e-5
    assert np.max(np.abs(r["eps_alpha"] * ev - alpha)) < 1e-5
    assert np.max(np.abs(r["eps_beta"] * ev - beta)) < 1e-5


@pytest.mark.parametrize("method,erep", [("PM6", 25.82052), ("AM1", 25.20936), ("MNDO", 25.27860)])
def test_ch_radical_repulsion(method, erep):
    x = np.array([[0, 0, 0], [2.0, 0, 0]]) * O.bohr_per_angstrom()
    r = O.scf_uhf(method, [6, 1], x, 2, max_iter=300)
    assert r["converged"]
    assert abs(r["e_rep"] * O.ev_per_hartree() - erep) < 1e-4


def test_closed_shell_uhf_is_restricted():
    x = np.array([[0, 0, 0], [0, 1.43, 1.1], [0, -1.43, 1.1]])
    ru = O.scf_uhf("PM6", [8, 1, 1], x, 1)
    rr = O.scf("PM6", [8, 1, 1], x)
    assert abs(ru["energy"] - rr["energy"]) < 1e-10
    assert np.max(np.abs(ru["gradient"] - rr["gradient"])) < 1e-8


@pytest.mark.parametrize("method", ["PM6", "AM1", "MNDO"])
def test_uhf_gradient_is_the_energy_derivative(method):
    # OH radical and the CH2 triplet
    for Z, x, mult in [([8, 1], np.array([[0, 0, 0], [0.1, 0.2, 1.85]]), 2),
                       ([6, 1, 1], np.array([[0, 0, 0], [0, 1.6, 1.1], [0, -1.6, 1.1]]), 3)]:
        r = O.scf_uhf(method, Z, x, mult, scc=1e-12, rmsd=1e-11)
        assert r["converged"]
        h = 1e-4
        for a in range(len(Z)):
            for d in range(3):
                xp, xm = x.copy(), x.copy()
                xp[a, d] += h
                xm[a, d] -= h
                ep = O.scf_uhf(method, Z, xp, mult, scc=1e-12, rmsd=1e-11, gradient=False)["energy"]
                em = O.scf_uhf(method, Z, xm, mult, scc=1e-12, rmsd=1e-11, gradient=False)["energy"]
                assert abs((ep - em) / (2 * h) - r["gradient"][a, d]) < 2e-6, (method, Z, a, d)


def test_multiplicity_must_match_the_electron_count():
    with pytest.raises(RuntimeError):
        O.scf_uhf("PM6", [8, 1, 1], np.array([[0, 0, 0], [0, 1.43, 1.1], [0, -1.43, 1.1]]), 2)
