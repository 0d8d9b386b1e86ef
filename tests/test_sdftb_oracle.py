"""The oracle's spin-polarised DFTB against the reference's DFTB+ known answers.

CH3 doublet (src/Sparrow/Tests/MethodsTests/Dftb/DFTB2Test.cpp:152-207,
mio-1-1; DFTB3Test.cpp:149-210, 3ob-2-1): energy at 1e-8 Hartree, Mulliken
charges and alpha / beta eigenvalues at 1e-6, forces at the reference's
per-atom norms (1e-5 DFTB2, 1e-4 DFTB3).  Plus: the DFTB2 gradient is the
derivative of the energy, and a closed-shell singlet gives the restricted
result.
"""
import numpy as np
import pytest

from tests import oracle_lib as O

CH3 = np.array([[0, 0, 0], [0.6287, 0.6287, 0.6287], [-0.6287, -0.6287, 0.6287], [-0.6287, 0.6287, -0.6287]])

KNOWN = {
    2: dict(parameters="mio-1-1", energy=-2.7458925732, force_tol=1e-5,
            charges=[-0.29151134, 0.09717045, 0.09717045, 0.09717045],
            alpha=[-0.58373525, -0.35004087, -0.35004087, -0.23077050, 0.33809319, 0.33809319, 0.51658701],
            beta=[-0.54684410, -0.32740014, -0.32740014, -0.18248896, 0.36091443, 0.36091443, 0.53408108],
            forces=[[-1.738173073648139E-002, 1.738173073648139E-002, 1.738173073648149E-002],
                    [1.136823505565547E-002, -3.006747840412945E-003, -3.006747840413014E-003],
                    [3.006747840413014E-003, -1.136823505565546E-002, -3.006747840412952E-003],
                    [3.006747840412931E-003, -3.006747840412986E-003, -1.136823505565552E-002]]),
    3: dict(parameters="3ob-2-1", energy=-2.7511893552, force_tol=1e-4,
            charges=[-0.36104148, 0.12034716, 0.12034716, 0.12034716],
            alpha=[-0.58235936, -0.34523459, -0.34523459, -0.23770995, 0.35065029, 0.35065029, 0.55071179],
            beta=[-0.54429011, -0.32206695, -0.32206695, -0.18935792, 0.37291251, 0.37291251, 0.56720722],
            forces=[[-1.929194902027242E-002, 1.929194902027246E-002, 1.929194902027252E-002],
                    [8.281673212401919E-003, -5.505137903935295E-003, -5.505137903935246E-003],
                    [5.505137903935246E-003, -8.281673212401953E-003, -5.505137903935316E-003],
                    [5.505137903935246E-003, -5.505137903935239E-003, -8.281673212401933E-003]]),
}


@pytest.mark.parametrize("order", [2, 3])
def test_ch3_matches_dftbplus(order):
    k = KNOWN[order]
    r = O.dftb_scf_uhf(order, [6, 1, 1, 1], CH3 * O.bohr_per_angstrom(), 2, parameters=k["parameters"], scc=1e-12,
                       rmsd=1e-10)
    assert r["converged"] and (r["n_alpha"], r["n_beta"]) == (4, 3)
    assert abs(r["energy"] - k["energy"]) < 1e-8
    assert np.max(np.abs(r["charges"] - k["charges"])) < 1e-6
    assert np.max(np.abs(r["eps_alpha"] - k["alpha"])) < 1e-6
    assert np.max(np.abs(r["eps_beta"] - k["beta"])) < 1e-6
    for a in range(4):
        assert np.linalg.norm(-r["gradient"][a] - k["forces"][a]) < k["force_tol"]


def test_dftb2_spin_gradient_is_the_energy_derivative():
    x = CH3 * O.bohr_per_angstrom() + np.array([[0, 0, 0.05], [0.02, 0, 0], [0, -0.03, 0], [0, 0, 0]])
    r = O.dftb_scf_uhf(2, [6, 1, 1, 1], x, 2, scc=1e-12, rmsd=1e-10)
    h = 1e-4
    for a in range(4):
        for d in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, d] += h
            xm[a, d] -= h
            ep = O.dftb_scf_uhf(2, [6, 1, 1, 1], xp, 2, scc=1e-12, rmsd=1e-10, gradient=False)["energy"]
            em = O.dftb_scf_uhf(2, [6, 1, 1, 1], xm, 2, scc=1e-12, rmsd=1e-10, gradient=False)["energy"]
            assert abs((ep - em) / (2 * h) - r["gradient"][a, d]) < 1e-7


@pytest.mark.parametrize("order", [2, 3])
def test_closed_shell_singlet_is_restricted(order):
    x = np.array([[0, 0, 0], [0, 1.43, 1.1], [0, -1.43, 1.1]])
    u = O.dftb_scf_uhf(order, [8, 1, 1], x, 1, scc=1e-12, rmsd=1e-10)
    r = O.dftb_scf(order, [8, 1, 1], x, scc=1e-12, rmsd=1e-10)
    assert abs(u["energy"] - r["energy"]) < 1e-10 and abs(u["e_spin"]) < 1e-12
    assert np.max(np.abs(u["gradient"] - r["gradient"])) < 1e-8
