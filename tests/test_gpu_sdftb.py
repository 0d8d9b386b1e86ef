"""Spin-polarised (unrestricted) DFTB2 / DFTB3 on the GPU.

Against the reference's DFTB+ CH3 doublet (src/Sparrow/Tests/MethodsTests/Dftb/
DFTB2Test.cpp:152-207, DFTB3Test.cpp:149-210: energy 1e-8 Hartree,
eigenvalues 1e-6, forces at the reference's per-atom norms) and against the
oracle's spin-polarised SCC on a batch of radicals (energies 1e-6 Hartree,
gradients 1e-5 Hartree/bohr).
"""
import numpy as np
import pytest

import sparrow_b200
from sparrow_b200 import geometry
from tests import oracle_lib as O
from tests.test_sdftb_oracle import CH3, KNOWN

pytestmark = pytest.mark.gpu

E_TOL = 1e-6
G_TOL = 1e-5


@pytest.mark.parametrize("order", [2, 3])
def test_ch3_matches_dftbplus(order):
    k = KNOWN[order]
    c = sparrow_b200.get_calculator("DFTB%d" % order)
    c.set_structure([6, 1, 1, 1], CH3 * O.bohr_per_angstrom())
    c.settings["method_parameters"] = k["parameters"]
    c.settings["spin_multiplicity"] = 2
    c.settings["self_consistence_criterion"] = 1e-12
    c.settings["density_rmsd_criterion"] = 1e-10
    c.settings["max_scf_iterations"] = 500
    c.set_required_properties(["energy", "gradients"])
    r = c.calculate()
    assert r.successful_calculation
    assert abs(r.energy - k["energy"]) < 1e-8
    assert np.max(np.abs(np.sort(c.orbital_energies()) - k["alpha"])) < 1e-6
    assert np.max(np.abs(np.sort(c.beta_orbital_energies()) - k["beta"])) < 1e-6
    for a in range(4):
        assert np.linalg.norm(-r.gradients[a] - k["forces"][a]) < k["force_tol"]


def _radicals():
    b = O.bohr_per_angstrom()
    # (no linear radicals such as OH: the shell-resolved spin shifts keep their
    # beta pi pair exactly degenerate across the Fermi level, so no aufbau state
    # is self-consistent and neither the oracle nor the engine converges)
    out = [([6, 8, 1, 1, 1], np.array([[0, 0, 0], [1.37, 0, 0], [1.70, 0.90, 0], [-0.55, 0.93, 0.10],
                                       [-0.55, -0.93, 0.10]]) * b, 0, 2),                             # CH2OH
           ([6, 1, 1, 1], CH3 * b + 0.02, 0, 2),
           ([6, 1, 1], np.array([[0, 0, 0], [0, 0.99, 0.62], [0, -0.99, 0.62]]) * b, 0, 3),
           ([7, 1, 1], np.array([[0, 0, 0], [0, 0.8, 0.62], [0, -0.8, 0.62]]) * b, 0, 2),
           ([8, 1, 1], np.array([[0, 0, 0], [0, 0.79, 0.6], [0, -0.79, 0.6]]) * b, 1, 2),
           ([8, 1, 1], np.array([[0, 0, 0], [0, 0.76, 0.59], [0, -0.76, 0.59]]) * b, 0, 1)]
    for z, x in geometry.alkane_batch(3, seed=41, n_min=3, n_max=7):
        out.append((np.asarray(z)[:-1], geometry.to_bohr(x)[:-1], 0, 2))
    return out


@pytest.mark.parametrize("order", [2, 3])
def test_radical_batch_matches_oracle(order):
    mols = _radicals()
    b = sparrow_b200.Batch("DFTB%d" % order, [(z, x) for z, x, _, _ in mols], charges=[c for _, _, c, _ in mols],
                           multiplicities=[m for _, _, _, m in mols], scc=1e-11, rmsd=1e-9, max_iter=500)
    b.run(gradients=True)
    e, g, _, conv = b.results()
    assert conv.all()
    for i, (Z, x, ch, mult) in enumerate(mols):
        ref = O.dftb_scf_uhf(order, Z, x, mult, charge=ch, scc=1e-11, rmsd=1e-9)
        assert ref["converged"]
        assert abs(e[i] - ref["energy"]) < E_TOL, (order, i)
        assert np.max(np.abs(g[i] - ref["gradient"])) < G_TOL, (order, i)


def test_unrestricted_singlets_equal_restricted():
    mols = [(z, geometry.to_bohr(x)) for z, x in geometry.polyene_batch(4, seed=3, k_min=3, k_max=8)]
    r = sparrow_b200.Batch("DFTB3", mols, scc=1e-11, rmsd=1e-9)
    r.run(gradients=True)
    u = sparrow_b200.Batch("DFTB3", mols, scc=1e-11, rmsd=1e-9, unrestricted=True)
    u.run(gradients=True)
    er, gr, _, cr = r.results()
    eu, gu, _, cu = u.results()
    assert cr.all() and cu.all()
    assert np.max(np.abs(er - eu)) < 1e-8
    assert max(np.max(np.abs(a - c)) for a, c in zip(gr, gu)) < 1e-7
