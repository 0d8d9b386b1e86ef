"""Unrestricted (UHF) NDDO SCF on the GPU against the oracle and the reference's known answers.

Tolerances: energies 1e-6 Hartree and gradients 1e-5 Hartree/bohr against the
oracle's unrestricted SCF; the reference's MOPAC doublet atoms at its own
1e-5 eV (src/Sparrow/Tests/MethodsTests/Pm6/PM6Test.cpp:211-234,
Am1/AM1Test.cpp:193-216, Mndo/MNDOTest.cpp:187-210).
"""
import numpy as np
import pytest

import sparrow_b200
from sparrow_b200 import geometry
from tests import oracle_lib as O
from tests import param_sets as PS

E_TOL = 1e-6
G_TOL = 1e-5
ATOM = np.array([[-0.1058354421, 0.1058354421, -0.1587531632]])


def _radicals():
    """(Z, xyz bohr, charge, multiplicity) of small open- and closed-shell species."""
    b = O.bohr_per_angstrom()
    out = [
        ([8, 1], np.array([[0, 0, 0], [0.05, 0.1, 0.97]]) * b, 0, 2),                                # OH
        ([6, 1, 1, 1], np.array([[0, 0, 0], [1.08, 0, 0.02], [-0.54, 0.935, -0.03],
                                 [-0.54, -0.935, 0.01]]) * b, 0, 2),                                  # CH3
        ([6, 1, 1], np.array([[0, 0, 0], [0, 0.99, 0.62], [0, -0.99, 0.62]]) * b, 0, 3),            # CH2 triplet
        ([8, 8], np.array([[0, 0, 0], [0.02, 0, 1.21]]) * b, 0, 3),                                  # O2 triplet
        ([7, 1, 1], np.array([[0, 0, 0], [0, 0.8, 0.62], [0, -0.8, 0.62]]) * b, 0, 2),              # NH2
        ([8, 1, 1], np.array([[0, 0, 0], [0, 0.79, 0.6], [0, -0.79, 0.6]]) * b, 1, 2),              # H2O+
        ([8, 1, 1], np.array([[0, 0, 0], [0, 0.76, 0.59], [0, -0.76, 0.59]]) * b, 0, 1),            # H2O singlet
    ]
    # larger doublets: alkyl radicals (an alkane without its last hydrogen)
    for z, x in geometry.alkane_batch(3, seed=31, n_min=4, n_max=9):
        out.append((np.asarray(z)[:-1], geometry.to_bohr(x)[:-1], 0, 2))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("method,Z,energy,alpha,beta", [
    ("PM6", 5, -49.53668, [-11.74716, -5.78067, -0.09376, -0.09376], [-10.49432, 0.62041, 0.62041, 2.04873]),
    ("AM1", 3, -4.93844, [-4.93844, 5.45631, 5.45631, 5.45631], [0.46149, 5.85628, 5.85628, 5.85628]),
    ("MNDO", 5, -64.31595, [-16.20713, -5.81169, 1.54831, 1.54831], [-14.39713, 2.04831, 2.04831, 3.04831]),
])
def test_doublet_atoms_match_mopac(method, Z, energy, alpha, beta):
    ev = O.ev_per_hartree()
    c = sparrow_b200.get_calculator(method)
    c.set_structure([Z], ATOM * O.bohr_per_angstrom())
    c.settings["spin_multiplicity"] = 2            # spin_mode "any": unrestricted
    c.settings["density_rmsd_criterion"] = 1e-9
    c.settings["self_consistence_criterion"] = 1e-10
    res = c.calculate()
    assert res.successful_calculation
    assert abs(res.energy * ev - energy) < 1e-5
    assert np.max(np.abs(np.sort(c.orbital_energies()) * ev - alpha)) < 1e-5
    assert np.max(np.abs(np.sort(c.beta_orbital_energies()) * ev - beta)) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["PM6", "AM1", "MNDO"])
def test_radical_batch_matches_oracle(method):
    mols = _radicals()
    b = sparrow_b200.Batch(method, [(z, x) for z, x, _, _ in mols], charges=[c for _, _, c, _ in mols],
                           multiplicities=[m for _, _, _, m in mols], scc=1e-10, rmsd=1e-9, max_iter=500)
    assert b.unrestricted
    b.run(gradients=True)
    e, g, it, conv = b.results()
    assert conv.all()
    for i, (Z, x, ch, mult) in enumerate(mols):
        ref = O.scf_uhf(method, Z, x, mult, charge=ch)
        assert ref["converged"]
        assert abs(e[i] - ref["energy"]) < E_TOL, (method, i)
        assert np.max(np.abs(g[i] - ref["gradient"])) < G_TOL, (method, i)


@pytest.mark.gpu
def test_unrestricted_singlets_equal_restricted():
    mols = [(z, geometry.to_bohr(x)) for z, x in geometry.alkane_batch(6, seed=8, n_min=2, n_max=12)]
    Z, xa = geometry.water_cluster(6, seed=1)
    mols.append((Z, geometry.to_bohr(xa)))
    r = sparrow_b200.Batch("PM6", mols, scc=1e-10, rmsd=1e-9)
    r.run(gradients=True)
    u = sparrow_b200.Batch("PM6", mols, scc=1e-10, rmsd=1e-9, unrestricted=True)
    u.run(gradients=True)
    er, gr, _, cr = r.results()
    eu, gu, _, cu = u.results()
    assert cr.all() and cu.all()
    assert np.max(np.abs(er - eu)) < 1e-8
    assert max(np.max(np.abs(a - c)) for a, c in zip(gr, gu)) < 1e-7


@pytest.mark.gpu
def test_calculator_spin_modes():
    Z, x, _, _ = _radicals()[0]  # OH
    c = sparrow_b200.get_calculator("PM6")
    c.set_structure(Z, x)
    c.set_required_properties(["energy", "gradients"])
    c.settings["density_rmsd_criterion"] = 1e-9
    c.settings["spin_multiplicity"] = 2
    c.settings["spin_mode"] = "restricted"
    with pytest.raises(sparrow_b200.SparrowError):
        c.calculate()
    c.settings["spin_mode"] = "unrestricted"
    r = c.calculate()
    ref = O.scf_uhf("PM6", Z, x, 2)
    assert r.successful_calculation and abs(r.energy - ref["energy"]) < E_TOL
    assert np.max(np.abs(r.gradients - ref["gradient"])) < G_TOL
    # a restricted closed-shell run has no beta orbital energies
    w, xw = _radicals()[6][:2]
    c.set_structure(w, xw)
    c.settings["spin_multiplicity"] = 1
    c.settings["spin_mode"] = "any"
    assert c.calculate().successful_calculation
    with pytest.raises(sparrow_b200.SparrowError):
        c.beta_orbital_energies()


def test_unrestricted_batches_are_checked_on_the_host(tmp_path):
    oh = [(np.array([8, 1]), np.array([[0, 0, 0], [0, 0, 1.84]]))]
    with pytest.raises(sparrow_b200.SparrowError) as ei:   # 7 electrons cannot be a triplet
        sparrow_b200.Batch("PM6", oh, multiplicities=[3])
    assert ei.value.code == 5
    with pytest.raises(sparrow_b200.SparrowError) as ei:   # nor a restricted singlet
        sparrow_b200.Batch("PM6", oh)
    assert ei.value.code == 5
    with pytest.raises(ValueError):
        sparrow_b200.Batch("PM6", oh, multiplicities=[2], unrestricted=False)
    with pytest.raises(sparrow_b200.SparrowError) as ei:   # spin-polarised DFTB needs spin constants
        d = tmp_path / "no-spin"
        PS.write_skf_directory(str(d), "mio-1-1", spin=False)
        sparrow_b200.Batch("DFTB2:" + str(d), oh, multiplicities=[2])
    assert ei.value.code == 3 and "spin constants" in str(ei.value)


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["PM6", "AM1", "MNDO"])
def test_edge_occupations(method):
    # H atom (no beta electron), N atom quartet (alpha shell full), NH3+ doublet
    # (ionised from the non-degenerate lone pair; a Jahn-Teller radical such as
    # tetrahedral CH4+ has several broken-symmetry UHF solutions, so two
    # solvers may rightly land on different ones)
    b = O.bohr_per_angstrom()
    cases = [([1], ATOM * b, 0, 2), ([7], ATOM * b, 0, 4),
             ([7, 1, 1, 1], np.array([[0, 0, 0], [0.94, 0, 0.38], [-0.47, 0.814, 0.38], [-0.47, -0.814, 0.38]]) * b,
              1, 2)]
    for Z, x, ch, mult in cases:
        c = sparrow_b200.get_calculator(method)
        c.set_structure(Z, x)
        c.settings["molecular_charge"] = ch
        c.settings["spin_multiplicity"] = mult
        c.settings["density_rmsd_criterion"] = 1e-9
        c.settings["self_consistence_criterion"] = 1e-10
        c.settings["max_scf_iterations"] = 500
        c.set_required_properties(["energy", "gradients"])
        r = c.calculate()
        ref = O.scf_uhf(method, Z, x, mult, charge=ch, scc=1e-10, rmsd=1e-9)
        assert r.successful_calculation and ref["converged"], (method, Z)
        assert abs(r.energy - ref["energy"]) < E_TOL, (method, Z)
        assert np.max(np.abs(r.gradients - ref["gradient"])) < G_TOL, (method, Z)
        assert np.max(np.abs(np.sort(c.orbital_energies()) - ref["eps_alpha"])) < 1e-6
        assert np.max(np.abs(np.sort(c.beta_orbital_energies()) - ref["eps_beta"])) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["PM6", "DFTB2"])
def test_spin_density_warm_start(method):
    # getState / loadState of an open shell: a restart from the converged spin
    # densities is converged at once, with the same energy
    Z, x, _, _ = _radicals()[1]  # CH3
    c = sparrow_b200.get_calculator(method)
    c.set_structure(Z, x)
    c.settings["spin_multiplicity"] = 2
    c.settings["density_rmsd_criterion"] = 1e-9
    c.settings["self_consistence_criterion"] = 1e-10
    r1 = c.calculate()
    Pa, Pb = c.spin_densities()
    if method == "PM6":  # orthonormal basis: the traces count the electrons of each spin
        assert abs(np.trace(Pa) - 4) < 1e-9 and abs(np.trace(Pb) - 3) < 1e-9
    assert np.max(np.abs(Pa + Pb - c.density())) < 1e-12
    c.set_spin_densities(Pa, Pb)
    r2 = c.calculate()
    assert r1.successful_calculation and r2.successful_calculation
    assert r2.iterations <= 3 < r1.iterations
    assert abs(r1.energy - r2.energy) < 1e-9
