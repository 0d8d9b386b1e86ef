"""Large-molecule SCF path: one NDDO molecule over the whole GPU.

The path (grid-wide Fock build, DIIS on FP64 GEMMs, SP2 purification) must
give the same converged state as the oracle and as the batched kernel:
total energy within 1e-6 Hartree, gradient within 1e-5 Hartree/bohr.  The
mixed-precision form (split-BF16 purification products until rms(dP) < 1e-5,
then FP64) must land on the FP64 result within the same energy tolerance.
"""
import numpy as np
import pytest

import sparrow_b200
from sparrow_b200 import geometry
from tests import oracle_lib as O

pytestmark = pytest.mark.gpu

E_TOL = 1e-6
G_TOL = 1e-5


def run_one(method, Z, x, path, rmsd=1e-8, gradients=True, max_iter=200):
    b = sparrow_b200.Batch(method, [(Z, x)], rmsd=rmsd, max_iter=max_iter, scf_path=path)
    b.run(gradients=gradients)
    e, g, it, conv = b.results()
    return b, e[0], (g[0] if g is not None else None), int(it[0]), bool(conv[0])


@pytest.mark.parametrize("path", ["large", "large_mixed"])
@pytest.mark.parametrize("method", ["PM6", "AM1", "MNDO"])
def test_small_cluster_matches_oracle(method, path):
    Z, xa = geometry.water_cluster(8, seed=4)
    x = geometry.to_bohr(xa)
    _, e, g, it, conv = run_one(method, Z, x, path)
    ref = O.scf(method, Z, x)
    assert conv and ref["converged"]
    assert abs(e - ref["energy"]) < E_TOL
    assert np.max(np.abs(g - ref["gradient"])) < G_TOL


@pytest.mark.parametrize("path", ["large", "large_mixed"])
def test_water32_matches_oracle(path):
    Z, xa = geometry.water_cluster(32, seed=0)
    x = geometry.to_bohr(xa)
    _, e, g, it, conv = run_one("PM6", Z, x, path)
    ref = O.scf("PM6", Z, x)
    assert conv
    assert abs(e - ref["energy"]) < E_TOL
    assert np.max(np.abs(g - ref["gradient"])) < G_TOL


def test_large_path_equals_batched_kernel():
    # 960 AOs: the largest size class both paths take
    Z, xa = geometry.water_cluster(160, seed=2)
    x = geometry.to_bohr(xa)
    _, e_b, g_b, _, conv_b = run_one("PM6", Z, x, "batched")
    _, e_l, g_l, _, conv_l = run_one("PM6", Z, x, "large")
    assert conv_b and conv_l
    assert abs(e_b - e_l) < E_TOL
    assert np.max(np.abs(g_b - g_l)) < G_TOL


def test_mixed_precision_water256():
    # (H2O)_256, 1536 AOs: mixed-precision purification against FP64
    Z, xa = geometry.water_cluster(256, seed=0)
    x = geometry.to_bohr(xa)
    b64, e64, _, it64, c64 = run_one("PM6", Z, x, "large", gradients=False)
    bmx, emx, _, itmx, cmx = run_one("PM6", Z, x, "large_mixed", gradients=False)
    assert c64 and cmx
    assert abs(e64 - emx) < E_TOL
    nmixed, nsteps, _ = bmx.scf_stats()
    assert nmixed[0] >= 1 and nsteps[0] > 0
    assert b64.scf_stats()[0][0] == 0


def test_calculator_takes_large_path_above_1024_aos():
    Z, xa = geometry.water_cluster(176, seed=3)  # 1056 AOs
    x = geometry.to_bohr(xa)
    c = sparrow_b200.get_calculator("PM6")
    c.set_structure(Z, x)
    c.settings["density_rmsd_criterion"] = 1e-8
    c.set_required_properties(["energy"])
    res = c.calculate()
    assert res.successful_calculation and res.n_aos == 1056
    _, e, _, _, conv = run_one("PM6", Z, x, "large", gradients=False)
    assert conv and abs(res.energy - e) < 1e-9
    # density purification: no orbitals, so no orbital energies
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        c.orbital_energies()
    assert ei.value.code == 9


def test_large_path_rejects_batches_and_dftb():
    mols = [(np.array([1, 1]), np.array([[0, 0, 0], [0, 0, 1.4]], float))] * 2
    with pytest.raises(sparrow_b200.SparrowError):
        sparrow_b200.Batch("PM6", mols, scf_path="large")
    with pytest.raises(sparrow_b200.SparrowError):
        sparrow_b200.Batch("DFTB2", mols[:1], scf_path="large")
    with pytest.raises(ValueError):
        sparrow_b200.Batch("PM6", mols[:1], scf_path="fast")


def _fixtures():
    import glob
    import os
    return sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "large_water_pm6_*.json")))


@pytest.mark.parametrize("fixture", _fixtures())
def test_large_clusters_match_oracle_fixture(fixture):
    # the oracle's converged (H2O)_256 / (H2O)_512 PM6 energies and gradients
    # (tests/golden/make_large_water_golden.py), FP64 and mixed-precision paths.
    # The oracle sums its energy with compensated summation, so the fixtures
    # hold the energy to ~1e-11 Hartree and the check can be 1e-8.
    import json
    gold = json.load(open(fixture))
    Z, xa = geometry.water_cluster(gold["waters"], seed=gold["seed"])
    x = geometry.to_bohr(xa)
    for path in ("large", "large_mixed"):
        _, e, g, it, conv = run_one("PM6", Z, x, path)
        assert conv
        assert abs(e - gold["energy"]) < 1e-8, path
        assert np.max(np.abs(g.reshape(-1) - np.array(gold["gradient"]))) < G_TOL, path
