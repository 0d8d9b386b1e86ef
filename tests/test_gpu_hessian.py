"""Semi-numerical Hessian on the GPU (6 n_atoms displaced geometries per batch).

Against the oracle's Hessian built from the same central differences: 1e-5
Hartree/bohr^2 (the gradients agree to well below 1e-5 Hartree/bohr, and the
difference quotient divides their error by 0.02 bohr).  Against the
reference's frequencies (tests/golden/hessian_known_answers.json) at the
tolerances of the oracle's test.
"""
import numpy as np
import pytest

import sparrow_b200
from tests import harmonic
from tests import oracle_lib as O
from tests.test_hessian_oracle import GOLD, oracle_hessian, structure

H_TOL = 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLD["cases"], ids=lambda c: c["structure"] + "-" + c["method"])
def test_gpu_hessian_matches_oracle_and_reference(case):
    Z, x = structure(case["structure"])
    H, nc = sparrow_b200.hessian(case["method"], Z, x, scc=1e-10, rmsd=1e-10, max_iter=500)
    assert nc == 0
    assert np.max(np.abs(H - H.T)) == 0.0
    if case["structure"] == "sft_1" and case["method"] in ("PM6", "DFTB3"):
        assert np.max(np.abs(H - oracle_hessian(case["method"], Z, x))) < H_TOL
    f = harmonic.frequencies(Z, x, H)
    tol = 0.1 if case["structure"] == "ethane_opt" else 0.02
    assert abs(f[case["index"]] - case["frequency"]) < tol, (case, f[:4])


@pytest.mark.gpu
def test_calculator_hessian_property():
    Z, x = structure("ethane_opt")
    c = sparrow_b200.get_calculator("AM1")
    c.set_structure(Z, x)
    c.settings["self_consistence_criterion"] = 1e-10
    c.settings["density_rmsd_criterion"] = 1e-10
    c.set_required_properties(["energy", "gradients", "hessian"])
    r = c.calculate()
    assert r.successful_calculation and r.hessian.shape == (18, 18)
    H, _ = sparrow_b200.hessian("AM1", Z, x, scc=1e-10, rmsd=1e-10)
    assert np.max(np.abs(r.hessian - H)) < 1e-9
    assert np.max(np.abs(H - oracle_hessian("AM1", Z, x))) < H_TOL


@pytest.mark.gpu
def test_unrestricted_hessian_matches_oracle():
    Z = [8, 1]
    x = np.array([[0, 0, 0], [0.1, 0.2, 1.85]])
    H, nc = sparrow_b200.hessian("PM6", Z, x, multiplicity=2, scc=1e-11, rmsd=1e-10, max_iter=500)
    assert nc == 0
    ref = np.zeros((6, 6))
    for k in range(6):
        xp, xm = x.copy().reshape(-1), x.copy().reshape(-1)
        xp[k] += 0.01
        xm[k] -= 0.01
        gp = O.scf_uhf("PM6", Z, xp.reshape(-1, 3), 2, scc=1e-11, rmsd=1e-10)["gradient"].reshape(-1)
        gm = O.scf_uhf("PM6", Z, xm.reshape(-1, 3), 2, scc=1e-11, rmsd=1e-10)["gradient"].reshape(-1)
        ref[k] = (gp - gm) / 0.02
    ref = 0.5 * (ref + ref.T)
    assert np.max(np.abs(H - ref)) < H_TOL


def test_hessian_arguments_are_checked_on_the_host():
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.hessian("PM6", [], np.zeros((0, 3)))
    assert ei.value.code == 4
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.hessian("XTB", [1, 1], np.array([[0, 0, 0], [0, 0, 1.4]]))
    assert ei.value.code == 2
    with pytest.raises(sparrow_b200.SparrowError) as ei:  # OH is a doublet
        sparrow_b200.hessian("PM6", [8, 1], np.array([[0, 0, 0], [0, 0, 1.8]]))
    assert ei.value.code == 5
