"""Semi-numerical Hessian of the oracle against the reference's frequencies.

The reference's Hessian is the symmetrised central difference of analytic
gradients (Utils::NumericalHessianCalculator, step 0.01 bohr); its app tests
assert harmonic frequencies (tests/golden/hessian_known_answers.json).  The
oracle's gradients with the same differences reproduce them: sft_1 within
0.02 cm^-1 for MNDO, AM1, PM6, DFTB2 and DFTB3; ethane within 0.1 cm^-1 (the
asserted 2788.55 is rounded from the reference's own run, whose SCF settings
are its app defaults).
"""
import json
import os

import numpy as np
import pytest

from tests import harmonic
from tests import oracle_lib as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "hessian_known_answers.json")))
SYM = {"H": 1, "C": 6, "N": 7, "O": 8}
STEP = 0.01


def structure(name):
    s = GOLD["structures"][name]
    return [SYM[e] for e in s["elements"]], np.array(s["xyz_angstrom"]) * O.bohr_per_angstrom()


def oracle_gradient(method, Z, x):
    if method.startswith("DFTB"):
        return O.dftb_scf(int(method[-1]), Z, x, scc=1e-10, rmsd=1e-10)["gradient"].reshape(-1)
    return O.scf(method, Z, x, scc=1e-10, rmsd=1e-10)["gradient"].reshape(-1)


def oracle_hessian(method, Z, x, step=STEP):
    n3 = 3 * len(Z)
    H = np.zeros((n3, n3))
    for k in range(n3):
        xp, xm = x.copy().reshape(-1), x.copy().reshape(-1)
        xp[k] += step
        xm[k] -= step
        H[k] = (oracle_gradient(method, Z, xp.reshape(-1, 3)) - oracle_gradient(method, Z, xm.reshape(-1, 3))) / (2 * step)
    return 0.5 * (H + H.T)


@pytest.mark.parametrize("case", GOLD["cases"], ids=lambda c: c["structure"] + "-" + c["method"])
def test_oracle_frequencies_match_the_reference(case):
    Z, x = structure(case["structure"])
    f = harmonic.frequencies(Z, x, oracle_hessian(case["method"], Z, x))
    tol = 0.1 if case["structure"] == "ethane_opt" else 0.02
    assert abs(f[case["index"]] - case["frequency"]) < tol, (case, f[:4])
