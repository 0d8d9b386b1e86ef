"""Elements beyond H, C, N, O on the GPU: every s/p element the methods
parameterise is accepted (Li, Be, B, F, Na, Mg here); batches of small
molecules with them match the oracle within 1e-6 Hartree and 1e-5
Hartree/bohr, and an element a method has no parameters for (boron under
AM1) is rejected with SG_ERR_UNSUPPORTED_ELEMENT by the engine as by the
oracle."""
import numpy as np
import pytest

import sparrow_b200
from tests import oracle_lib as O

E_TOL = 1e-6
G_TOL = 1e-5
MOLS = {
    "HF": ([9, 1], [[0, 0, 0], [0, 0, 0.92]]),
    "CF4": ([6, 9, 9, 9, 9], [[0, 0, 0], [0.77, 0.77, 0.77], [-0.77, -0.77, 0.77], [-0.77, 0.77, -0.77],
                              [0.77, -0.77, -0.77]]),
    "BH3": ([5, 1, 1, 1], [[0, 0, 0], [1.19, 0, 0], [-0.595, 1.03, 0], [-0.595, -1.03, 0]]),
    "BF3": ([5, 9, 9, 9], [[0, 0, 0], [1.31, 0, 0], [-0.655, 1.134, 0], [-0.655, -1.134, 0]]),
    "LiH": ([3, 1], [[0, 0, 0], [0, 0, 1.6]]),
    "LiF": ([3, 9], [[0, 0, 0], [0, 0, 1.56]]),
    "BeH2": ([4, 1, 1], [[0, 0, 0], [0, 0, 1.33], [0, 0, -1.33]]),
    "NaH": ([11, 1], [[0, 0, 0], [0, 0, 1.89]]),
    "MgH2": ([12, 1, 1], [[0, 0, 0], [0, 0, 1.7], [0, 0, -1.7]]),
    "CH3F": ([6, 9, 1, 1, 1], [[0, 0, 0], [1.38, 0, 0], [-0.36, 1.03, 0], [-0.36, -0.51, 0.89],
                               [-0.36, -0.51, -0.89]]),
}


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["PM6", "AM1", "MNDO"])
def test_light_elements_match_oracle(method):
    mols = []
    for name, (Z, x) in MOLS.items():
        x = np.array(x) * O.bohr_per_angstrom()
        try:
            ref = O.scf(method, Z, x, scc=1e-10, rmsd=1e-9)
        except RuntimeError:
            with pytest.raises(sparrow_b200.SparrowError) as ei:
                sparrow_b200.Batch(method, [(Z, x)])
            assert ei.value.code == 3, name
            continue
        mols.append((name, Z, x, ref))
    assert len(mols) >= 8
    b = sparrow_b200.Batch(method, [(Z, x) for _, Z, x, _ in mols], scc=1e-10, rmsd=1e-9, max_iter=300)
    b.run(gradients=True)
    e, g, _, conv = b.results()
    assert conv.all()
    for i, (name, Z, x, ref) in enumerate(mols):
        assert ref["converged"], name
        assert abs(e[i] - ref["energy"]) < E_TOL, (method, name)
        assert np.max(np.abs(g[i] - ref["gradient"])) < G_TOL, (method, name)
