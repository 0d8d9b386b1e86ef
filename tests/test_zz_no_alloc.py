"""Allocation-free entry point sg_calculate_static against the batched engine.

The file is collected last on purpose: the static-scratch call must give the
same results after every other test has used the device, and alone in a fresh
process.
"""
import numpy as np
import pytest

import sparrow_b200
from sparrow_b200 import geometry

E_TOL = 1e-6   # Hartree
G_TOL = 1e-5   # Hartree / bohr


def _co2_cluster(n, seed):
    """(CO2)_n: linear O=C=O (1.16 A) on a 3.4 A cubic grid, random
    orientations, all-heavy atoms (4 AOs each): 12 AOs per molecule."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(n ** (1.0 / 3.0)))
    Z, X = [], []
    for k in range(n):
        c = 3.4 * np.array([k % side, (k // side) % side, k // (side * side)], float)
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        for z, s in ((6, 0.0), (8, 1.16), (8, -1.16)):
            Z.append(z)
            X.append(c + s * u)
    return np.asarray(Z, dtype=np.int32), geometry.to_bohr(np.array(X))


def _water(n, seed):
    Z, X = geometry.water_cluster(n, seed)
    return np.asarray(Z, dtype=np.int32), geometry.to_bohr(X)


def test_limits_rejected_before_device_use():
    # checked on the host before any CUDA call, so this runs without a GPU
    Z = np.ones(sparrow_b200.SG_STATIC_MAX_ATOMS + 2, dtype=np.int32)
    X = np.arange(3 * Z.size, dtype=np.float64) * 1.7
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.calculate_static("PM6", Z, X)
    assert ei.value.code == 1 and "allocation-free limit" in str(ei.value)
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.calculate_static("XTB", Z[:2], X[:6])
    assert ei.value.code == 2


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["PM6", "AM1", "MNDO"])
def test_static_matches_batched_engine_twice(method):
    Z, X = _water(8, 3)
    e_ref, g_ref, it_ref, conv_ref = sparrow_b200.batch_calculate(method, [(Z, X)], scc=1e-9, rmsd=1e-8,
                                                                  gradients=True)
    assert conv_ref[0]
    for _ in range(2):  # two calls in a row reuse the same scratch
        e, g, it, conv = sparrow_b200.calculate_static(method, Z, X, scc=1e-9, rmsd=1e-8, gradients=True)
        assert conv
        assert abs(e - e_ref[0]) < E_TOL
        assert np.max(np.abs(g - g_ref[0])) < G_TOL


@pytest.mark.gpu
def test_static_alternating_sizes_and_limits():
    # a small molecule after a large one: nothing stale may leak between calls
    Zb, Xb = _water(21, 5)                     # 63 atoms, 126 AOs
    Zs, Xs = _water(2, 7)
    rng = np.random.default_rng(4)
    Za, Xa = geometry.alkane(20, rng)         # C20H42: 62 atoms, 122 AOs
    Xa = geometry.to_bohr(Xa)
    ref = sparrow_b200.batch_calculate("PM6", [(Zb, Xb), (Zs, Xs), (np.asarray(Za, np.int32), Xa)],
                                       scc=1e-9, rmsd=1e-8, gradients=True)
    for rep in range(2):
        for i, (Z, X) in enumerate([(Zb, Xb), (Zs, Xs), (np.asarray(Za, np.int32), Xa)]):
            e, g, it, conv = sparrow_b200.calculate_static("PM6", Z, X, scc=1e-9, rmsd=1e-8, gradients=True)
            assert conv
            assert abs(e - ref[0][i]) < E_TOL
            assert np.max(np.abs(g - ref[1][i])) < G_TOL


@pytest.mark.gpu
def test_static_energy_only_and_errors():
    Z, X = _water(3, 11)
    e1, g1, _, _ = sparrow_b200.calculate_static("PM6", Z, X)
    e2, g2, _, _ = sparrow_b200.calculate_static("PM6", Z, X, gradients=True)
    assert g1 is None and g2.shape == (9, 3)
    assert abs(e1 - e2) < 1e-12
    with pytest.raises(sparrow_b200.SparrowError) as ei:   # odd electron count
        sparrow_b200.calculate_static("PM6", np.array([1], np.int32), np.zeros(3))
    assert ei.value.code == 5
    # one atom over the limit
    Zc = np.full(65, 6, dtype=np.int32)
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.calculate_static("PM6", Zc, np.arange(3 * 65, dtype=np.float64) * 3.0)
    assert ei.value.code == 1


@pytest.mark.gpu
@pytest.mark.parametrize("n_co2", [17, 21])
def test_static_at_the_upper_size_limit(n_co2):
    # 204 and 252 AOs (51 and 63 atoms): the eigensolver's tiled matrix no
    # longer fits shared memory above 192 AOs and runs from the static
    # scratch; static, batched and oracle agree
    from tests import oracle_lib as O
    Z, X = _co2_cluster(n_co2, 2)
    assert 200 <= 12 * n_co2 <= sparrow_b200.SG_STATIC_MAX_AOS
    e_ref, g_ref, _, conv_ref = sparrow_b200.batch_calculate("PM6", [(Z, X)], scc=1e-9, rmsd=1e-8, gradients=True)
    assert conv_ref[0]
    ref = O.scf("PM6", Z, X, scc=1e-9, rmsd=1e-8)
    assert abs(e_ref[0] - ref["energy"]) < E_TOL
    for _ in range(2):
        e, g, it, conv = sparrow_b200.calculate_static("PM6", Z, X, scc=1e-9, rmsd=1e-8, gradients=True)
        assert conv
        assert abs(e - e_ref[0]) < E_TOL
        assert np.max(np.abs(g - g_ref[0])) < G_TOL
        assert np.max(np.abs(g - ref["gradient"])) < G_TOL
