"""Synthetic structure generators: sizes, bond lengths, reproducibility."""
import numpy as np

from sparrow_b200 import geometry


def _dist(x, i, j):
    return float(np.linalg.norm(x[i] - x[j]))


def test_water_cluster_32_shape_and_geometry():
    Z, x = geometry.water_cluster(32, seed=0)
    assert len(Z) == 96 and (Z == 8).sum() == 32
    for w in range(32):
        o, h1, h2 = 3 * w, 3 * w + 1, 3 * w + 2
        assert abs(_dist(x, o, h1) - 0.96) < 1e-12 and abs(_dist(x, o, h2) - 0.96) < 1e-12
        v1, v2 = x[h1] - x[o], x[h2] - x[o]
        ang = np.degrees(np.arccos(v1 @ v2 / (np.linalg.norm(v1) * np.linalg.norm(v2))))
        assert abs(ang - 104.5) < 1e-9
    Z2, x2 = geometry.water_cluster(32, seed=0)
    assert np.array_equal(x, x2)


def test_alkane_composition_and_bonds():
    rng = np.random.default_rng(3)
    for n in (1, 2, 3, 7, 30):
        Z, x = geometry.alkane(n, rng)
        assert (Z == 6).sum() == n and (Z == 1).sum() == 2 * n + 2
        for k in range(n - 1):
            assert abs(_dist(x, k, k + 1) - 1.54) < 1e-9
        # every hydrogen 1.09 from its nearest carbon
        for h in np.where(Z == 1)[0]:
            d = min(_dist(x, h, c) for c in range(n))
            assert abs(d - 1.09) < 1e-9
        # no clashes
        d = np.linalg.norm(x[:, None] - x[None], axis=-1) + np.eye(len(Z)) * 10
        assert d.min() > 0.9


def test_alkane_batch_sizes_cover_range():
    mols = geometry.alkane_batch(4096, seed=1)
    ns = np.array([(z == 6).sum() for z, _ in mols])
    assert ns.min() == 2 and ns.max() == 30
    naos = 6 * ns + 2
    assert naos.min() == 14 and naos.max() == 182


def test_polyene_composition():
    rng = np.random.default_rng(6)
    Z, x = geometry.polyene(5, rng)
    assert (Z == 6).sum() == 10 and (Z == 1).sum() == 12
    d = np.linalg.norm(x[:, None] - x[None], axis=-1) + np.eye(len(Z)) * 10
    assert d.min() > 0.9
