"""Request server (continuous batching): each result is the same alone and in
the mix, and requests of different sizes and methods interleave."""
import threading

import numpy as np
import pytest

import sparrow_b200
from sparrow_b200 import geometry
from tests import oracle_lib as O

E_TOL = 1e-6   # Hartree
G_TOL = 1e-5   # Hartree / bohr


def _mix(count, seed):
    rng = np.random.default_rng(seed)
    mols = []
    for k in range(count):
        if rng.random() < 0.5:
            z, x = geometry.alkane(int(rng.integers(1, 14)), rng)
        else:
            z, x = geometry.water_cluster(int(rng.integers(2, 9)), seed=int(rng.integers(1 << 30)))
        r = rng.random()
        mols.append((np.asarray(z, np.int32), geometry.to_bohr(x), "PM6" if r < 0.6 else ("DFTB2" if r < 0.85 else "AM1")))
    return mols


def test_submit_validation_without_gpu_work():
    # invalid requests are refused at submission, before any device work
    if not sparrow_b200.lib():
        pytest.skip("library missing")
    try:
        srv = sparrow_b200.Server(device_budget_gb=1.0)
    except sparrow_b200.SparrowError as e:
        assert e.code == 7  # no CUDA device here
        return
    with srv:
        with pytest.raises(sparrow_b200.SparrowError) as e:
            srv.submit("PM6", [1], np.zeros(3))
        assert e.value.code == 5
        with pytest.raises(sparrow_b200.SparrowError) as e:
            srv.submit("PM6", [1, 1], np.zeros(6))
        assert e.value.code == 1
        with pytest.raises(sparrow_b200.SparrowError) as e:
            srv.submit("PM6", [17, 17], np.array([0, 0, 0, 3.8, 0, 0.0]))
        assert e.value.code == 3
        with pytest.raises(sparrow_b200.SparrowError) as e:  # 7 electrons: no triplet
            srv.submit("PM6", [8, 1], np.array([0, 0, 0, 0, 0, 1.8]), multiplicity=3)
        assert e.value.code == 5


@pytest.mark.gpu
def test_alone_equals_in_the_mix():
    mols = _mix(40, seed=3)
    with sparrow_b200.Server(device_budget_gb=4.0, slots=3, scc=1e-9, rmsd=1e-8) as srv:
        alone = []
        for z, x, m in mols:  # one request in flight at a time
            alone.append(srv.wait(srv.submit(m, z, x)))
        order = np.random.default_rng(5).permutation(len(mols))
        ids = {int(i): srv.submit(mols[i][2], mols[i][0], mols[i][1]) for i in order}
        mixed = {i: srv.wait(r) for i, r in ids.items()}
        st = srv.stats()
    assert st["max_batch"] > 1  # the second phase really batched
    for i, a in enumerate(alone):
        b = mixed[i]
        assert a.successful_calculation and b.successful_calculation
        assert abs(a.energy - b.energy) < E_TOL
        assert np.max(np.abs(a.gradients - b.gradients)) < G_TOL


@pytest.mark.gpu
def test_served_results_match_oracle_and_clients_overlap():
    mols = _mix(12, seed=9)
    results = {}
    with sparrow_b200.Server(device_budget_gb=2.0, slots=2, scc=1e-9, rmsd=1e-8) as srv:
        def client(idx):
            for i in idx:
                z, x, m = mols[i]
                results[i] = srv.wait(srv.submit(m, z, x))
        threads = [threading.Thread(target=client, args=(range(k, len(mols), 3),)) for k in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    for i, (z, x, m) in enumerate(mols):
        if m == "DFTB2":
            ref = O.dftb_scf(2, z, x, scc=1e-10, rmsd=1e-9)
        else:
            ref = O.scf(m, z, x, scc=1e-9, rmsd=1e-8)
        assert abs(results[i].energy - ref["energy"]) < E_TOL
        assert np.max(np.abs(results[i].gradients - ref["gradient"])) < G_TOL
        assert results[i].latency_s > 0


@pytest.mark.gpu
def test_tiny_budget_still_makes_progress():
    mols = _mix(10, seed=11)
    with sparrow_b200.Server(device_budget_gb=1e-6, slots=2) as srv:  # every batch exceeds the budget
        ids = [srv.submit(m, z, x, gradients=False) for z, x, m in mols]
        res = [srv.wait(r, timeout=120) for r in ids]
        st = srv.stats()
    assert all(r is not None and r.successful_calculation for r in res)
    assert st["max_batch"] == 1  # admitted one at a time


@pytest.mark.gpu
def test_open_shells_are_served_beside_closed_shells():
    # radicals (unrestricted) and closed shells (restricted) interleaved; batches
    # never mix the two spin treatments, and each result matches the oracle
    from tests.test_gpu_sdftb import _radicals as dftb_radicals
    from tests.test_gpu_uhf import _radicals as nddo_radicals
    reqs = [("PM6", z, x, c, m) for z, x, c, m in nddo_radicals()]
    reqs += [("DFTB2", z, x, c, m) for z, x, c, m in dftb_radicals()]
    reqs += [(m, z, x, 0, 1) for z, x, m in _mix(12, seed=9)]
    order = np.random.default_rng(2).permutation(len(reqs))
    with sparrow_b200.Server(device_budget_gb=4.0, slots=3, scc=1e-10, rmsd=1e-9, max_iter=500) as srv:
        ids = {int(i): srv.submit(reqs[i][0], reqs[i][1], reqs[i][2], charge=reqs[i][3], multiplicity=reqs[i][4])
               for i in order}
        res = {i: srv.wait(r) for i, r in ids.items()}
    for i, (method, Z, x, ch, mult) in enumerate(reqs):
        r = res[i]
        assert r.successful_calculation, (method, i)
        if mult == 1 and method != "DFTB2":
            ref = O.scf(method, Z, x, charge=ch, scc=1e-10, rmsd=1e-9)
        elif mult == 1:
            ref = O.dftb_scf(2, Z, x, charge=ch, scc=1e-10, rmsd=1e-9)
        elif method == "DFTB2":
            ref = O.dftb_scf_uhf(2, Z, x, mult, charge=ch, scc=1e-10, rmsd=1e-9)
        else:
            ref = O.scf_uhf(method, Z, x, mult, charge=ch, scc=1e-10, rmsd=1e-9)
        assert abs(r.energy - ref["energy"]) < E_TOL, (method, i)
        assert np.max(np.abs(r.gradients - ref["gradient"])) < G_TOL, (method, i)

