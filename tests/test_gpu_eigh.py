"""The SCF kernels' CTA eigensolver (Householder tridiagonalisation, Sturm
multisection, twisted-factorisation vectors, blocked back-transformation)
against numpy.linalg.eigh, through the test harness library
tests/csrc/libeigh_probe.so: eigenvalues, eigenvector residuals and
orthogonality, the shared- and global-memory placements of the matrix, and
the fallback signal on degenerate spectra."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(ROOT, "csrc", "libeigh_probe.so")


def _tiled(n):
    nt = (n + 31) // 32
    return nt * (nt + 1) // 2 * 32 * 33


def run_probe(mats, nvecs, smem_limit=0):
    import torch
    if not os.path.exists(LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "csrc")])
    L = ctypes.CDLL(LIB)
    dev = torch.device("cuda:0")
    Ns = [m.shape[0] for m in mats]
    off = np.cumsum([0] + [n * n for n in Ns])[:-1]
    eoff = np.cumsum([0] + Ns)[:-1]
    asz = [max(n * n, _tiled(n)) for n in Ns]
    aoff = np.cumsum([0] + asz)[:-1]
    F = torch.tensor(np.concatenate([m.reshape(-1) for m in mats]), dtype=torch.float64, device=dev)
    Ct = torch.zeros_like(F)
    gZ = torch.zeros_like(F)
    gV = torch.zeros_like(F)
    eps = torch.zeros(sum(Ns), dtype=torch.float64, device=dev)
    gA = torch.zeros(int(sum(asz)), dtype=torch.float64, device=dev)
    st = torch.zeros(len(mats), dtype=torch.int32, device=dev)
    t_n = torch.tensor(Ns, dtype=torch.int32, device=dev)
    t_off = torch.tensor(off, dtype=torch.int64, device=dev)
    t_eoff = torch.tensor(eoff, dtype=torch.int64, device=dev)
    t_aoff = torch.tensor(aoff, dtype=torch.int64, device=dev)
    t_nv = torch.tensor(nvecs, dtype=torch.int32, device=dev)
    vp = ctypes.c_void_p
    rc = L.eigh_probe(len(mats), vp(t_n.data_ptr()), vp(t_off.data_ptr()), vp(t_eoff.data_ptr()),
                      vp(t_aoff.data_ptr()), vp(t_nv.data_ptr()), vp(F.data_ptr()), vp(Ct.data_ptr()),
                      vp(eps.data_ptr()), vp(gA.data_ptr()), vp(gZ.data_ptr()), vp(gV.data_ptr()), vp(st.data_ptr()),
                      ctypes.c_int(smem_limit))
    assert rc == 0
    Ct, eps, st = Ct.cpu().numpy(), eps.cpu().numpy(), st.cpu().numpy()
    out = []
    for m, n in enumerate(Ns):
        out.append((eps[eoff[m]:eoff[m] + n], Ct[off[m]:off[m] + n * n].reshape(n, n)[:nvecs[m]], int(st[m])))
    return out


def _sym(rng, n, spread=1.0):
    a = rng.standard_normal((n, n)) * spread
    return 0.5 * (a + a.T)


def _check(A, lam, X, nvec, tol=1e-11):
    w = np.linalg.eigvalsh(A)
    scale = max(1.0, np.max(np.abs(w)))
    assert np.max(np.abs(lam - w)) < tol * scale * len(A)
    if nvec:
        res = A @ X.T - X.T * lam[:nvec]
        assert np.max(np.abs(res)) < 50 * tol * scale * len(A)
        assert np.max(np.abs(X @ X.T - np.eye(nvec))) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("smem_limit", [0, 64 * 1024])
def test_random_symmetric_matrices(smem_limit):
    # sizes around every tile boundary, shared and global placement
    rng = np.random.default_rng(7)
    sizes = [1, 2, 3, 4, 5, 8, 17, 31, 32, 33, 63, 64, 65, 96, 97, 128, 129, 160, 182, 192, 193, 224, 256, 257, 300]
    mats = [_sym(rng, n) for n in sizes]
    nvecs = [max(1, n // 2) for n in sizes]
    for A, nv, (lam, X, st) in zip(mats, nvecs, run_probe(mats, nvecs, smem_limit)):
        assert st == 0, len(A)
        _check(A, lam, X, nv)


@pytest.mark.gpu
def test_fock_like_spectra_all_vectors():
    # graded diagonal plus coupling (core levels near -20, valence near 0),
    # every vector requested (the canonical-orbital pass)
    rng = np.random.default_rng(11)
    mats, nvecs = [], []
    for n in (14, 50, 98, 146, 182):
        d = np.sort(np.concatenate([rng.uniform(-25, -15, n // 8), rng.uniform(-2, 1, n - n // 8)]))
        A = np.diag(d) + 0.3 * _sym(rng, n) / np.sqrt(n)
        mats.append(A)
        nvecs.append(n)
    for A, nv, (lam, X, st) in zip(mats, nvecs, run_probe(mats, nvecs)):
        assert st == 0
        _check(A, lam, X, nv)


@pytest.mark.gpu
def test_degenerate_spectra_ask_for_the_fallback():
    # exactly repeated eigenvalues among the requested vectors, and a
    # degenerate frontier, are reported (status 1) instead of returning
    # non-orthogonal vectors; a matrix that is already diagonal with distinct
    # entries is solved
    rng = np.random.default_rng(3)
    n = 40
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    d = np.arange(n, dtype=float)
    d[5] = d[6] = 5.5
    A1 = Q @ np.diag(d) @ Q.T
    d2 = np.arange(n, dtype=float)
    d2[20] = d2[19]
    A2 = Q @ np.diag(d2) @ Q.T
    A3 = np.diag(np.arange(n, dtype=float) * 0.1 - 1.0)
    res = run_probe([A1, A2, A3], [20, 20, 20])
    assert res[0][2] == 1
    assert res[1][2] == 1
    assert res[2][2] == 0
    _check(A3, res[2][0], res[2][1], 20)
