"""ctypes access to the CPU oracle (oracle/liboracle_nddo.so).

Test infrastructure: the oracle is the checker for the CUDA engine and is only
loaded by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "liboracle_nddo.so")

_lib = None

SYMBOLS = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Ne": 10, "Na": 11,
           "Mg": 12, "Al": 13, "Si": 14, "P": 15, "S": 16, "Cl": 17, "Ar": 18, "K": 19, "Ca": 20, "Fe": 26,
           "Zn": 30, "Br": 35, "Xe": 54, "I": 53}

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
        L = ctypes.CDLL(LIB)
        L.oracle_ev_per_hartree.restype = ctypes.c_double
        L.oracle_bohr_per_angstrom.restype = ctypes.c_double
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_scf.argtypes = [ctypes.c_char_p, ctypes.c_int, _I, _D, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int, ctypes.c_int, _D, _D, _D, ctypes.c_void_p,
                                 ctypes.c_void_p]
        L.oracle_one_electron.argtypes = [ctypes.c_char_p, ctypes.c_int, _I, _D, ctypes.c_int, _D, _D, _I]
        L.oracle_pair_blocks.argtypes = [ctypes.c_char_p, ctypes.c_int, _I, _D, _D, _D, _D, _I]
        L.oracle_local_block.argtypes = [ctypes.c_double, _D, _D, _D, _D, _D]
        L.oracle_charge_separations.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, _D]
        L.oracle_element_params.argtypes = [ctypes.c_char_p, ctypes.c_int, _D]
        L.oracle_energy_at_density.argtypes = [ctypes.c_char_p, ctypes.c_int, _I, _D, _D, _D, _D]
        _lib = L
    return _lib


def ev_per_hartree():
    return lib().oracle_ev_per_hartree()


def bohr_per_angstrom():
    return lib().oracle_bohr_per_angstrom()


def _arr(Z, xyz_bohr):
    Z = np.ascontiguousarray(Z, dtype=np.int32)
    x = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1)
    return Z, x


def scf(method, Z, xyz_bohr, charge=0, scc=1e-7, rmsd=1e-8, max_iter=1000, gradient=True, want_density=False):
    """Converged restricted SCF: returns dict(energy, gradient, e_el, e_rep, iterations, converged, nao, nocc, P, eps)."""
    Z, x = _arr(Z, xyz_bohr)
    e = ctypes.c_double()
    g = np.zeros(x.size)
    info = np.zeros(8)
    nao_guess = 4 * len(Z)
    P = np.zeros(nao_guess * nao_guess) if want_density else None
    eps = np.zeros(nao_guess) if want_density else None
    rc = lib().oracle_scf(method.encode(), len(Z), Z.ctypes.data_as(_I), x.ctypes.data_as(_D), int(charge), scc,
                          rmsd, max_iter, 1 if gradient else 0, ctypes.byref(e), g.ctypes.data_as(_D),
                          info.ctypes.data_as(_D), P.ctypes.data if P is not None else None,
                          eps.ctypes.data if eps is not None else None)
    if rc != 0:
        raise RuntimeError("oracle_scf failed (%d): %s" % (rc, lib().oracle_last_error().decode()))
    n = int(info[4])
    out = dict(energy=e.value, gradient=g.reshape(-1, 3), e_el=info[0], e_rep=info[1], iterations=int(info[2]),
               converged=bool(info[3]), nao=n, nocc=int(info[5]), nel=int(info[6]))
    if want_density:
        out["P"] = P[: n * n].reshape(n, n)
        out["eps"] = eps[:n]
    return out


def scf_uhf(method, Z, xyz_bohr, multiplicity, charge=0, scc=1e-9, rmsd=1e-9, max_iter=1000, gradient=True):
    """Converged unrestricted SCF: dict(energy, gradient, e_el, e_rep, iterations, converged, nao, n_alpha,
    n_beta, eps_alpha, eps_beta)."""
    Z, x = _arr(Z, xyz_bohr)
    e = ctypes.c_double()
    g = np.zeros(x.size)
    info = np.zeros(8)
    n_max = 4 * len(Z)
    ea, eb = np.zeros(n_max), np.zeros(n_max)
    L = lib()
    L.oracle_scf_uhf.argtypes = [ctypes.c_char_p, ctypes.c_int, _I, _D, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D]
    rc = L.oracle_scf_uhf(method.encode(), len(Z), Z.ctypes.data_as(_I), x.ctypes.data_as(_D), int(charge),
                          int(multiplicity), scc, rmsd, max_iter, 1 if gradient else 0, ctypes.byref(e),
                          g.ctypes.data_as(_D), info.ctypes.data_as(_D), ea.ctypes.data_as(_D), eb.ctypes.data_as(_D))
    if rc != 0:
        raise RuntimeError("oracle_scf_uhf failed (%d): %s" % (rc, L.oracle_last_error().decode()))
    n = int(info[4])
    return dict(energy=e.value, gradient=g.reshape(-1, 3), e_el=info[0], e_rep=info[1], iterations=int(info[2]),
                converged=bool(info[3]), nao=n, n_alpha=int(info[5]), n_beta=int(info[6]), eps_alpha=ea[:n],
                eps_beta=eb[:n])


def one_electron(method, Z, xyz_bohr, charge=0):
    Z, x = _arr(Z, xyz_bohr)
    n_max = 4 * len(Z)
    H = np.zeros(n_max * n_max)
    S = np.zeros(n_max * n_max)
    nao = ctypes.c_int()
    rc = lib().oracle_one_electron(method.encode(), len(Z), Z.ctypes.data_as(_I), x.ctypes.data_as(_D), charge,
                                   H.ctypes.data_as(_D), S.ctypes.data_as(_D), ctypes.byref(nao))
    if rc != 0:
        raise RuntimeError("oracle_one_electron failed (%d): %s" % (rc, lib().oracle_last_error().decode()))
    n = nao.value
    return H[: n * n].reshape(n, n), S[: n * n].reshape(n, n)


def pair_blocks(method, Z, xyz_bohr):
    Z, x = _arr(Z, xyz_bohr)
    n = len(Z)
    npair_max = n * (n - 1) // 2
    G = np.zeros(max(npair_max, 1) * 100)
    VA = np.zeros(max(npair_max, 1) * 10)
    VB = np.zeros(max(npair_max, 1) * 10)
    npairs = ctypes.c_int()
    rc = lib().oracle_pair_blocks(method.encode(), n, Z.ctypes.data_as(_I), x.ctypes.data_as(_D),
                                  G.ctypes.data_as(_D), VA.ctypes.data_as(_D), VB.ctypes.data_as(_D),
                                  ctypes.byref(npairs))
    if rc != 0:
        raise RuntimeError("oracle_pair_blocks failed (%d)" % rc)
    k = npairs.value
    return G[: k * 100].reshape(k, 10, 10), VA[: k * 10].reshape(k, 10), VB[: k * 10].reshape(k, 10)


def energy_at_density(method, Z, xyz_bohr, P):
    Z, x = _arr(Z, xyz_bohr)
    P = np.ascontiguousarray(P, dtype=np.float64)
    e = ctypes.c_double()
    g = np.zeros(x.size)
    rc = lib().oracle_energy_at_density(method.encode(), len(Z), Z.ctypes.data_as(_I), x.ctypes.data_as(_D),
                                        P.ctypes.data_as(_D), ctypes.byref(e), g.ctypes.data_as(_D))
    if rc != 0:
        raise RuntimeError("oracle_energy_at_density failed (%d)" % rc)
    return e.value, g.reshape(-1, 3)


def set_parameters(method, records=None):
    """Make the oracle use caller-given raw records for a method (the output of
    tests.param_sets.oracle_records), or its published set again (None)."""
    L = lib()
    L.oracle_set_parameters.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_int]
    if records is None:
        rc = L.oracle_set_parameters(method.encode(), None, -1, None, 0)
    else:
        arr, n, darr, nd = records
        rc = L.oracle_set_parameters(method.encode(), ctypes.cast(arr, ctypes.c_void_p), n,
                                     ctypes.cast(darr, ctypes.c_void_p), nd)
    if rc != 0:
        raise RuntimeError("oracle_set_parameters failed")


def element_params(method, Z):
    out = np.zeros(20)
    rc = lib().oracle_element_params(method.encode(), Z, out.ctypes.data_as(_D))
    if rc != 0:
        raise RuntimeError("no parameters")
    return out


def local_block(R, rhoA, DA, rhoB, DB):
    out = np.zeros(100)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rhoA, DA, rhoB, DB)]
    lib().oracle_local_block(R, *[a.ctypes.data_as(_D) for a in arrs], out.ctypes.data_as(_D))
    return out.reshape(10, 10)


def charge_separations(ns, np_, zs, zp):
    out = np.zeros(2)
    lib().oracle_charge_separations(ns, np_, zs, zp, out.ctypes.data_as(_D))
    return out


# ---------------------------------------------------------------------------
# DFTB2 / DFTB3 oracle (oracle/liboracle_dftb.so)
# ---------------------------------------------------------------------------
LIB_DFTB = os.path.join(ROOT, "oracle", "liboracle_dftb.so")
_dlib = None


def dftb_lib():
    global _dlib
    if _dlib is None:
        if not os.path.exists(LIB_DFTB):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
        L = ctypes.CDLL(LIB_DFTB)
        L.dftb_oracle_last_error.restype = ctypes.c_char_p
        L.dftb_oracle_scf.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _I, _D, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D, _D, _D,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.dftb_oracle_matrices.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _I, _D, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _I]
        L.dftb_oracle_tddftb.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _I, _D, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         _D, ctypes.c_void_p, _D]
        L.dftb_oracle_set_dense_casida_limit.argtypes = [ctypes.c_int]
        _dlib = L
    return _dlib


DFTB_DEFAULT_SET = {2: "mio-1-1", 3: "3ob-3-1"}


def set_dense_casida_limit(limit):
    """Transitions up to which the oracle's TD-DFTB solves the Casida problem
    densely (default 2000; the matrix-free Davidson iteration above)."""
    dftb_lib().dftb_oracle_set_dense_casida_limit(int(limit))


def dftb_scf(order, Z, xyz_bohr, charge=0, parameters=None, scc=1e-7, rmsd=1e-8, max_iter=1000, gradient=True,
             want_density=False):
    """Converged restricted DFTB2/DFTB3: dict(energy, gradient, e_el, e_rep, iterations, converged, nao, nocc,
    charges, eps[, P])."""
    Z, x = _arr(Z, xyz_bohr)
    n = len(Z)
    params = parameters or DFTB_DEFAULT_SET[order]
    e = ctypes.c_double()
    g = np.zeros(x.size)
    info = np.zeros(8)
    q = np.zeros(n)
    eps = np.zeros(4 * n)
    P = np.zeros(16 * n * n) if want_density else None
    rc = dftb_lib().dftb_oracle_scf(params.encode(), order, n, Z.ctypes.data_as(_I), x.ctypes.data_as(_D),
                                    int(charge), scc, rmsd, max_iter, 1 if gradient else 0, ctypes.byref(e),
                                    g.ctypes.data_as(_D), info.ctypes.data_as(_D), q.ctypes.data, eps.ctypes.data,
                                    P.ctypes.data if P is not None else None)
    if rc not in (0, 3):
        raise RuntimeError(dftb_lib().dftb_oracle_last_error().decode())
    nao = int(info[4])
    out = dict(energy=e.value, gradient=g.reshape(-1, 3), e_el=info[0], e_rep=info[1], iterations=int(info[2]),
               converged=bool(info[3]), nao=nao, nocc=int(info[5]), charges=q, eps=eps[:nao])
    if P is not None:
        out["P"] = P[:nao * nao].reshape(nao, nao)
    return out


def dftb_scf_uhf(order, Z, xyz_bohr, multiplicity, charge=0, parameters=None, scc=1e-9, rmsd=1e-9, max_iter=1000,
                 gradient=True):
    """Converged spin-polarised DFTB2/DFTB3: dict(energy, gradient, e_el, e_rep, e_spin, iterations, converged,
    nao, n_alpha, n_beta, charges, eps_alpha, eps_beta)."""
    Z, x = _arr(Z, xyz_bohr)
    n = len(Z)
    params = parameters or DFTB_DEFAULT_SET[order]
    e = ctypes.c_double()
    g = np.zeros(x.size)
    info = np.zeros(8)
    q = np.zeros(n)
    ea, eb = np.zeros(4 * n), np.zeros(4 * n)
    L = dftb_lib()
    L.dftb_oracle_scf_uhf.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _I, _D, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D,
                                      _D, _D, _D, _D, _D]
    rc = L.dftb_oracle_scf_uhf(params.encode(), order, n, Z.ctypes.data_as(_I), x.ctypes.data_as(_D), int(charge),
                               int(multiplicity), scc, rmsd, max_iter, 1 if gradient else 0, ctypes.byref(e),
                               g.ctypes.data_as(_D), info.ctypes.data_as(_D), q.ctypes.data_as(_D),
                               ea.ctypes.data_as(_D), eb.ctypes.data_as(_D))
    if rc not in (0, 3):
        raise RuntimeError(L.dftb_oracle_last_error().decode())
    nao = int(info[4])
    return dict(energy=e.value, gradient=g.reshape(-1, 3), e_el=info[0], e_rep=info[1], e_spin=info[7],
                iterations=int(info[2]), converged=bool(info[3]), nao=nao, n_alpha=int(info[5]), n_beta=int(info[6]),
                charges=q, eps_alpha=ea[:nao], eps_beta=eb[:nao])


def dftb_matrices(order, Z, xyz_bohr, parameters=None):
    """H0, S (N x N), gamma (nat x nat) and Gamma (nat x nat, DFTB3) at a geometry."""
    Z, x = _arr(Z, xyz_bohr)
    n = len(Z)
    params = parameters or DFTB_DEFAULT_SET[order]
    N = 4 * n
    H0 = np.zeros(N * N)
    S = np.zeros(N * N)
    gam = np.zeros(n * n)
    Gam = np.zeros(n * n)
    nao = ctypes.c_int()
    rc = dftb_lib().dftb_oracle_matrices(params.encode(), order, n, Z.ctypes.data_as(_I), x.ctypes.data_as(_D),
                                         H0.ctypes.data, S.ctypes.data, gam.ctypes.data, Gam.ctypes.data,
                                         ctypes.byref(nao))
    if rc != 0:
        raise RuntimeError(dftb_lib().dftb_oracle_last_error().decode())
    N = nao.value
    return H0[:N * N].reshape(N, N), S[:N * N].reshape(N, N), gam.reshape(n, n), Gam.reshape(n, n)


def dftb_tddftb(order, Z, xyz_bohr, nroots=8, triplet=False, charge=0, parameters=None, scc=1e-9, rmsd=1e-9,
                max_iter=1000):
    """TD-DFTB excitation energies (Hartree, ascending) and singlet transition dipoles (nroots x 3, e bohr)."""
    Z, x = _arr(Z, xyz_bohr)
    n = len(Z)
    params = parameters or DFTB_DEFAULT_SET[order]
    om = np.zeros(nroots)
    dip = np.zeros(3 * nroots)
    info = np.zeros(4)
    rc = dftb_lib().dftb_oracle_tddftb(params.encode(), order, n, Z.ctypes.data_as(_I), x.ctypes.data_as(_D),
                                       int(charge), scc, rmsd, max_iter, 1 if triplet else 0, nroots,
                                       om.ctypes.data_as(_D), dip.ctypes.data, info.ctypes.data_as(_D))
    if rc != 0:
        raise RuntimeError(dftb_lib().dftb_oracle_last_error().decode())
    nt = int(info[3])
    k = min(nroots, nt)
    return dict(omega=om[:k], dipoles=dip[:3 * k].reshape(k, 3), energy=info[0], nao=int(info[1]),
                nocc=int(info[2]), transitions=nt)
