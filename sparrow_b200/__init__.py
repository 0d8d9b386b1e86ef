"""sparrow_b200: batched NDDO (MNDO/AM1/PM6) SCF on the NVIDIA B200.

Python mirror of the reference's calculator interface (qcscine/sparrow,
src/Sparrow/Sparrow/Implementations/GenericMethodWrapper.h:51-134 and the
Python usage in src/Sparrow/Python/Tests/CalculatorTest.py): a Calculator with
a structure, string-keyed settings, required properties and calculate()
returning results (energy, gradients, success flag).  Positions are in bohr,
energies in Hartree, gradients in Hartree/bohr.

Every call goes through the C-ABI of libsparrow_b200.so (include/sparrow_b200.h),
which runs hand-written sm_100a kernels.  There is no CPU path: if the library
or a CUDA device is missing, calls raise.
"""
import ctypes
import os

import numpy as np

__all__ = ["Calculator", "Batch", "Results", "get_calculator", "batch_calculate", "library_path", "SparrowError",
           "element_parameters", "diatomic_parameters", "hessian"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsparrow_b200.so")
_lib = None

SG_PROP_ENERGY = 1
SG_PROP_GRADIENTS = 2
SG_PROP_HESSIAN = 4
SG_PROP_ATOMIC_CHARGES = 8
SG_PROP_DIPOLE = 16
SG_ERR_NOT_CONVERGED = 6
SG_ERR_TIMEOUT = 12
SG_PENDING = 13
SG_ERR_PARAMETERS = 14
SG_NDDO_ELEMENT_VALUES = 57
SG_DFTB_ELEMENT_VALUES = 8
SG_STATIC_MAX_ATOMS = 64
SG_STATIC_MAX_AOS = 256

_D = ctypes.POINTER(ctypes.c_double)
_I32 = ctypes.POINTER(ctypes.c_int32)
_VP = ctypes.c_void_p


class SparrowError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("sparrow_b200 error %d: %s" % (code, message))
        self.code = code


def library_path():
    return _LIB_PATH


def lib():
    """Load libsparrow_b200.so (built by __graft_entry__.build() / `make -C sparrow_b200/csrc`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError("libsparrow_b200.so is not built: run `make -C sparrow_b200/csrc`")
    L = ctypes.CDLL(_LIB_PATH)
    sig = {
        "sg_version": (ctypes.c_char_p, []),
        "sg_create": (ctypes.c_int32, [ctypes.c_char_p, ctypes.POINTER(_VP)]),
        "sg_destroy": (None, [_VP]),
        "sg_clone": (ctypes.c_int32, [_VP, ctypes.POINTER(_VP)]),
        "sg_last_error": (ctypes.c_char_p, [_VP]),
        "sg_set_structure": (ctypes.c_int32, [_VP, ctypes.c_int32, _I32, _D]),
        "sg_modify_positions": (ctypes.c_int32, [_VP, _D]),
        "sg_get_positions": (ctypes.c_int32, [_VP, _D]),
        "sg_get_n_atoms": (ctypes.c_int32, [_VP, _I32]),
        "sg_set_setting_int": (ctypes.c_int32, [_VP, ctypes.c_char_p, ctypes.c_int64]),
        "sg_set_setting_double": (ctypes.c_int32, [_VP, ctypes.c_char_p, ctypes.c_double]),
        "sg_set_setting_string": (ctypes.c_int32, [_VP, ctypes.c_char_p, ctypes.c_char_p]),
        "sg_get_setting_double": (ctypes.c_int32, [_VP, ctypes.c_char_p, _D]),
        "sg_get_setting_int": (ctypes.c_int32, [_VP, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]),
        "sg_set_required_properties": (ctypes.c_int32, [_VP, ctypes.c_uint32]),
        "sg_calculate": (ctypes.c_int32, [_VP]),
        "sg_get_energy": (ctypes.c_int32, [_VP, _D]),
        "sg_get_gradients": (ctypes.c_int32, [_VP, _D]),
        "sg_get_scf_info": (ctypes.c_int32, [_VP, _I32, _I32, _I32, _I32]),
        "sg_get_orbital_energies": (ctypes.c_int32, [_VP, _D]),
        "sg_get_density": (ctypes.c_int32, [_VP, _D]),
        "sg_calculate_excitations": (ctypes.c_int32, [_VP, ctypes.c_int32, ctypes.c_int32, _D, _VP]),
        "sg_batch_excitations": (ctypes.c_int32, [_VP, ctypes.c_int32, ctypes.c_int32, _D, _VP, _VP]),
        "sg_batch_excitation_cycles": (ctypes.c_int32, [_VP, _VP]),
        "sg_set_density": (ctypes.c_int32, [_VP, _D]),
        "sg_get_beta_orbital_energies": (ctypes.c_int32, [_VP, _D]),
        "sg_get_hessian": (ctypes.c_int32, [_VP, _D]),
        "sg_get_atomic_charges": (ctypes.c_int32, [_VP, _D]),
        "sg_get_dipole": (ctypes.c_int32, [_VP, _D]),
        "sg_get_spin_densities": (ctypes.c_int32, [_VP, _D, _D]),
        "sg_set_spin_densities": (ctypes.c_int32, [_VP, _D, _D]),
        "sg_calculate_hessian": (ctypes.c_int32, [ctypes.c_char_p, ctypes.c_int32, _I32, _D, ctypes.c_int32,
                                                  ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                                  ctypes.c_int32, ctypes.c_double, _D, _I32, ctypes.c_char_p,
                                                  ctypes.c_int32]),
        "sg_batch_create_unrestricted": (ctypes.c_int32, [ctypes.c_char_p, ctypes.c_int32, _I32, _I32, _D, _I32,
                                                          _I32, ctypes.POINTER(_VP)]),
        "sg_batch_create": (ctypes.c_int32, [ctypes.c_char_p, ctypes.c_int32, _I32, _I32, _D, _I32,
                                             ctypes.POINTER(_VP)]),
        "sg_batch_destroy": (None, [_VP]),
        "sg_batch_last_error": (ctypes.c_char_p, [_VP]),
        "sg_batch_set_scf": (ctypes.c_int32, [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int32]),
        "sg_batch_set_scf_path": (ctypes.c_int32, [_VP, ctypes.c_int32]),
        "sg_batch_set_mixed_switch": (ctypes.c_int32, [_VP, ctypes.c_double]),
        "sg_batch_set_tuning": (ctypes.c_int32, [_VP, ctypes.c_int32, ctypes.c_int32]),
        "sg_tuning_table": (ctypes.c_int32, [_I32, _I32, ctypes.c_int32]),
        "sg_batch_set_positions": (ctypes.c_int32, [_VP, _D]),
        "sg_batch_run": (ctypes.c_int32, [_VP, ctypes.c_uint32]),
        "sg_batch_results": (ctypes.c_int32, [_VP, _D, _D, _I32, _I32]),
        "sg_batch_launches": (ctypes.c_int32, [_VP]),
        "sg_batch_stream": (_VP, [_VP]),
        "sg_batch_stage_times": (ctypes.c_int32, [_VP, _D]),
        "sg_batch_record_event": (ctypes.c_int32, [_VP, ctypes.c_int32]),
        "sg_batch_event_elapsed": (ctypes.c_int32, [_VP, ctypes.c_int32, ctypes.c_int32, _D]),
        "sg_batch_transfer_bytes": (ctypes.c_int32, [_VP, ctypes.POINTER(ctypes.c_int64),
                                                     ctypes.POINTER(ctypes.c_int64)]),
        "sg_release_cached_memory": (None, []),
        "sg_batch_scf_stats": (ctypes.c_int32, [_VP, _I32, _I32, ctypes.POINTER(ctypes.c_int64)]),
        "sg_batch_calculate": (ctypes.c_int32, [ctypes.c_char_p, ctypes.c_int32, _I32, _I32, _D, _I32,
                                                ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_uint32,
                                                _D, _D, _I32, _I32, ctypes.c_char_p, ctypes.c_int32]),
        "sg_server_create": (ctypes.c_int32, [ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_int32, ctypes.POINTER(_VP)]),
        "sg_server_destroy": (None, [_VP]),
        "sg_server_last_error": (ctypes.c_char_p, []),
        "sg_server_submit_spin": (ctypes.c_int32, [_VP, ctypes.c_char_p, ctypes.c_int32, _I32, _D, ctypes.c_int32,
                                                   ctypes.c_int32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int64)]),
        "sg_server_submit": (ctypes.c_int32, [_VP, ctypes.c_char_p, ctypes.c_int32, _I32, _D, ctypes.c_int32,
                                              ctypes.c_uint32, ctypes.POINTER(ctypes.c_int64)]),
        "sg_server_wait": (ctypes.c_int32, [_VP, ctypes.c_int64, ctypes.c_double, _D, _D, _I32, _I32, _D]),
        "sg_server_poll": (ctypes.c_int32, [_VP, ctypes.c_int64, _D, _D, _I32, _I32, _D]),
        "sg_server_drain": (ctypes.c_int32, [_VP]),
        "sg_server_stats": (ctypes.c_int32, [_VP] + [ctypes.POINTER(ctypes.c_int64)] * 4),
        "sg_element_parameters": (ctypes.c_int32, [ctypes.c_char_p, ctypes.c_int32, _D, ctypes.c_int32,
                                                   ctypes.c_char_p, ctypes.c_int32]),
        "sg_diatomic_parameters": (ctypes.c_int32, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, _D,
                                                    ctypes.c_char_p, ctypes.c_int32]),
        "sg_calculate_static": (ctypes.c_int32, [ctypes.c_char_p, ctypes.c_int32, _I32, _D, ctypes.c_int32,
                                                 ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_uint32,
                                                 _VP, _D, _D, _I32, _I32, ctypes.c_char_p, ctypes.c_int32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _dptr(a):
    return a.ctypes.data_as(_D)


def _iptr(a):
    return a.ctypes.data_as(_I32)


class Results:
    """Results of one calculation (subset of the reference's Utils::Results)."""

    def __init__(self, energy, gradients, successful_calculation, iterations, n_aos, n_occupied):
        self.energy = energy
        self.gradients = gradients
        self.successful_calculation = successful_calculation
        self.iterations = iterations
        self.n_aos = n_aos
        self.n_occupied = n_occupied
        self.hessian = None  # (3 n_atoms, 3 n_atoms) when "hessian" was required
        self.atomic_charges = None  # (n_atoms,) when "atomic_charges" was required
        self.dipole = None  # (3,) e bohr when "dipole" was required


class _Settings:
    """String-keyed settings with the reference's names and defaults."""

    _INT = ("molecular_charge", "spin_multiplicity", "max_scf_iterations")
    _REAL = ("self_consistence_criterion", "density_rmsd_criterion")
    _STR = ("spin_mode", "scf_mixer", "method_parameters", "scf_path")

    def __init__(self, calc):
        self._calc = calc
        self._str = {"spin_mode": "any", "scf_mixer": "diis", "method_parameters": "", "scf_path": "auto"}

    def __setitem__(self, key, value):
        L, h = lib(), self._calc._h
        if key in self._INT:
            rc = L.sg_set_setting_int(h, key.encode(), int(value))
        elif key in self._REAL:
            rc = L.sg_set_setting_double(h, key.encode(), float(value))
        elif key in self._STR:
            rc = L.sg_set_setting_string(h, key.encode(), str(value).encode())
            if rc == 0:
                self._str[key] = str(value)
        else:
            raise KeyError("unknown setting %r" % key)
        self._calc._check(rc)

    def __getitem__(self, key):
        L, h = lib(), self._calc._h
        if key in self._INT:
            v = ctypes.c_int64()
            self._calc._check(L.sg_get_setting_int(h, key.encode(), ctypes.byref(v)))
            return v.value
        if key in self._REAL:
            v = ctypes.c_double()
            self._calc._check(L.sg_get_setting_double(h, key.encode(), ctypes.byref(v)))
            return v.value
        if key in self._STR:
            return self._str[key]
        raise KeyError("unknown setting %r" % key)


class Calculator:
    """Single-structure calculator ("PM6", "AM1" or "MNDO")."""

    def __init__(self, method="PM6", _handle=None):
        L = lib()
        if _handle is None:
            h = _VP()
            rc = L.sg_create(method.encode(), ctypes.byref(h))
            if rc != 0:
                raise SparrowError(rc, L.sg_last_error(None).decode())
            _handle = h
        self._h = _handle
        self.method = method.upper()
        self.settings = _Settings(self)
        self._n_atoms = 0

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.sg_destroy(self._h)
            self._h = None

    def _check(self, rc, allow=()):
        if rc != 0 and rc not in allow:
            raise SparrowError(rc, lib().sg_last_error(self._h).decode())
        return rc

    def set_structure(self, atomic_numbers, positions_bohr):
        Z = np.ascontiguousarray(atomic_numbers, dtype=np.int32)
        x = np.ascontiguousarray(positions_bohr, dtype=np.float64).reshape(-1)
        if x.size != 3 * Z.size:
            raise ValueError("positions must be (n_atoms, 3)")
        self._check(lib().sg_set_structure(self._h, Z.size, _iptr(Z), _dptr(x)))
        self._n_atoms = Z.size

    @property
    def structure(self):
        return self._n_atoms

    @structure.setter
    def structure(self, value):
        self.set_structure(*value)

    @property
    def positions(self):
        out = np.zeros(3 * self._n_atoms)
        self._check(lib().sg_get_positions(self._h, _dptr(out)))
        return out.reshape(-1, 3)

    @positions.setter
    def positions(self, xyz_bohr):
        x = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1)
        if x.size != 3 * self._n_atoms:
            raise ValueError("positions must be (n_atoms, 3)")
        self._check(lib().sg_modify_positions(self._h, _dptr(x)))

    def set_required_properties(self, props):
        mask = 0
        for p in props:
            p = p.lower()
            if p == "energy":
                mask |= SG_PROP_ENERGY
            elif p in ("gradients", "gradient"):
                mask |= SG_PROP_GRADIENTS | SG_PROP_ENERGY
            elif p == "hessian":
                mask |= SG_PROP_HESSIAN | SG_PROP_ENERGY
            elif p in ("atomic_charges", "charges"):
                mask |= SG_PROP_ATOMIC_CHARGES | SG_PROP_ENERGY
            elif p == "dipole":
                mask |= SG_PROP_DIPOLE | SG_PROP_ENERGY
            else:
                raise ValueError("unsupported property %r" % p)
        self._check(lib().sg_set_required_properties(self._h, mask))
        self._mask = mask

    def calculate(self):
        L = lib()
        rc = self._check(L.sg_calculate(self._h), allow=(SG_ERR_NOT_CONVERGED,))
        e = ctypes.c_double()
        self._check(L.sg_get_energy(self._h, ctypes.byref(e)))
        it, conv, nao, nocc = (ctypes.c_int32() for _ in range(4))
        self._check(L.sg_get_scf_info(self._h, ctypes.byref(it), ctypes.byref(conv), ctypes.byref(nao),
                                      ctypes.byref(nocc)))
        grad = None
        if getattr(self, "_mask", SG_PROP_ENERGY) & SG_PROP_GRADIENTS:
            g = np.zeros(3 * self._n_atoms)
            self._check(L.sg_get_gradients(self._h, _dptr(g)))
            grad = g.reshape(-1, 3)
        self._nao = nao.value
        res = Results(e.value, grad, rc == 0 and bool(conv.value), it.value, nao.value, nocc.value)
        if getattr(self, "_mask", SG_PROP_ENERGY) & SG_PROP_ATOMIC_CHARGES:
            q = np.zeros(self._n_atoms)
            self._check(L.sg_get_atomic_charges(self._h, _dptr(q)))
            res.atomic_charges = q
        if getattr(self, "_mask", SG_PROP_ENERGY) & SG_PROP_DIPOLE:
            d = np.zeros(3)
            self._check(L.sg_get_dipole(self._h, _dptr(d)))
            res.dipole = d
        if getattr(self, "_mask", SG_PROP_ENERGY) & SG_PROP_HESSIAN:
            n3 = 3 * self._n_atoms
            H = np.zeros(n3 * n3)
            self._check(L.sg_get_hessian(self._h, _dptr(H)))
            res.hessian = H.reshape(n3, n3)
        return res

    def excitations(self, nroots=8, triplet=False):
        """TD-DFTB on the last DFTB2/DFTB3 calculation: (omega [nroots] Hartree,
        transition dipoles [nroots, 3] e bohr)."""
        om = np.zeros(nroots)
        dp = np.zeros(3 * nroots)
        self._check(lib().sg_calculate_excitations(self._h, nroots, 1 if triplet else 0, _dptr(om),
                                                   dp.ctypes.data_as(_VP)))
        return om, dp.reshape(nroots, 3)

    def density(self):
        n = self._nao
        P = np.zeros(n * n)
        self._check(lib().sg_get_density(self._h, _dptr(P)))
        return P.reshape(n, n)

    def orbital_energies(self):
        """Orbital energies (the alpha ones after an unrestricted calculation)."""
        e = np.zeros(self._nao)
        self._check(lib().sg_get_orbital_energies(self._h, _dptr(e)))
        return e

    def spin_densities(self):
        """(P_alpha, P_beta) of an unrestricted calculation."""
        n = self._nao
        Pa, Pb = np.zeros(n * n), np.zeros(n * n)
        self._check(lib().sg_get_spin_densities(self._h, _dptr(Pa), _dptr(Pb)))
        return Pa.reshape(n, n), Pb.reshape(n, n)

    def set_spin_densities(self, Pa, Pb):
        """Start spin densities of the next unrestricted calculate()."""
        Pa = np.ascontiguousarray(Pa, dtype=np.float64)
        Pb = np.ascontiguousarray(Pb, dtype=np.float64)
        self._check(lib().sg_set_spin_densities(self._h, _dptr(Pa), _dptr(Pb)))

    def beta_orbital_energies(self):
        """Beta orbital energies of an unrestricted calculation."""
        e = np.zeros(self._nao)
        self._check(lib().sg_get_beta_orbital_energies(self._h, _dptr(e)))
        return e

    def set_density(self, P):
        P = np.ascontiguousarray(P, dtype=np.float64)
        self._check(lib().sg_set_density(self._h, _dptr(P)))

    def clone(self):
        h = _VP()
        self._check(lib().sg_clone(self._h, ctypes.byref(h)))
        c = Calculator(self.method, _handle=h)
        c._n_atoms = self._n_atoms
        c._str = dict(self.settings._str)
        if hasattr(self, "_mask"):
            c._mask = self._mask
        return c


def get_calculator(method="PM6"):
    """Equivalent of ModuleManager.get('calculator', method) in the reference."""
    return Calculator(method)


def _flatten(molecules):
    n_atoms = np.array([len(z) for z, _ in molecules], dtype=np.int32)
    Z = np.ascontiguousarray(np.concatenate([np.asarray(z) for z, _ in molecules]), dtype=np.int32)
    X = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64).reshape(-1) for _, x in molecules]))
    return n_atoms, Z, X


class Batch:
    """Many independent molecules resident on the device.

    molecules: list of (atomic_numbers, positions_bohr).  run() enqueues the
    integral, SCF and (optionally) gradient kernels; results() waits and
    copies the energies / gradients back.
    """

    SCF_PATHS = {"auto": 0, "batched": 1, "large": 2, "large_mixed": 3}

    def __init__(self, method, molecules, charges=None, scc=1e-7, rmsd=1e-5, max_iter=100, scf_path="auto",
                 multiplicities=None, unrestricted=None):
        """multiplicities / unrestricted: an unrestricted (UHF) batch when unrestricted is
        True, or when it is None and some multiplicity differs from 1 (the reference's
        spin_mode "any")."""
        L = lib()
        self.n_atoms, Z, X = _flatten(molecules)
        ch = None if charges is None else np.ascontiguousarray(charges, dtype=np.int32)
        mult = None if multiplicities is None else np.ascontiguousarray(multiplicities, dtype=np.int32)
        if unrestricted is None:
            unrestricted = mult is not None and bool(np.any(mult != 1))
        self.unrestricted = bool(unrestricted)
        h = _VP()
        if self.unrestricted:
            rc = L.sg_batch_create_unrestricted(method.encode(), len(molecules), _iptr(self.n_atoms), _iptr(Z),
                                                _dptr(X), _iptr(ch) if ch is not None else None,
                                                _iptr(mult) if mult is not None else None, ctypes.byref(h))
        elif mult is not None and np.any(mult != 1):
            raise ValueError("a restricted batch needs multiplicity 1 for every molecule")
        else:
            rc = L.sg_batch_create(method.encode(), len(molecules), _iptr(self.n_atoms), _iptr(Z), _dptr(X),
                                   _iptr(ch) if ch is not None else None, ctypes.byref(h))
        if rc != 0:
            raise SparrowError(rc, L.sg_batch_last_error(None).decode())
        self._h = h
        self.n_molecules = len(molecules)
        self._check(L.sg_batch_set_scf(h, scc, rmsd, max_iter))
        self.set_scf_path(scf_path)
        self._props = SG_PROP_ENERGY

    def set_scf_path(self, path):
        """"auto", "batched", "large" (one NDDO molecule, grid-wide FP64 SCF with
        SP2 purification) or "large_mixed" (split-BF16 purification products
        until rms(dP) < 1e-5, then FP64)."""
        if path not in self.SCF_PATHS:
            raise ValueError(f"unknown scf_path {path!r}")
        self._check(lib().sg_batch_set_scf_path(self._h, self.SCF_PATHS[path]))

    ORBITAL_UPDATES = {"exact": 0, "hybrid": 1, "rotation": 2}

    def set_tuning(self, orbital_update=None, diis_size=None):
        """Override the library's tuned table for every molecule of the batch:
        orbital_update "exact" (tridiagonal diagonalisation every iteration),
        "hybrid" (tridiagonal start, then occupied-virtual rotations) or
        "rotation" (Jacobi start, then rotations); diis_size 1..6.  None keeps
        the table's choice."""
        mode = -1 if orbital_update is None else self.ORBITAL_UPDATES[orbital_update]
        self._check(lib().sg_batch_set_tuning(self._h, mode, -1 if diis_size is None else int(diis_size)))

    def set_mixed_switch(self, rmsd):
        """rms(dP) below which "large_mixed" purifies in FP64 (default 1e-5)."""
        self._check(lib().sg_batch_set_mixed_switch(self._h, rmsd))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.sg_batch_destroy(self._h)
            self._h = None

    def _check(self, rc, allow=()):
        if rc != 0 and rc not in allow:
            raise SparrowError(rc, lib().sg_batch_last_error(self._h).decode())
        return rc

    def set_positions(self, xyz_bohr_all):
        x = np.ascontiguousarray(xyz_bohr_all, dtype=np.float64).reshape(-1)
        self._check(lib().sg_batch_set_positions(self._h, _dptr(x)))

    def run(self, gradients=False):
        self._props = SG_PROP_ENERGY | (SG_PROP_GRADIENTS if gradients else 0)
        self._check(lib().sg_batch_run(self._h, self._props))

    def results(self):
        n = self.n_molecules
        e = np.zeros(n)
        it = np.zeros(n, dtype=np.int32)
        conv = np.zeros(n, dtype=np.int32)
        g = np.zeros(3 * int(self.n_atoms.sum())) if self._props & SG_PROP_GRADIENTS else None
        rc = lib().sg_batch_results(self._h, _dptr(e), _dptr(g) if g is not None else None, _iptr(it), _iptr(conv))
        self._check(rc, allow=(SG_ERR_NOT_CONVERGED,))
        grads = None
        if g is not None:
            grads = np.split(g.reshape(-1, 3), np.cumsum(self.n_atoms)[:-1])
        return e, grads, it, conv.astype(bool)

    def excitations(self, nroots=8, triplet=False):
        """TD-DFTB of every molecule after run() on a DFTB batch: omega [n, nroots]
        (Hartree), transition dipoles [n, nroots, 3] (e bohr), status [n]
        (0 ok, 1 Davidson not converged, 2-4 failures)."""
        n = self.n_molecules
        om = np.zeros(n * nroots)
        dp = np.zeros(3 * n * nroots)
        st = np.zeros(n, dtype=np.int32)
        self._check(lib().sg_batch_excitations(self._h, nroots, 1 if triplet else 0, _dptr(om),
                                               dp.ctypes.data_as(_VP), st.ctypes.data_as(_VP)),
                    allow=(SG_ERR_NOT_CONVERGED,))
        return om.reshape(n, nroots), dp.reshape(n, nroots, 3), st

    def excitation_cycles(self):
        """SM cycles per molecule of the last excitations(): canonical orbitals,
        transition charges, Davidson ([n, 3])."""
        c = np.zeros(3 * self.n_molecules, dtype=np.int64)
        self._check(lib().sg_batch_excitation_cycles(self._h, c.ctypes.data_as(_VP)))
        return c.reshape(-1, 3)

    @property
    def launches(self):
        return lib().sg_batch_launches(self._h)

    def stage_times(self):
        """Device ms of the last run: pair integrals, one-electron, SCF, gradient."""
        ms = np.zeros(4)
        self._check(lib().sg_batch_stage_times(self._h, _dptr(ms)))
        return ms

    def record_event(self, slot):
        self._check(lib().sg_batch_record_event(self._h, slot))

    def elapsed_ms(self, s0, s1):
        v = ctypes.c_double()
        self._check(lib().sg_batch_event_elapsed(self._h, s0, s1, ctypes.byref(v)))
        return v.value

    def scf_stats(self):
        """Per molecule: full diagonalisations, Jacobi sweeps, SM cycles per SCF phase
        (Fock build, DIIS, occupied-virtual rotation, full diagonalisation, density)."""
        n = self.n_molecules
        nf = np.zeros(n, dtype=np.int32)
        sw = np.zeros(n, dtype=np.int32)
        cyc = np.zeros(5 * n, dtype=np.int64)
        self._check(lib().sg_batch_scf_stats(self._h, _iptr(nf), _iptr(sw),
                                              cyc.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return nf, sw, cyc.reshape(n, 5)

    def convergence(self):
        """Per molecule, of the last SCF iteration: |Delta E| (Hartree) and rms(Delta P)."""
        n = self.n_molecules
        de = np.zeros(n)
        dp = np.zeros(n)
        self._check(lib().sg_batch_convergence(self._h, _dptr(de), _dptr(dp)))
        return de, dp

    def transfer_bytes(self):
        h, d = ctypes.c_int64(), ctypes.c_int64()
        self._check(lib().sg_batch_transfer_bytes(self._h, ctypes.byref(h), ctypes.byref(d)))
        return h.value, d.value

    @property
    def stream(self):
        return lib().sg_batch_stream(self._h)


def tuning_table():
    """The library's tuned SCF choices per molecule-size bin of 32 AOs:
    list of (first AO count of the bin, orbital update, Pulay subspace size)."""
    names = {v: k for k, v in Batch.ORBITAL_UPDATES.items()}
    modes = np.zeros(64, dtype=np.int32)
    diis = np.zeros(64, dtype=np.int32)
    n = lib().sg_tuning_table(_iptr(modes), _iptr(diis), 64)
    return [(32 * k, names[int(modes[k])], int(diis[k])) for k in range(n)]


def element_parameters(method, Z):
    """Runtime (atomic-unit) parameters of element Z as the engine uploads them.

    method is "METHOD" or "METHOD:parameters" (a parameters.json path for
    MNDO/AM1/PM6; an embedded set name or a Slater-Koster directory for DFTB).
    NDDO: dict with nao, core, Uss, Upp, betaS, betaP, alpha, D (D_sp1, D_pp2),
    rho (ss0, sp1, pp0, pp2), pcore, gss, gsp, gpp, gp2, hsp, hpp, s_exp,
    s_coef, p_exp, p_coef, gauss (list of (a, b, c)).  DFTB: dict with nao,
    occupation, es, ep, U, hubbard_derivative, W, has_W.  Host only.
    """
    L = lib()
    out = np.zeros(max(SG_NDDO_ELEMENT_VALUES, SG_DFTB_ELEMENT_VALUES))
    err = ctypes.create_string_buffer(512)
    rc = L.sg_element_parameters(method.encode(), int(Z), _dptr(out), out.size, err, 512)
    if rc != 0:
        raise SparrowError(rc, err.value.decode())
    if method.split(":")[0].upper().startswith("DFTB"):
        keys = ["nao", "occupation", "es", "ep", "U", "hubbard_derivative", "W", "has_W"]
        return dict(zip(keys, out[:SG_DFTB_ELEMENT_VALUES].tolist()))
    v = out
    ng = int(v[44])
    return {"nao": int(v[0]), "core": v[1], "Uss": v[2], "Upp": v[3], "betaS": v[4], "betaP": v[5], "alpha": v[6],
            "D": v[7:9].copy(), "rho": v[9:13].copy(), "pcore": v[13], "gss": v[14], "gsp": v[15], "gpp": v[16],
            "gp2": v[17], "hsp": v[18], "hpp": v[19], "s_exp": v[20:26].copy(), "s_coef": v[26:32].copy(),
            "p_exp": v[32:38].copy(), "p_coef": v[38:44].copy(),
            "gauss": [(v[45 + k], v[49 + k], v[53 + k]) for k in range(ng)], "vector": v[:20].copy()}


def diatomic_parameters(method, Z1, Z2):
    """PM6 diatomic core-repulsion pair (alpha_AB in atomic units, x_AB).  Host only."""
    L = lib()
    out = np.zeros(2)
    err = ctypes.create_string_buffer(512)
    rc = L.sg_diatomic_parameters(method.encode(), int(Z1), int(Z2), _dptr(out), err, 512)
    if rc != 0:
        raise SparrowError(rc, err.value.decode())
    return float(out[0]), float(out[1])


def hessian(method, atomic_numbers, xyz_bohr, charge=0, multiplicity=1, unrestricted=False, scc=1e-7, rmsd=1e-5,
            max_iter=100, step=0.01):
    """Semi-numerical Hessian (Hartree/bohr^2): symmetrised central differences of
    analytic gradients, the 6 n_atoms displaced geometries in one batch.  Returns
    (H of shape (3n, 3n), number of displaced SCFs that did not converge)."""
    L = lib()
    Z = np.ascontiguousarray(atomic_numbers, dtype=np.int32)
    X = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1)
    n3 = 3 * Z.size
    H = np.zeros(n3 * n3)
    nc = ctypes.c_int32()
    err = ctypes.create_string_buffer(512)
    rc = L.sg_calculate_hessian(method.encode(), Z.size, _iptr(Z), _dptr(X), int(charge), int(multiplicity),
                                1 if unrestricted else 0, scc, rmsd, max_iter, step, _dptr(H), ctypes.byref(nc), err,
                                512)
    if rc != 0:
        raise SparrowError(rc, err.value.decode())
    return H.reshape(n3, n3), nc.value


def batch_calculate(method, molecules, charges=None, scc=1e-7, rmsd=1e-5, max_iter=100, gradients=False):
    """One call from host arrays to host results (sg_batch_calculate)."""
    L = lib()
    n_atoms, Z, X = _flatten(molecules)
    n = len(molecules)
    ch = None if charges is None else np.ascontiguousarray(charges, dtype=np.int32)
    e = np.zeros(n)
    it = np.zeros(n, dtype=np.int32)
    conv = np.zeros(n, dtype=np.int32)
    g = np.zeros(3 * int(n_atoms.sum())) if gradients else None
    msg = ctypes.create_string_buffer(512)
    props = SG_PROP_ENERGY | (SG_PROP_GRADIENTS if gradients else 0)
    rc = L.sg_batch_calculate(method.encode(), n, _iptr(n_atoms), _iptr(Z), _dptr(X),
                              _iptr(ch) if ch is not None else None, scc, rmsd, max_iter, props, _dptr(e),
                              _dptr(g) if g is not None else None, _iptr(it), _iptr(conv), msg, 512)
    if rc != 0 and rc != SG_ERR_NOT_CONVERGED:
        raise SparrowError(rc, msg.value.decode())
    grads = np.split(g.reshape(-1, 3), np.cumsum(n_atoms)[:-1]) if g is not None else None
    return e, grads, it, conv.astype(bool)


def flatten_molecules(molecules):
    """(n_atoms, Z, xyz) flat arrays of a list of (atomic_numbers, positions_bohr):
    the layout batch_calculate_flat and the C-ABI batch entry points take."""
    return _flatten(molecules)


def batch_calculate_flat(method, n_atoms, Z, xyz_bohr, charges=None, scc=1e-7, rmsd=1e-5, max_iter=100,
                         gradients=False):
    """batch_calculate on flat host arrays (n_atoms [n], Z [sum n_atoms], xyz
    [3 sum n_atoms], bohr): no per-molecule Python work on either side.
    Returns (energies [n], gradients [sum n_atoms, 3] or None, iterations [n],
    converged [n])."""
    L = lib()
    n_atoms = np.ascontiguousarray(n_atoms, dtype=np.int32)
    Z = np.ascontiguousarray(Z, dtype=np.int32)
    X = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1)
    if X.size != 3 * Z.size or int(n_atoms.sum()) != Z.size:
        raise ValueError("n_atoms, Z and xyz sizes disagree")
    n = n_atoms.size
    ch = None if charges is None else np.ascontiguousarray(charges, dtype=np.int32)
    e = np.zeros(n)
    it = np.zeros(n, dtype=np.int32)
    conv = np.zeros(n, dtype=np.int32)
    g = np.zeros(3 * Z.size) if gradients else None
    msg = ctypes.create_string_buffer(512)
    props = SG_PROP_ENERGY | (SG_PROP_GRADIENTS if gradients else 0)
    rc = L.sg_batch_calculate(method.encode(), n, _iptr(n_atoms), _iptr(Z), _dptr(X),
                              _iptr(ch) if ch is not None else None, scc, rmsd, max_iter, props, _dptr(e),
                              _dptr(g) if g is not None else None, _iptr(it), _iptr(conv), msg, 512)
    if rc != 0 and rc != SG_ERR_NOT_CONVERGED:
        raise SparrowError(rc, msg.value.decode())
    return e, (g.reshape(-1, 3) if g is not None else None), it, conv.astype(bool)


def calculate_static(method, atomic_numbers, xyz_bohr, charge=0, scc=1e-7, rmsd=1e-5, max_iter=100,
                     gradients=False, stream=None):
    """One molecule through the allocation-free entry point (sg_calculate_static).

    All device scratch is a fixed array inside the library (at most
    SG_STATIC_MAX_ATOMS atoms and SG_STATIC_MAX_AOS AOs); overlapping calls
    race.  stream: an integer cudaStream_t handle or None for the default
    stream.  Returns (energy, gradient (n, 3) or None, iterations, converged).
    """
    L = lib()
    Z = np.ascontiguousarray(atomic_numbers, dtype=np.int32)
    X = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1)
    if X.size != 3 * Z.size:
        raise ValueError("positions must have 3 entries per atom")
    e = ctypes.c_double(0.0)
    it = ctypes.c_int32(0)
    conv = ctypes.c_int32(0)
    g = np.zeros(3 * Z.size) if gradients else None
    msg = ctypes.create_string_buffer(512)
    props = SG_PROP_ENERGY | (SG_PROP_GRADIENTS if gradients else 0)
    rc = L.sg_calculate_static(method.encode(), int(Z.size), _iptr(Z), _dptr(X), int(charge), scc, rmsd, max_iter,
                               props, stream, ctypes.byref(e), _dptr(g) if g is not None else None,
                               ctypes.byref(it), ctypes.byref(conv), msg, 512)
    if rc != 0 and rc != SG_ERR_NOT_CONVERGED:
        raise SparrowError(rc, msg.value.decode())
    return e.value, (g.reshape(-1, 3) if g is not None else None), it.value, bool(conv.value)


class ServerResult:
    """Result of one served request: energy (Hartree), gradients ((n, 3)
    Hartree/bohr or None), iterations, status (0, or 6 = not converged with
    results), latency_s (completion - submission)."""

    def __init__(self, energy, gradients, iterations, status, latency_s):
        self.energy = energy
        self.gradients = gradients
        self.iterations = iterations
        self.status = status
        self.latency_s = latency_s

    @property
    def successful_calculation(self):
        return self.status == 0


class Server:
    """Continuous-batching request server on the current GPU (sg_server_*).

    submit() queues a single point (and gradient); requests that arrive while
    others run are admitted into free batch slots as memory allows."""

    def __init__(self, device_budget_gb=16.0, slots=2, max_batch=4096, scc=1e-7, rmsd=1e-5, max_iter=100):
        h = _VP()
        rc = lib().sg_server_create(int(device_budget_gb * 1e9), slots, max_batch, scc, rmsd, max_iter,
                                    ctypes.byref(h))
        if rc != 0:
            raise SparrowError(rc, lib().sg_server_last_error().decode())
        self._h = h
        self._req = {}

    def submit(self, method, atomic_numbers, xyz_bohr, charge=0, gradients=True, multiplicity=1):
        """Queue one molecule; multiplicity != 1 runs the unrestricted SCF."""
        Z = np.ascontiguousarray(atomic_numbers, dtype=np.int32)
        X = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1)
        rid = ctypes.c_int64()
        props = SG_PROP_ENERGY | (SG_PROP_GRADIENTS if gradients else 0)
        rc = lib().sg_server_submit_spin(self._h, method.encode(), int(Z.size), _iptr(Z), _dptr(X), int(charge),
                                         int(multiplicity), props, ctypes.byref(rid))
        if rc != 0:
            raise SparrowError(rc, lib().sg_server_last_error().decode())
        self._req[rid.value] = (int(Z.size), gradients)
        return rid.value

    def _result(self, rid, fn, *args):
        n, grads = self._req[rid]
        e = ctypes.c_double()
        it = ctypes.c_int32()
        st = ctypes.c_int32()
        lat = ctypes.c_double()
        g = np.zeros(3 * n) if grads else None
        rc = fn(self._h, rid, *args, ctypes.byref(e), _dptr(g) if g is not None else None, ctypes.byref(it),
                ctypes.byref(st), ctypes.byref(lat))
        if rc in (SG_PENDING, SG_ERR_TIMEOUT):
            return None
        if rc != 0:
            raise SparrowError(rc, lib().sg_server_last_error().decode())
        del self._req[rid]
        if st.value not in (0, SG_ERR_NOT_CONVERGED):
            raise SparrowError(st.value, lib().sg_server_last_error().decode())
        return ServerResult(e.value, g.reshape(-1, 3) if g is not None else None, it.value, st.value, lat.value)

    def wait(self, rid, timeout=None):
        """Block until request rid is done (None on timeout)."""
        return self._result(rid, lib().sg_server_wait, -1.0 if timeout is None else float(timeout))

    def poll(self, rid):
        """The result of request rid, or None while it is in flight."""
        return self._result(rid, lib().sg_server_poll)

    def drain(self):
        lib().sg_server_drain(self._h)

    def stats(self):
        v = [ctypes.c_int64() for _ in range(4)]
        lib().sg_server_stats(self._h, *[ctypes.byref(x) for x in v])
        return dict(zip(("submitted", "completed", "batches", "max_batch"), (x.value for x in v)))

    def close(self):
        if getattr(self, "_h", None):
            lib().sg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
