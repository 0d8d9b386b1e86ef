"""C-ABI library checks that need no GPU: it loads, exports every declared
entry point, and rejects bad input on the host before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

import sparrow_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "sparrow_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const char\*|int32_t|void\*|void)\s+(sg_\w+)\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = sparrow_b200.lib()
    names = _declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n


def test_version_string():
    assert b"sm_100a" in sparrow_b200.lib().sg_version()


def test_unknown_method_is_rejected():
    with pytest.raises(sparrow_b200.SparrowError) as e:
        sparrow_b200.get_calculator("HF")
    assert e.value.code == 2


def test_settings_round_trip_and_validation():
    c = sparrow_b200.get_calculator("AM1")
    assert c.settings["self_consistence_criterion"] == pytest.approx(1e-7)
    assert c.settings["density_rmsd_criterion"] == pytest.approx(1e-5)
    assert c.settings["max_scf_iterations"] == 100
    c.settings["molecular_charge"] = 1
    c.settings["density_rmsd_criterion"] = 1e-8
    assert c.settings["molecular_charge"] == 1
    assert c.settings["density_rmsd_criterion"] == pytest.approx(1e-8)
    with pytest.raises(sparrow_b200.SparrowError):
        c.settings["max_scf_iterations"] = 0
    with pytest.raises(sparrow_b200.SparrowError):
        c.settings["scf_mixer"] = "ediis"
    with pytest.raises(KeyError):
        c.settings["no_such_key"] = 1
    assert c.settings["scf_path"] == "auto"
    for path in ("batched", "large", "large_mixed", "auto"):
        c.settings["scf_path"] = path
        assert c.settings["scf_path"] == path
    with pytest.raises(sparrow_b200.SparrowError):
        c.settings["scf_path"] = "fast"
    assert c.settings["scf_path"] == "auto"


def test_empty_structure_and_bad_input_fail_on_host():
    c = sparrow_b200.get_calculator("PM6")
    with pytest.raises(sparrow_b200.SparrowError) as e:
        c.calculate()
    assert e.value.code == 4
    with pytest.raises(ValueError):
        c.set_structure([1, 1], np.zeros((3, 3)))
    # no results before a calculation
    L = sparrow_b200.lib()
    e_out = ctypes.c_double()
    assert L.sg_get_energy(c._h, ctypes.byref(e_out)) == 9


def test_clone_keeps_settings_and_structure():
    c = sparrow_b200.get_calculator("PM6")
    c.set_structure([8, 1, 1], np.array([[0, 0, 0], [1.8, 0, 0], [-0.4, 1.7, 0.0]]))
    c.settings["molecular_charge"] = 0
    c.settings["self_consistence_criterion"] = 1e-9
    d = c.clone()
    assert d.settings["self_consistence_criterion"] == pytest.approx(1e-9)
    assert np.allclose(d.positions, c.positions)


def test_excitation_entry_points_check_their_arguments():
    # argument checks happen on the host, before any device work
    L = sparrow_b200.lib()
    om = np.zeros(4)
    om_p = om.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert L.sg_calculate_excitations(None, 4, 0, om_p, None) == 1
    assert L.sg_batch_excitations(None, 4, 0, om_p, None, None) == 1
    assert L.sg_batch_set_scf_path(None, 2) == 1
    assert L.sg_batch_set_mixed_switch(None, 1e-5) == 1


def test_property_getters_check_their_arguments():
    # charges, dipole, Hessian and the open-shell getters: null arguments are
    # SG_ERR_INVALID_ARGUMENT, a handle without a calculation SG_ERR_NO_RESULTS
    L = sparrow_b200.lib()
    c = sparrow_b200.get_calculator("PM6")
    buf = np.zeros(64)
    p = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for name in ("sg_get_hessian", "sg_get_atomic_charges", "sg_get_dipole", "sg_get_beta_orbital_energies"):
        fn = getattr(L, name)
        assert fn(None, p) == 1, name
        assert fn(c._h, None) == 1, name
        assert fn(c._h, p) == 9, name
    assert L.sg_get_spin_densities(None, p, p) == 1
    assert L.sg_get_spin_densities(c._h, p, None) == 1
    assert L.sg_get_spin_densities(c._h, p, p) == 9
    assert L.sg_set_spin_densities(None, p, p) == 1
    assert L.sg_set_spin_densities(c._h, None, p) == 1


def test_electron_count_beyond_the_orbitals_is_rejected_on_host():
    # a charge that leaves more than two electrons per orbital (or overflows
    # the electron count) is SG_ERR_ODD_ELECTRONS before any device work, in
    # the batch entry points and in the allocation-free call
    L = sparrow_b200.lib()
    Z = np.array([8, 1, 1], dtype=np.int32)
    X = np.array([0.0, 0.0, 0.0, 1.8, 0.0, 0.0, -0.4, 1.7, 0.0])
    nat = np.array([3], dtype=np.int32)
    buf = ctypes.create_string_buffer(256)
    for charge in (-8, -(2 ** 31), -(2 ** 31 - 1)):
        ch = np.array([charge], dtype=np.int32)
        h = ctypes.c_void_p()
        rc = L.sg_batch_create(b"PM6", 1, nat.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                               Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                               X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               ch.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(h))
        assert rc == 5, (charge, rc)
        assert not h.value
        mult = np.array([1], dtype=np.int32)
        rc = L.sg_batch_create_unrestricted(b"PM6", 1, nat.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                            Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                            X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            ch.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                            mult.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(h))
        assert rc == 5, (charge, rc)
        e = ctypes.c_double()
        it = ctypes.c_int32()
        cv = ctypes.c_int32()
        rc = L.sg_calculate_static(b"PM6", 3, Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                   X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), charge, 1e-7, 1e-5, 50, 1,
                                   None, ctypes.byref(e), None, ctypes.byref(it), ctypes.byref(cv), buf, 256)
        assert rc == 5, (charge, rc, buf.value)
        assert b"orbital" in buf.value
    # a huge multiplicity overflows n_alpha in 32 bits: rejected the same way
    mult = np.array([2 ** 31 - 1], dtype=np.int32)
    ch = np.array([0], dtype=np.int32)
    h = ctypes.c_void_p()
    rc = L.sg_batch_create_unrestricted(b"PM6", 1, nat.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                        Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                        X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        ch.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                        mult.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(h))
    assert rc == 5
