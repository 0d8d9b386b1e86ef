"""Run-time parameter files: NDDO parameters.json and DFTB Slater-Koster directories.

The reference reads its method parameters at initialize() from the
"method_parameters" setting (Nddo/Pm6/Wrapper/PM6MethodWrapper.cpp:62-75,
Dftb/Utils/DFTBCommon.cpp:112-120).  CPU tests: the engine's reading of the
files (sg_element_parameters, sg_diatomic_parameters and the host checks of
sg_batch_create) against the embedded sets, bit for bit, and against the
oracle given the same records.  GPU tests: energies through a file equal the
embedded set's bit for bit (gradients to 1e-12: their atomic accumulation
order varies), and a changed set matches the oracle within 1e-6 Hartree /
1e-5 Hartree/bohr.
"""
import copy
import os

import numpy as np
import pytest

import sparrow_b200
from sparrow_b200 import geometry
from tests import oracle_lib as O
from tests import param_sets as PS

E_TOL = 1e-6
G_TOL = 1e-5
CHON = [1, 6, 7, 8]


def _engine_vector(spec, Z):
    p = sparrow_b200.element_parameters(spec, Z)
    return np.concatenate([p["vector"], p["s_exp"], p["s_coef"], p["p_exp"], p["p_coef"],
                           np.array([len(p["gauss"])] + [x for g in p["gauss"] for x in g])])


@pytest.fixture
def oracle_override():
    used = []

    def apply(method, records):
        used.append(method)
        O.set_parameters(method, records)

    yield apply
    for m in used:
        O.set_parameters(m, None)


# ---------------------------------------------------------------------------
# NDDO parameters.json
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("method", ["MNDO", "AM1", "PM6"])
def test_nddo_file_of_the_embedded_set_is_bit_identical(method, tmp_path):
    atoms, diat = PS.nddo_embedded(method)
    path = str(tmp_path / "parameters.json")
    PS.write_nddo_json(path, atoms, diat)
    compared = 0
    for z in sorted(atoms):
        try:
            ref = _engine_vector(method, z)
        except sparrow_b200.SparrowError as e:
            assert e.code == 3  # elements with d shells
            with pytest.raises(sparrow_b200.SparrowError) as ei:
                _engine_vector(method + ":" + path, z)
            assert ei.value.code == 3
            continue
        got = _engine_vector(method + ":" + path, z)
        assert np.array_equal(ref, got), z
        compared += 1
    assert compared >= 10
    if method == "PM6":
        for a in CHON + [9]:
            for b in CHON + [9]:
                assert sparrow_b200.diatomic_parameters("PM6", a, b) == \
                    sparrow_b200.diatomic_parameters("PM6:" + path, a, b)


def _changed_pm6():
    atoms, diat = PS.nddo_embedded("PM6")
    emb = copy.deepcopy(atoms)
    atoms[8]["v"]["zetaS"] *= 1.07
    atoms[8]["v"]["zetaP"] *= 0.93
    atoms[1]["v"]["zetaS"] *= 1.10
    atoms[6]["v"]["Uss"] += 0.1
    atoms[7]["v"]["gss"] *= 1.02
    atoms[7]["v"]["hsp"] *= 0.9
    atoms[6]["v"]["betaP"] -= 0.2
    atoms[1]["ga"][0] *= 1.3
    for d in diat:
        if {d["z1"], d["z2"]} == {1, 8}:
            d["factor"] *= 1.05
    return atoms, diat, emb


def test_changed_exponents_rescale_sto6g_and_match_the_oracle(tmp_path, oracle_override):
    atoms, diat, emb = _changed_pm6()
    path = str(tmp_path / "pm6-changed.json")
    PS.write_nddo_json(path, atoms, diat)
    oracle_override("PM6", PS.oracle_records(atoms, diat, emb))
    for z in CHON:
        eng = sparrow_b200.element_parameters("PM6:" + path, z)
        ref = O.element_params("PM6", z)
        assert np.allclose(eng["vector"], ref, rtol=1e-13, atol=0), z
        for l, (en, cn) in enumerate([("s_exp", "s_coef"), ("p_exp", "p_coef")]):
            if z == 1 and l == 1:
                continue
            e, c = PS.rescaled_sto6g(emb[z], l, atoms[z]["v"]["zetaS" if l == 0 else "zetaP"])
            assert np.allclose(eng[en], e, rtol=1e-15, atol=0) and np.allclose(eng[cn], c, rtol=1e-15, atol=0)
    # the scaling law itself: exponents ~ zeta^2, coefficients ~ zeta^(l + 3/2)
    base = sparrow_b200.element_parameters("PM6", 8)
    new = sparrow_b200.element_parameters("PM6:" + path, 8)
    assert np.allclose(new["s_exp"] / base["s_exp"], 1.07 ** 2, rtol=1e-14)
    assert np.allclose(new["p_coef"] / base["p_coef"], 0.93 ** 2.5, rtol=1e-14)
    a_ref = sparrow_b200.diatomic_parameters("PM6", 1, 8)
    a_new = sparrow_b200.diatomic_parameters("PM6:" + path, 8, 1)
    assert a_new[0] == a_ref[0] and abs(a_new[1] / a_ref[1] - 1.05) < 1e-14


def _mols():
    return [(np.array([8, 1, 1]), np.array([[0, 0, 0], [0, 1.43, 1.1], [0, -1.43, 1.1]]))]


def test_nddo_file_errors(tmp_path):
    mols = _mols()
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.Batch("PM6:" + str(tmp_path / "missing.json"), mols)
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS and "does not exist" in str(ei.value)
    bad = tmp_path / "truncated.json"
    bad.write_text('{"atomic": [{"key": 1, "value": {"pack": {')
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.Batch("PM6:" + str(bad), mols)
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS and "line" in str(ei.value)
    atoms, diat = PS.nddo_embedded("PM6")
    good = str(tmp_path / "hc.json")
    PS.write_nddo_json(good, atoms, diat, elements={1, 6})
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.Batch("PM6:" + good, mols)  # no oxygen in the file
    assert ei.value.code == 3 and "Z=8" in str(ei.value)
    nogss = tmp_path / "nogss.json"
    text = open(good).read().replace('"gss"', '"gss_"', 1)
    nogss.write_text(text)
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.element_parameters("PM6:" + str(nogss), 1)
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS and "'gss'" in str(ei.value)
    five = copy.deepcopy(atoms)
    five[1]["n_gauss"] = 5
    five[1]["ga"] += [0.1]
    five[1]["gb"] += [1.0]
    five[1]["gc"] += [1.0]
    p5 = str(tmp_path / "five.json")
    PS.write_nddo_json(p5, five, diat, elements={1})
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.element_parameters("PM6:" + p5, 1)
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS and "four Gaussian" in str(ei.value)
    nodiat = str(tmp_path / "nodiat.json")
    PS.write_nddo_json(nodiat, atoms, [d for d in diat if {d["z1"], d["z2"]} != {1, 8}], elements={1, 8})
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.Batch("PM6:" + nodiat, mols)
    assert ei.value.code == 3 and "diatomic" in str(ei.value)


def test_calculator_setting_reports_a_bad_file(tmp_path):
    c = sparrow_b200.get_calculator("AM1")
    Z, X = _mols()[0]
    c.set_structure(Z, X)
    c.settings["method_parameters"] = str(tmp_path / "nothing.json")
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        c.calculate()
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS


def test_file_changes_are_picked_up(tmp_path):
    atoms, diat = PS.nddo_embedded("AM1")
    path = str(tmp_path / "am1.json")
    PS.write_nddo_json(path, atoms, diat, elements=set(CHON))
    u0 = sparrow_b200.element_parameters("AM1:" + path, 6)["Uss"]
    atoms[6]["v"]["Uss"] += 1.0
    PS.write_nddo_json(path, atoms, diat, elements=set(CHON))
    os.utime(path, ns=(os.stat(path).st_mtime_ns + 10**9,) * 2)
    u1 = sparrow_b200.element_parameters("AM1:" + path, 6)["Uss"]
    assert abs((u1 - u0) * O.ev_per_hartree() - 1.0) < 1e-12


# ---------------------------------------------------------------------------
# DFTB Slater-Koster directories
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("method,set_name", [("DFTB2", "mio-1-1"), ("DFTB3", "3ob-3-1"), ("DFTB3", "3ob-2-1")])
def test_skf_directory_of_an_embedded_set_is_identical(method, set_name, tmp_path):
    d = str(tmp_path / set_name)
    PS.write_skf_directory(d, set_name)
    for z in CHON:
        assert sparrow_b200.element_parameters(method + ":" + set_name, z) == \
            sparrow_b200.element_parameters(method + ":" + d, z), z


def test_skf_directory_errors(tmp_path):
    co = [(np.array([6, 8]), np.array([[0, 0, 0], [0, 0, 2.13]]))]
    d1 = str(tmp_path / "no-co")
    PS.write_skf_directory(d1, "mio-1-1", skip_pairs={(6, 8)})
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.Batch("DFTB2:" + d1, co)
    assert ei.value.code == 3 and "Slater-Koster file" in str(ei.value)
    d2 = str(tmp_path / "no-hubbard")
    PS.write_skf_directory(d2, "3ob-3-1", hubbard=False)
    assert sparrow_b200.element_parameters("DFTB2:" + d2, 6)["nao"] == 4
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.Batch("DFTB3:" + d2, co)
    assert ei.value.code == 3 and "Hubbard derivative" in str(ei.value)
    d3 = str(tmp_path / "short-line")
    PS.write_skf_directory(d3, "mio-1-1", variants=False)
    hh = os.path.join(d3, "H-H.skf")
    lines = open(hh).read().splitlines()
    lines[5] = ", ".join(lines[5].split(", ")[:3])
    open(hh, "w").write("\n".join(lines) + "\n")
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.element_parameters("DFTB2:" + d3, 1)
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS and "fewer than 20" in str(ei.value)
    d4 = str(tmp_path / "bad-forward")
    PS.write_skf_directory(d4, "mio-1-1", variants=False)
    open(os.path.join(d4, "C-O.skf"), "w").write("CO-elsewhere.skf\n")
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.element_parameters("DFTB2:" + d4, 6)
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS and "forwarding" in str(ei.value)
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.element_parameters("DFTB2:" + str(tmp_path / "no-such-dir"), 6)
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS


# ---------------------------------------------------------------------------
# GPU: energies and gradients
# ---------------------------------------------------------------------------
def _batch_results(spec, mols, **kw):
    b = sparrow_b200.Batch(spec, mols, scc=1e-9, rmsd=1e-8, max_iter=300, **kw)
    b.run(gradients=True)
    return b.results()


def _test_molecules():
    mols = [(z, geometry.to_bohr(x)) for z, x in geometry.alkane_batch(4, seed=21, n_min=2, n_max=6)]
    Z, xa = geometry.water_cluster(4, seed=5)
    mols.append((Z, geometry.to_bohr(xa)))
    # N-H and C-N pairs
    mols.append((np.array([7, 1, 1, 1]), np.array([[0, 0, 0.0], [1.77, 0, 0.72], [-0.885, 1.533, 0.72],
                                                  [-0.885, -1.533, 0.72]])))
    mols.append((np.array([6, 7, 1]), np.array([[0, 0, 0.0], [0, 0, 2.19], [0, 0, -2.02]])))
    return mols


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["PM6", "AM1"])
def test_gpu_file_of_the_embedded_set_gives_identical_results(method, tmp_path):
    atoms, diat = PS.nddo_embedded(method)
    path = str(tmp_path / "p.json")
    PS.write_nddo_json(path, atoms, diat)
    mols = _test_molecules()
    e0, g0, it0, c0 = _batch_results(method, mols)
    e1, g1, it1, c1 = _batch_results(method + ":" + path, mols)
    assert c0.all() and c1.all()
    # gradients are gathered with atomic adds, so their last bits follow the summation order
    assert np.array_equal(e0, e1) and np.array_equal(it0, it1)
    assert max(np.max(np.abs(a - b)) for a, b in zip(g0, g1)) < 1e-12


@pytest.mark.gpu
def test_gpu_changed_pm6_set_matches_the_oracle(tmp_path, oracle_override):
    atoms, diat, emb = _changed_pm6()
    path = str(tmp_path / "pm6-changed.json")
    PS.write_nddo_json(path, atoms, diat)
    oracle_override("PM6", PS.oracle_records(atoms, diat, emb))
    mols = _test_molecules()
    e, g, it, conv = _batch_results("PM6:" + path, mols)
    e_emb = _batch_results("PM6", mols)[0]
    assert conv.all()
    for i, (Z, x) in enumerate(mols):
        ref = O.scf("PM6", Z, x)
        assert ref["converged"]
        assert abs(e[i] - ref["energy"]) < E_TOL, i
        assert np.max(np.abs(g[i] - ref["gradient"])) < G_TOL, i
        assert abs(e[i] - e_emb[i]) > 1e-4, i  # the changed parameters took effect


@pytest.mark.gpu
@pytest.mark.parametrize("method,set_name", [("DFTB3", "3ob-3-1"), ("DFTB2", "mio-1-1")])
def test_gpu_skf_directory_gives_identical_results(method, set_name, tmp_path):
    d = str(tmp_path / set_name)
    PS.write_skf_directory(d, set_name)
    mols = _test_molecules()
    e0, g0, _, c0 = _batch_results(method + ":" + set_name, mols)
    e1, g1, _, c1 = _batch_results(method + ":" + d, mols)
    assert c0.all() and c1.all()
    assert np.array_equal(e0, e1) and max(np.max(np.abs(a - b)) for a, b in zip(g0, g1)) < 1e-12
