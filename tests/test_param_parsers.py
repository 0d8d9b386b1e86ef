"""Robustness of the run-time parameter readers (host only, no device use).

parameters.json: numbers in exponent form and \\u escapes in member names
read to the same doubles; unknown members are ignored; syntax errors and
runaway nesting are reported with SG_ERR_PARAMETERS.  Slater-Koster files: Fortran-style
exponents (1.0D-3) are accepted in the atomic line and the integral rows (a
row that failed to parse would end the table early and fail the spline
check), and the element records read the same.
"""
import json
import os
import re

import numpy as np
import pytest

import sparrow_b200
from tests import param_sets as PS

CHON = [1, 6, 7, 8]


def _vector(spec, Z):
    p = sparrow_b200.element_parameters(spec, Z)
    return np.concatenate([p["vector"], p["s_exp"], p["s_coef"], p["p_exp"], p["p_coef"]])


def test_json_number_forms_escapes_and_unknown_members(tmp_path):
    atoms, diat = PS.nddo_embedded("PM6")
    path = str(tmp_path / "plain.json")
    PS.write_nddo_json(path, atoms, diat, elements=set(CHON))
    data = json.load(open(path))
    data["comment"] = {"note": ["free text", 1, None, True]}
    for a in data["atomic"]:
        a["value"]["pack"]["extra"] = "ignored"
    text = json.dumps(data)
    # every float in exponent form with 17 significant digits (the same doubles)
    text = re.sub(r"(?<![\w.])-?\d+\.\d+(?:e[-+]?\d+)?", lambda m: "%.16e" % float(m.group(0)), text)
    text = text.replace('"gss"', '"g\\u0073s"')
    other = tmp_path / "forms.json"
    other.write_text(text)
    for z in CHON:
        assert np.array_equal(_vector("PM6:" + path, z), _vector("PM6:" + str(other), z)), z


@pytest.mark.parametrize("text,fragment", [
    ('{"atomic": [1, 2,]}', "line"),
    ('{"atomic": [}', "line"),
    ('{"atomic": []} extra', "unexpected characters"),
    ('[' * 80 + ']' * 80, "nesting"),
    ('{"atomic": [{"key": 1.5, "value": {}}]}', "integer"),
])
def test_json_errors(tmp_path, text, fragment):
    p = tmp_path / "bad.json"
    p.write_text(text)
    with pytest.raises(sparrow_b200.SparrowError) as ei:
        sparrow_b200.element_parameters("PM6:" + str(p), 1)
    assert ei.value.code == sparrow_b200.SG_ERR_PARAMETERS and fragment in str(ei.value), str(ei.value)


def test_skf_fortran_exponents(tmp_path):
    d = str(tmp_path / "mio")
    PS.write_skf_directory(d, "mio-1-1", variants=False)
    ref = {z: sparrow_b200.element_parameters("DFTB2:" + d, z) for z in CHON}
    e = str(tmp_path / "mio-d")
    PS.write_skf_directory(e, "mio-1-1", variants=False)
    for name in os.listdir(e):
        if not name.endswith(".skf"):
            continue
        path = os.path.join(e, name)
        lines = open(path).read().splitlines()
        # integral rows and the atomic line: write each number as mantissa D exponent
        out = []
        for k, line in enumerate(lines):
            if 1 <= k and "Spline" not in line and not line.startswith("<") and re.match(r"^[-\d., *e]+$", line):
                line = re.sub(r"(?<![\w.*])(-?\d+\.\d+(?:e[-+]?\d+)?)(?![\w*])",
                              lambda m: ("%.17e" % float(m.group(1))).replace("e", "D"), line)
            out.append(line)
        open(path, "w").write("\n".join(out) + "\n")
    # the directory's modification time changes when files are replaced; read it fresh
    for z in CHON:
        assert sparrow_b200.element_parameters("DFTB2:" + e, z) == ref[z], z
