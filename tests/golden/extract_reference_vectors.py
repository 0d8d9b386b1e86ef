"""Extract the reference's NDDO known-answer vectors into nddo_known_answers.json.

The reference (qcscine/sparrow) pins its PM6/AM1 implementation with MOPAC
numbers written inline in its GoogleTest sources and with one Python binding
test.  This script reads those test sources as text and records, per test:
the geometry (Angstrom, or bohr for the Python test), the expected one-electron
matrix (eV), energies (eV or Hartree) and gradients, with the tolerance the
reference asserts and the source file:line it came from.

It runs only where the reference checkout exists (its path is the first argument);
the JSON it writes is committed and is what the tests read.

Usage: python tests/golden/extract_reference_vectors.py [reference_root]
"""
import json
import os
import re
import sys


def _reference_root():
    """The reference checkout, a required first command-line argument."""
    if len(sys.argv) < 2:
        sys.exit("usage: %s <path of the reference checkout>" % os.path.basename(sys.argv[0]))
    return sys.argv[1]

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "nddo_known_answers.json")

NUM = r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?"
XYZ_LINE = re.compile(r'"\s*([A-Z][a-z]?)\s+(' + NUM + r")\s+(" + NUM + r")\s+(" + NUM + r')\s*\\n"')


def test_blocks(text):
    """Yield (name, body, first_line) for every TEST_F in a GoogleTest file."""
    for m in re.finditer(r"TEST_F\(\s*\w+\s*,\s*(\w+)\s*\)\s*\{", text):
        start = m.end()
        depth = 1
        i = start
        while depth and i < len(text):
            if text[i] == "{":
                depth += 1
            elif text[i] == "}":
                depth -= 1
            i += 1
        yield m.group(1), text[start:i], text.count("\n", 0, m.start()) + 1


def parse_block(name, body, line, rel):
    rec = {"name": name, "source": "%s:%d" % (rel, line)}
    geo = XYZ_LINE.findall(body)
    if not geo:
        return None
    # only the first structure of a test (some tests read a second one)
    first_stream = body.split("XyzStreamHandler::read")[0]
    geo = XYZ_LINE.findall(first_stream)
    rec["elements"] = [g[0] for g in geo]
    rec["xyz_angstrom"] = [[float(g[1]), float(g[2]), float(g[3])] for g in geo]
    rec["unrestricted"] = "setUnrestrictedCalculation(true)" in body
    m = re.search(r"setMolecularCharge\((-?\d+)\)", body)
    rec["charge"] = int(m.group(1)) if m else 0
    m = re.search(r"expected\s*<<\s*([^;]+);", body)
    if m and "isApprox" in body:
        rec["one_electron_ev"] = [float(x) for x in re.findall(NUM, m.group(1))]
        t = re.search(r"isApprox\(expected\s*/\s*[\w:]*ev_per_hartree,\s*(" + NUM + r")\)", body)
        rec["one_electron_rel_tol"] = float(t.group(1))
    m = re.search(r"getOneElectronMatrix\(\)\.getMatrix\(\)\(0, 0\)\s*\*\s*[\w:]*ev_per_hartree,\s*DoubleNear\((" +
                  NUM + r"),\s*(" + NUM + r")\)", body)
    if m:
        rec["one_electron_00_ev"] = [float(m.group(1)), float(m.group(2))]
    for key, getter in (("repulsion_ev", "getRepulsionEnergy"), ("electronic_ev", "getElectronicEnergy"),
                        ("total_ev", "getEnergy")):
        m = re.search(getter + r"\(\)\s*\*\s*[\w:]*ev_per_hartree,\s*DoubleNear\((" + NUM + r"),\s*(" + NUM + r")\)",
                      body)
        if m:
            rec[key] = [float(m.group(1)), float(m.group(2))]
    rows = re.findall(r"RowVector3d\s+\w+Gradient\((" + NUM + r"),\s*(" + NUM + r"),\s*(" + NUM + r")\)", body)
    if rows:
        rec["gradient_kcal_per_mol_angstrom"] = [[float(a), float(b), float(c)] for a, b, c in rows]
        t = re.search(r"getGradients\(\)\.row\(0\)\s*-\s*\w+\)\.norm\(\)\s*<\s*(" + NUM + r")", body)
        rec["gradient_row_norm_tol_hartree_per_bohr"] = float(t.group(1)) if t else None
    m = re.search(r"getGradients\(\)\.row\(0\)\.norm\(\)\s*<\s*(" + NUM + r")", body)
    if m:
        rec["zero_gradient_row_norm_tol"] = float(m.group(1))
    return rec


def main():
    ref = _reference_root()
    tests = os.path.join(ref, "src", "Sparrow", "Tests", "MethodsTests")
    out = {"note": "transcribed from the reference's test sources by extract_reference_vectors.py",
           "methods": {}}
    for method, rel in (("PM6", "Pm6/PM6Test.cpp"), ("AM1", "Am1/AM1Test.cpp")):
        path = os.path.join(tests, rel)
        with open(path) as f:
            text = f.read()
        recs = []
        for name, body, line in test_blocks(text):
            rec = parse_block(name, body, line, "src/Sparrow/Tests/MethodsTests/" + rel)
            if rec is None:
                continue
            if not any(k in rec for k in ("one_electron_ev", "one_electron_00_ev", "repulsion_ev", "electronic_ev",
                                          "total_ev", "gradient_kcal_per_mol_angstrom")):
                continue
            recs.append(rec)
        out["methods"][method] = recs
    # Python binding test: PM6 H2 at +-0.7 bohr (scine_utilities positions are bohr)
    pyt = os.path.join(ref, "src", "Sparrow", "Python", "Tests", "CalculatorTest.py")
    with open(pyt) as f:
        text = f.read()
    e = re.search(r"results\.energy,\s*(" + NUM + r"),\s*places=(\d+)", text)
    g = re.search(r"expected_gradients\s*=\s*\[\[(" + NUM + r"),", text)
    out["python_h2"] = {
        "source": "src/Sparrow/Python/Tests/CalculatorTest.py:21-32",
        "method": "PM6", "elements": ["H", "H"], "xyz_bohr": [[-0.7, 0.0, 0.0], [0.7, 0.0, 0.0]],
        "energy_hartree": float(e.group(1)), "places": int(e.group(2)),
        "gradient_x_atom0": float(g.group(1)),
    }
    # Local C-O integral block (Tests/Nddo/LocalIntegralTest.cpp:20-385)
    lit = os.path.join(ref, "src", "Sparrow", "Tests", "Nddo", "LocalIntegralTest.cpp")
    with open(lit) as f:
        text = f.read()
    kl = {}
    for atom, pair, v in re.findall(r"K([COHV])\.set\(MultipolePair::(\w+),\s*(" + NUM + r")\)", text):
        kl.setdefault(atom, {})[pair] = float(v)
    ds = {a: [int(x) for x in ns.split(",")[:2]] + [float(x) for x in zs.split(",")]
          for a, ns, zs in re.findall(r"D([COHV])\.computeFromExponents\(([\d, ]+?),\s*(" + NUM + r",\s*" + NUM +
                                      r")\)", text)}
    m = re.search(r"GivesCorrectResultsForCOPair\)\s*\{\s*double R = (" + NUM + r");", text)
    em = re.search(r"expectedMatrix\s*<<\s*([^;]+);", text)
    out["local_CO"] = {
        "source": "src/Sparrow/Tests/Nddo/LocalIntegralTest.cpp:53-385",
        "R_bohr": float(m.group(1)), "klopman": {"C": kl["C"], "O": kl["O"]},
        "charge_separation_inputs": {"C": ds["C"], "O": ds["O"]},
        "expected_ev": [float(x) for x in re.findall(NUM, em.group(1))], "tol_ev": 1e-3,
    }
    # Klopman / charge-separation parameter checks (Tests/Nddo/MultipoleParametersTest.cpp)
    out["multipole_parameters"] = {
        "source": "src/Sparrow/Tests/Nddo/MultipoleParametersTest.cpp:39-148",
        "charge_separation": [
            {"ns": 1, "np": 2, "zs": 3.31320400, "zp": 3.65713300, "sp1": 0.24758191, "pp2_times_sqrt2": 0.29953658},
            {"ns": 6, "np": 5, "zs": 2.759787, "zp": 1.977446, "sp1": 1.15147932, "pp2_times_sqrt2": 1.83730955},
        ],
        "klopman_PM6": [{"Z": 1, "ss0": 0.94165599},
                        {"Z": 6, "ss0": 1.02025963, "pp0": 1.02025963, "sp1": 1.29184422, "pp2": 0.76267645}],
        "tol": 1e-6,
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
