"""Extract the reference's DFTB known-answer vectors into dftb_known_answers.json.

The reference pins its DFTB2 / DFTB3 implementation against DFTB+ with
numbers written inline in its GoogleTest sources
(src/Sparrow/Tests/MethodsTests/Dftb/DFTB2Test.cpp, DFTB3Test.cpp).  This
script reads those sources as text and records, for each active (not
commented-out) restricted test: the geometry (Angstrom), the parameter set,
the expected energy (Hartree) with its tolerance, Mulliken charges,
orbital energies and forces with their tolerances, and the source file:line.

It runs only where the reference checkout exists (its path is the first argument);
the JSON it writes is committed and is what the tests read.

Usage: python tests/golden/extract_dftb_vectors.py [reference_root]
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from extract_reference_vectors import NUM, XYZ_LINE, test_blocks  # noqa: E402


def _reference_root():
    """The reference checkout, a required first command-line argument."""
    if len(sys.argv) < 2:
        sys.exit("usage: %s <path of the reference checkout>" % os.path.basename(sys.argv[0]))
    return sys.argv[1]

OUT = os.path.join(HERE, "dftb_known_answers.json")


def strip_block_comments(text):
    # keep line numbers: replace commented characters by spaces, newlines kept
    return re.sub(r"/\*.*?\*/", lambda m: re.sub(r"[^\n]", " ", m.group(0)), text, flags=re.S)


def parse(name, body, line, rel, order):
    if "setUnrestrictedCalculation(true)" in body or "GetsSameResultAsDFTBPlusFor" not in "GetsSameResultAsDFTBPlusFor" + name:
        return None
    if not name.startswith("GetsSameResultAsDFTBPlusFor") or "Unrestricted" in name:
        return None
    geo = XYZ_LINE.findall(body.split("XyzStreamHandler::read")[0])
    if not geo:
        return None
    rec = {"name": name, "source": "%s:%d" % (rel, line), "order": order,
           "elements": [g[0] for g in geo], "xyz_angstrom": [[float(g[1]), float(g[2]), float(g[3])] for g in geo]}
    m = re.search(r'initializeFromParameterPath\("([^"]+)"\)', body)
    rec["parameters"] = m.group(1)
    m = re.search(r"getEnergy\(\),\s*DoubleNear\((" + NUM + r"),\s*(" + NUM + r")\)\)", body)
    rec["energy"], rec["energy_tol"] = float(m.group(1)), float(m.group(2))
    m = re.search(r"expectedCharges\s*=\s*\{([^}]*)\}", body)
    if m:
        rec["charges"] = [float(x) for x in re.findall(NUM, m.group(1))]
        t = re.search(r"getAtomicCharges\(\)\[i\],\s*DoubleNear\(expectedCharges\[i\],\s*(" + NUM + r")\)", body)
        rec["charges_tol"] = float(t.group(1))
    m = re.search(r"std::vector<double> expected\s*=\s*\{([^}]*)\}", body)
    if m:
        rec["orbital_energies"] = [float(x) for x in re.findall(NUM, m.group(1))]
        t = re.search(r"eigenvalues\[i\],\s*DoubleNear\(expected\[i\],\s*(" + NUM + r")\)", body)
        rec["orbital_energies_tol"] = float(t.group(1))
    forces = re.findall(r"RowVector3d f(\d)\((" + NUM + r"),\s*(" + NUM + r"),\s*(" + NUM + r")\)", body)
    if forces:
        rec["forces"] = [[float(f[1]), float(f[2]), float(f[3])] for f in sorted(forces, key=lambda f: int(f[0]))]
        t = re.search(r"\)\.norm\(\)\s*<\s*(" + NUM + r")\)", body)
        rec["forces_tol"] = float(t.group(1))
    if "getGradients().row(0).norm(), DoubleEq(0)" in body:
        rec["forces"] = [[0.0, 0.0, 0.0]]
        rec["forces_tol"] = 1e-12
    return rec


def main():
    ref = _reference_root()
    out = {"tests": []}
    for fname, order in (("DFTB2Test.cpp", 2), ("DFTB3Test.cpp", 3)):
        rel = "src/Sparrow/Tests/MethodsTests/Dftb/" + fname
        text = strip_block_comments(open(os.path.join(ref, rel)).read())
        for name, body, line in test_blocks(text):
            rec = parse(name, body, line, rel, order)
            if rec:
                out["tests"].append(rec)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT, [t["name"] + "/%d" % t["order"] for t in out["tests"]])


if __name__ == "__main__":
    main()
