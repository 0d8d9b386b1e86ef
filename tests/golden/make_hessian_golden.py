"""Known answers for the semi-numerical Hessian, from the reference's app tests.

The reference computes Hessians by central differences of analytic gradients
(Utils::NumericalHessianCalculator; GenericMethodWrapper.cpp:58-88) and its
app prints harmonic frequencies (cm^-1) from them.  Its tests assert, on two
structures of src/Sparrow/Tests/AppTests/:
- ethane_opt.xyz, PM6: frequency index 11 = 2788.55 (test_sparrow.py:379-388);
- sft_1.xyz, lowest (imaginary) frequency, test_sparrow.py:637-715:
  MNDO -320.713, AM1 -410.523, PM6 -125.561, DFTB2 -158.922, DFTB3 -69.2154.
This script copies the two geometries (Angstrom) and those values into
tests/golden/hessian_known_answers.json.  Run from the repository root with the
reference checkout at the given path (a required argument).
"""
import json
import os
import sys


def _reference_root():
    """The reference checkout, a required first command-line argument."""
    if len(sys.argv) < 2:
        sys.exit("usage: %s <path of the reference checkout>" % os.path.basename(sys.argv[0]))
    return sys.argv[1]

REF_TESTS = "src/Sparrow/Tests/AppTests"


def read_xyz(path):
    lines = open(path).read().splitlines()
    n = int(lines[0])
    elements, xyz = [], []
    for line in lines[2:2 + n]:
        t = line.split()
        elements.append(t[0])
        xyz.append([float(v) for v in t[1:4]])
    return elements, xyz


def main(ref_root):
    out = {"source": "reference app tests (test_sparrow.py) and their structures", "structures": {}, "cases": []}
    for name in ("ethane_opt", "sft_1"):
        el, xyz = read_xyz(os.path.join(ref_root, REF_TESTS, name + ".xyz"))
        out["structures"][name] = {"elements": el, "xyz_angstrom": xyz}
    out["cases"].append({"structure": "ethane_opt", "method": "PM6", "index": 11, "frequency": 2788.55,
                         "cite": "test_sparrow.py:379-388"})
    for method, value, cite in [("MNDO", -320.713, "637-646"), ("AM1", -410.523, "648-657"),
                                ("PM6", -125.561, "705-715"), ("DFTB2", -158.922, "680-690"),
                                ("DFTB3", -69.2154, "692-701")]:
        out["cases"].append({"structure": "sft_1", "method": method, "index": 0, "frequency": value,
                             "cite": "test_sparrow.py:" + cite})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hessian_known_answers.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main(_reference_root())
