"""Extract the reference's TD-DFTB known-answer vectors into tddftb_known_answers.json.

The reference pins its linear-response TD-DFTB against fixed numbers in
src/Sparrow/Tests/TimeDependent/TDDFTBTest.cpp: the ten lowest restricted
singlet and triplet excitation energies (eV) of a distorted methane with
mio-1-1 DFTB2, the DFTB+ gamma matrix and the mio-1-1 spin constants of the
same molecule.  This script reads that source as text and records, per
test, the geometry (Angstrom), the parameter set, the expected values with
their tolerances and the source file:line.

It runs only where the reference checkout exists (its path is the first argument);
the JSON it writes is committed and is what the tests read.

Usage: python tests/golden/extract_tddftb_vectors.py [reference_root]
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

OUT = os.path.join(HERE, "tddftb_known_answers.json")
REL = "src/Sparrow/Tests/TimeDependent/TDDFTBTest.cpp"


def main():
    ref = _reference_root()
    text = open(os.path.join(ref, REL)).read()
    out = {"source": REL, "tests": []}
    for name, body, line in test_blocks(text):
        spin = {"CanPerformRestrictedSingletTDDFTCalculation": "singlet",
                "CanPerformRestrictedTripletTDDFTCalculation": "triplet"}.get(name)
        if spin is None and name != "TDDFTBDataRecordsRightConstants":
            continue
        geo = XYZ_LINE.findall(body)
        params = re.search(r'methodParameters,\s*"([^"]+)"', body).group(1)
        rec = {"name": name, "line": line, "parameters": params, "method": "DFTB2",
               "elements": [g[0] for g in geo], "xyz_angstrom": [[float(v) for v in g[1:]] for g in geo]}
        if spin:
            vals = re.findall(r"EXPECT_THAT\(energies\((\d+)\),\s*DoubleNear\((" + NUM + r"),\s*(" + NUM + r")\)\)",
                              body)
            rec["spin"] = spin
            rec["energies_ev"] = [float(v[1]) for v in sorted(vals, key=lambda t: int(t[0]))]
            rec["tolerance_ev"] = max(float(v[2]) for v in vals)
        else:
            rec["spin_constants"] = [float(v) for v in re.findall(
                r"EXPECT_DOUBLE_EQ\(\(\*data\.spinConstants\)\(\d+\),\s*(" + NUM + r")\)", body)]
            m = re.search(r"refMatrix\s*<<(.*?);", body, flags=re.S)
            lower = [float(v) for v in re.findall(NUM, m.group(1))]
            n = int(round(len(lower) ** 0.5))
            rec["gamma_lower_rowmajor"] = lower
            rec["gamma_n"] = n
            rec["gamma_tolerance"] = float(re.search(r"DoubleNear\(refMatrix\(row, col\),\s*(" + NUM + r")\)",
                                                     body).group(1))
        out["tests"].append(rec)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT, len(out["tests"]), "tests")


if __name__ == "__main__":
    main()
