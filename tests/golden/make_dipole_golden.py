"""Known answers for the dipole moment, from the reference's dipole tests.

src/Sparrow/Tests/Dipole/MopacDipoleTest.cpp defines three structures (HF,
CO2, ethanol; Angstrom) and asserts, with the NDDO approximation of the
dipole and PM6 (MOPAC values, |mu| in Debye = |mu| e bohr x 2.541746,
tolerance 0.001 D):
  HF 1.436 (MopacDipoleTest.cpp:82-88), CO2 0.013 (:90-98), ethanol 2.133 (:100-107);
and with DFTB2 on ethanol the DFTB+ vector (-0.36023764, -0.21653604,
-0.38972594) e bohr at 1e-6 (:220-230).  This script copies the structures
out of the test file and writes tests/golden/dipole_known_answers.json.
Run from the repository root with the reference checkout at the given path
(a required argument).
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

TEST = "src/Sparrow/Tests/Dipole/MopacDipoleTest.cpp"


def structure(src, name):
    block = re.search(r"std::stringstream %s\((.*?)\);" % name, src, re.S).group(1)
    text = "".join(re.findall(r'"((?:[^"\\]|\\.)*)"', block)).replace("\\n", "\n")
    lines = text.splitlines()
    n = int(lines[0])
    elements, xyz = [], []
    for line in lines[2:2 + n]:
        t = line.split()
        elements.append(t[0])
        xyz.append([float(v) for v in t[1:4]])
    return {"elements": elements, "xyz_angstrom": xyz}


def main(ref_root):
    src = open(os.path.join(ref_root, TEST)).read()
    out = {"source": TEST, "debye_per_e_bohr": 2.541746,
           "structures": {k: structure(src, k + "ss") for k in ("HF", "CO2", "Ethanol")},
           "pm6_norm_debye": [{"structure": "HF", "value": 1.436, "tolerance": 0.001, "cite": "MopacDipoleTest.cpp:82-88"},
                              {"structure": "CO2", "value": 0.013, "tolerance": 0.001, "cite": "MopacDipoleTest.cpp:90-98"},
                              {"structure": "Ethanol", "value": 2.133, "tolerance": 0.001,
                               "cite": "MopacDipoleTest.cpp:100-107"}],
           "dftb2_vector_e_bohr": {"structure": "Ethanol", "value": [-0.36023764, -0.21653604, -0.38972594],
                                   "tolerance": 1e-6, "cite": "MopacDipoleTest.cpp:220-230"}}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dipole_known_answers.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main(_reference_root())
