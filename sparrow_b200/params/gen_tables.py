"""Generate the NDDO parameter tables compiled into the engine and the oracle.

Reads the reference's published method parameters (MNDO, AM1, PM6) and the
STO-6G expansions that the reference embeds for them, and writes
``sparrow_b200/csrc/nddo_tables.inc``: plain C aggregate initialisers for the
structs declared in ``sparrow_b200/csrc/nddo_raw.h``.  Every floating-point
number is written as a C99 hexadecimal literal so the tables are bit-identical
to the values the reference loads at run time.

Sources (paths relative to the reference checkout):
  src/Sparrow/Sparrow/Resources/{Mndo,Am1,Pm6}/parameters.json
      atomic "pack" (eV / Angstrom units, Parameters.h:20-138) and the PM6
      diatomic (exponent, factor) pairs.
  src/Sparrow/Sparrow/Resources/{Mndo,Am1,Pm6}/STO-6G.cpp
      per element (angular momentum, exponent, normalised coefficient)
      triples; the reference's own test (Tests/Nddo/Sto6gBasisTest.cpp:127-160)
      pins them to the run-time Slater-to-Gaussian expansion.

Usage:  python sparrow_b200/params/gen_tables.py [reference_root]
The output is committed; this script is only needed to regenerate it.
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
OUT = os.path.join(HERE, "..", "csrc", "nddo_tables.inc")

METHODS = [("MNDO", "Mndo"), ("AM1", "Am1"), ("PM6", "Pm6")]
TRIPLE = re.compile(r"\{(\d), (-?0x[0-9a-fA-Fp.+\-]+), (-?0x[0-9a-fA-Fp.+\-]+)\}")


def hx(x):
    return float(x).hex()


def read_sto6g(path):
    """Map Z -> {l: [(exponent, coefficient)]} from an embedded STO-6G.cpp."""
    table = {}
    line_re = re.compile(r"^\s*\{(\d+), \{Utils::GtoExpansion")
    with open(path) as f:
        for line in f:
            m = line_re.match(line)
            if not m:
                continue
            z = int(m.group(1))
            shells = {}
            for l, e, c in TRIPLE.findall(line):
                shells.setdefault(int(l), []).append((float.fromhex(e), float.fromhex(c)))
            table[z] = shells
    return table


def main():
    ref = _reference_root()
    res = os.path.join(ref, "src", "Sparrow", "Sparrow", "Resources")
    out = []
    out.append("// Generated by sparrow_b200/params/gen_tables.py from the reference's published\n")
    out.append("// MNDO/AM1/PM6 parameter files and embedded STO-6G expansions. Do not edit by hand.\n")
    out.append("// Units as published: energies eV, lengths Angstrom, pcore bohr.\n\n")
    for name, folder in METHODS:
        with open(os.path.join(res, folder, "parameters.json")) as f:
            params = json.load(f)
        sto = read_sto6g(os.path.join(res, folder, "STO-6G.cpp"))
        atoms = sorted(params["atomic"], key=lambda a: a["key"])
        out.append("static const NddoRawAtomic k%sAtomic[] = {\n" % name)
        for a in atoms:
            z = a["key"]
            p = a["value"]["pack"]
            g = a["value"].get("gaussianRepulsion", [])
            if len(g) > 4:
                raise SystemExit("more than 4 Gaussian repulsion terms for Z=%d" % z)
            ga = [x["a"] for x in g] + [0.0] * (4 - len(g))
            gb = [x["b"] for x in g] + [0.0] * (4 - len(g))
            gc = [x["c"] for x in g] + [0.0] * (4 - len(g))
            shells = sto.get(z, {})
            s = shells.get(0, [(0.0, 0.0)] * 6)
            pp = shells.get(1, [(0.0, 0.0)] * 6)
            if len(s) != 6 or len(pp) != 6:
                raise SystemExit("unexpected STO-6G length for Z=%d" % z)
            vals = [p["oneCenterEnergy"]["s"], p["oneCenterEnergy"]["p"], p["beta"]["s"], p["beta"]["p"],
                    p["orbitalExponent"]["s"], p["orbitalExponent"]["p"], p["gss"], p["gpp"], p["gsp"],
                    p["gp2"], p["hsp"], p["pcore"], p["alpha"]]
            has_d = 1 if (p["oneCenterEnergy"]["d"] != 0 or p["orbitalExponent"]["d"] != 0) else 0
            out.append("  {%d, %d, {%s}, %d, {%s}, {%s}, {%s}, {%s}, {%s}, {%s}, {%s}},\n" % (
                z, has_d, ", ".join(hx(v) for v in vals), len(g),
                ", ".join(hx(v) for v in ga), ", ".join(hx(v) for v in gb), ", ".join(hx(v) for v in gc),
                ", ".join(hx(e) for e, _ in s), ", ".join(hx(c) for _, c in s),
                ", ".join(hx(e) for e, _ in pp), ", ".join(hx(c) for _, c in pp)))
        out.append("};\n\n")
        diat = params.get("diatomic") or []
        out.append("static const NddoRawDiatomic k%sDiatomic[] = {\n" % name)
        if not diat:
            out.append("  {0, 0, 0x0p+0, 0x0p+0},\n")
        for d in sorted(diat, key=lambda d: (d["key"]["first"], d["key"]["second"])):
            out.append("  {%d, %d, %s, %s},\n" % (d["key"]["first"], d["key"]["second"],
                                                  hx(d["value"]["exponent"]), hx(d["value"]["factor"])))
        out.append("};\n")
        out.append("static const int k%sNumDiatomic = %d;\n\n" % (name, len(diat)))
    with open(OUT, "w") as f:
        f.write("".join(out))
    print("wrote", os.path.normpath(OUT))


if __name__ == "__main__":
    main()
