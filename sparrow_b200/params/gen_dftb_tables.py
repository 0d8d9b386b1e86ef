"""Generate sparrow_b200/csrc/dftb_tables.inc from the reference's DFTB parameter sets.

Reads the Slater-Koster files (`X-Y.skf`) and `hubbard.dat` of the parameter
sets the engine embeds (mio-1-1 for DFTB2, 3ob-3-1 for DFTB3 and 3ob-2-1, the
set of the reference's DFTB3 tests) for the s/p elements H, C, N, O, and
writes them as C++ initialisers.  The parse follows the reference's SKF
grammar (src/Sparrow/Sparrow/Implementations/Dftb/Utils/SkfParser.cpp:62-180):

  line 1       grid distance, grid count (unused), optional integer
  (homonuclear) Ed Ep Es SPE Ud Up Us fd fp fs
  one line     mass and polynomial coefficients (ignored)
  table        every following line of numbers up to the `Spline` keyword,
               20 columns each; `n*v` stands for n copies of v; row i holds
               the integrals at distance (i + 1) * grid distance
  Spline       n_int cutoff / a1 a2 a3 / n_int lines start end c0 c1 c2 c3,
               the last one followed by c4 c5

Of the 20 columns (Hdd0 Hdd1 Hdd2 Hpd0 Hpd1 Hpp0 Hpp1 Hsd0 Hsp0 Hss0, then
the same ten overlaps) the s/p engine keeps eight: Sss Hss Ssp Hsp Spp0 Hpp0
Spp1 Hpp1 (columns 19 9 18 8 15 5 16 6).  Numbers are written back verbatim
from the files, so the compiled doubles are the ones the reference parses.

Usage:  python sparrow_b200/params/gen_dftb_tables.py [reference_root]
"""
import os
import re
import sys


def _reference_root():
    """The reference checkout, a required first command-line argument."""
    if len(sys.argv) < 2:
        sys.exit("usage: %s <path of the reference checkout>" % os.path.basename(sys.argv[0]))
    return sys.argv[1]

ELEMENTS = ["H", "C", "N", "O"]
Z = {"H": 1, "C": 6, "N": 7, "O": 8}
SETS = ["mio-1-1", "3ob-3-1", "3ob-2-1"]
KEEP = [19, 9, 18, 8, 15, 5, 16, 6]
NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eEdD][-+]?\d+)?"


def tokens(line):
    """Numbers of a line as strings, with n*v expanded."""
    out = []
    for t in re.split(r"[\s,]+", line.strip()):
        if not t:
            continue
        m = re.fullmatch(r"(\d+)\*(" + NUM + ")", t)
        if m:
            out += [m.group(2)] * int(m.group(1))
        elif re.fullmatch(NUM, t):
            out.append(t)
        else:
            return None
    return out


def parse_skf(path, homonuclear):
    with open(path) as f:
        lines = f.read().splitlines()
    k = 0
    head = tokens(lines[k])
    k += 1
    grid = head[0]
    atomic = None
    if homonuclear:
        t = tokens(lines[k])
        if t is not None and len(t) == 10 and "*" not in lines[k]:
            atomic = t
            k += 1
    k += 1  # mass / polynomial line
    table = []
    while k < len(lines):
        s = lines[k].strip()
        if s.startswith("Spline"):
            break
        if s:
            t = tokens(s)
            if t is None:
                break
            if len(t) < 20:
                raise ValueError("%s:%d: integral line with %d numbers" % (path, k + 1, len(t)))
            table.append(t[:20])
        k += 1
    assert lines[k].strip().startswith("Spline"), path
    k += 1
    while not lines[k].strip():
        k += 1
    n_int, cutoff = tokens(lines[k])[:2]
    k += 1
    a1, a2, a3 = tokens(lines[k])[:3]
    k += 1
    splines = []
    c4 = c5 = "0.0"
    for i in range(int(n_int)):
        t = tokens(lines[k])
        k += 1
        splines.append(t[:6])
        if i == int(n_int) - 1:
            if len(t) >= 8:
                c4, c5 = t[6], t[7]
    return {"grid": grid, "atomic": atomic, "table": table, "n_int": int(n_int), "cutoff": cutoff, "a": (a1, a2, a3),
            "splines": splines, "c4": c4, "c5": c5}


def lit(s):
    s = s.replace("D", "E").replace("d", "e")
    if not re.search(r"[.eE]", s):
        s += ".0"
    return s


def main():
    ref = _reference_root()
    base = os.path.join(ref, "src/Sparrow/Sparrow/Resources/Dftb")
    here = os.path.dirname(os.path.abspath(__file__))
    out = os.path.join(here, "..", "csrc", "dftb_tables.inc")
    elems, pairs, table, spl, sets = [], [], [], [], []
    for sname in SETS:
        d = os.path.join(base, sname)
        hub = {}
        hp = os.path.join(d, "hubbard.dat")
        if os.path.exists(hp):
            toks = open(hp).read().split()
            for i in range(0, len(toks) - 1, 2):
                hub[toks[i]] = toks[i + 1]
        # spin constants (spin.dat): W_ss and W_pp per element, for triplet TD-DFTB
        spin = {}
        sp_path = os.path.join(d, "spin.dat")
        if os.path.exists(sp_path):
            for line in open(sp_path):
                t = line.split()
                if len(t) >= 5 and not t[0].startswith("#"):
                    spin[t[0]] = (t[1], t[4], t[2], t[3])  # W_ss, W_pp, W_sp, W_ps
        e0, p0 = len(elems), len(pairs)
        for a in ELEMENTS:
            for b in ELEMENTS:
                r = parse_skf(os.path.join(d, "%s-%s.skf" % (a, b)), a == b)
                if a == b:
                    Ed, Ep, Es, SPE, Ud, Up, Us, fd, fp, fs = r["atomic"]
                    wss, wpp, wsp, wps = spin.get(a, ("0.0", "0.0", "0.0", "0.0"))
                    elems.append("{%d, %s, %s, %s, %s, %s, %s, %s, %s, %s, %s, %d, %s, %s, %d, %s, %s}" % (
                        Z[a], lit(Es), lit(Ep), lit(Ed), lit(Us), lit(Up), lit(Ud), lit(fs), lit(fp), lit(fd),
                        lit(hub.get(a, "0.0")), 1 if a in hub else 0, lit(wss), lit(wpp), 1 if a in spin else 0,
                        lit(wsp), lit(wps)))
                t0, s0 = len(table), len(spl)
                for row in r["table"]:
                    table.append(", ".join(lit(row[c]) for c in KEEP))
                for sp in r["splines"]:
                    spl.append("{%s}" % ", ".join(lit(v) for v in sp))
                a1, a2, a3 = r["a"]
                pairs.append("{%d, %d, %s, %d, %d, %d, %s, %s, %s, %s, %s, %s, %d}" % (
                    Z[a], Z[b], lit(r["grid"]), len(r["table"]), t0, r["n_int"], lit(r["cutoff"]), lit(a1), lit(a2),
                    lit(a3), lit(r["c4"]), lit(r["c5"]), s0))
        sets.append('{"%s", %d, %d, %d, %d}' % (sname, e0, len(elems) - e0, p0, len(pairs) - p0))
    with open(out, "w") as f:
        f.write("// Generated by sparrow_b200/params/gen_dftb_tables.py from the reference's DFTB\n")
        f.write("// parameter sets (Resources/Dftb/{%s}); do not edit.\n" % ",".join(SETS))
        f.write("// Elements: Z, Es, Ep, Ed, Us, Up, Ud, fs, fp, fd, Hubbard derivative, has it,\n")
        f.write("// spin constants W_ss, W_pp, has them, W_sp, W_ps.\n")
        f.write("static const DftbElemRaw kDftbElemRaw[] = {\n  %s};\n" % ",\n  ".join(elems))
        f.write("// Pairs (file Z1-Z2): Z1, Z2, grid distance, rows, first row, spline count, cutoff,\n")
        f.write("// a1, a2, a3, c4, c5, first spline.\n")
        f.write("static const DftbPairRaw kDftbPairRaw[] = {\n  %s};\n" % ",\n  ".join(pairs))
        f.write("// Table rows: Sss Hss Ssp Hsp Spp0 Hpp0 Spp1 Hpp1 at distance (row + 1) * grid distance.\n")
        f.write("static const double kDftbTable[][8] = {\n  {%s}};\n" % "},\n  {".join(table))
        f.write("// Repulsion splines: start, end, c0, c1, c2, c3.\n")
        f.write("static const DftbSplineRaw kDftbSplineRaw[] = {\n  %s};\n" % ",\n  ".join(spl))
        f.write("static const DftbSetRaw kDftbSetRaw[] = {\n  %s};\n" % ",\n  ".join(sets))
    print("wrote", out, len(elems), "elements", len(pairs), "pairs", len(table), "rows", len(spl), "splines")


if __name__ == "__main__":
    main()
