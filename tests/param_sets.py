"""Parameter files for the run-time parameter tests, written from the embedded tables.

Test infrastructure.  The embedded NDDO and DFTB tables
(sparrow_b200/csrc/nddo_tables.inc, dftb_tables.inc) are read back as text and
written out in the reference's file formats:

- NDDO: parameters.json in the layout of the reference's Parameters::write
  (src/Sparrow/Sparrow/Implementations/Nddo/Parameters.cpp:20-93);
- DFTB: Slater-Koster files X-Y.skf with hubbard.dat and spin.dat in the
  grammar of Dftb/Utils/SkfParser.cpp:62-330, with the variations that grammar
  allows (n*v runs, comma separators, forwarding files, lower-case and
  dash-less names, trailing documentation after the spline block).

It also turns a parameter set into oracle records (nddo_raw.h layout) with
the STO-6G expansion rescaled for a new orbital exponent, independently of the
engine's own rescaling, so the oracle can take the same set.
"""
import ctypes
import json
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NDDO_INC = os.path.join(ROOT, "sparrow_b200", "csrc", "nddo_tables.inc")
DFTB_INC = os.path.join(ROOT, "sparrow_b200", "csrc", "dftb_tables.inc")

RAW_KEYS = ["Uss", "Upp", "betaS", "betaP", "zetaS", "zetaP", "gss", "gpp", "gsp", "gp2", "hsp", "pcore", "alpha"]
SYMBOL = {1: "H", 2: "He", 3: "Li", 4: "Be", 5: "B", 6: "C", 7: "N", 8: "O", 9: "F", 10: "Ne"}


def _hexes(s):
    return [float.fromhex(x.strip()) for x in s.split(",")]


def nddo_embedded(method):
    """(atomic records, diatomic records) of a method as dicts, from nddo_tables.inc."""
    src = open(NDDO_INC).read()
    blk = src.split("static const NddoRawAtomic k%sAtomic[] = {" % method)[1].split("};")[0]
    atoms = {}
    pat = re.compile(r"\s*\{(\d+), (\d), \{([^}]*)\}, (\d), " + r", ".join([r"\{([^}]*)\}"] * 7) + r"\},")
    for line in blk.strip().splitlines():
        m = pat.match(line)
        z = int(m.group(1))
        v = _hexes(m.group(3))
        atoms[z] = {"Z": z, "has_d": int(m.group(2)), "v": dict(zip(RAW_KEYS, v)), "n_gauss": int(m.group(4)),
                    "ga": _hexes(m.group(5)), "gb": _hexes(m.group(6)), "gc": _hexes(m.group(7)),
                    "s_exp": _hexes(m.group(8)), "s_coef": _hexes(m.group(9)),
                    "p_exp": _hexes(m.group(10)), "p_coef": _hexes(m.group(11))}
    dblk = src.split("static const NddoRawDiatomic k%sDiatomic[] = {" % method)[1].split("};")[0]
    ndiat = int(re.search(r"k%sNumDiatomic = (\d+);" % method, src).group(1))
    diat = []
    for line in dblk.strip().splitlines()[:ndiat]:
        m = re.match(r"\s*\{(\d+), (\d+), ([^,]+), ([^}]+)\}", line)
        diat.append({"z1": int(m.group(1)), "z2": int(m.group(2)), "exponent": float.fromhex(m.group(3).strip()),
                     "factor": float.fromhex(m.group(4).strip())})
    return atoms, diat


def write_nddo_json(path, atoms, diat, elements=None):
    """parameters.json in the reference's layout (numbers written to round-trip exactly)."""
    out = {"atomic": [], "diatomic": []}
    for z in sorted(atoms):
        if elements is not None and z not in elements:
            continue
        a = atoms[z]
        v = a["v"]
        pack = {
            "oneCenterEnergy": {"s": v["Uss"], "p": v["Upp"], "d": 0.0},
            "beta": {"s": v["betaS"], "p": v["betaP"], "d": 0.0},
            "orbitalExponent": {"s": v["zetaS"], "p": v["zetaP"], "d": 0.0},
            "internalExponent": {"s": 0.0, "p": 0.0, "d": 0.0},
            "gss": v["gss"], "gpp": v["gpp"], "gsp": v["gsp"], "gp2": v["gp2"], "hsp": v["hsp"],
            "pcore": v["pcore"], "f0sd": 0.0, "g2sd": 0.0, "alpha": v["alpha"],
        }
        gauss = [{"a": a["ga"][k], "b": a["gb"][k], "c": a["gc"][k]} for k in range(a["n_gauss"])]
        out["atomic"].append({"key": z, "value": {"pack": pack, "gaussianRepulsion": gauss}})
    for d in diat:
        if elements is not None and (d["z1"] not in elements or d["z2"] not in elements):
            continue
        out["diatomic"].append({"key": {"first": d["z1"], "second": d["z2"]},
                                "value": {"exponent": d["exponent"], "factor": d["factor"]}})
    with open(path, "w") as f:
        json.dump(out, f, indent=4)


def rescaled_sto6g(atom, l, zeta_new):
    """STO-6G exponents / normalised coefficients of shell l for a new Slater
    exponent: exponents scale as zeta^2, coefficients as zeta^(l + 3/2)."""
    z0 = atom["v"]["zetaS" if l == 0 else "zetaP"]
    e0 = np.array(atom["s_exp" if l == 0 else "p_exp"])
    c0 = np.array(atom["s_coef" if l == 0 else "p_coef"])
    if zeta_new == z0:
        return e0.tolist(), c0.tolist()
    r = zeta_new / z0
    return (e0 * r ** 2).tolist(), (c0 * r ** (l + 1.5)).tolist()


class RawAtomic(ctypes.Structure):
    _fields_ = [("Z", ctypes.c_int), ("has_d", ctypes.c_int), ("v", ctypes.c_double * 13),
                ("n_gauss", ctypes.c_int), ("ga", ctypes.c_double * 4), ("gb", ctypes.c_double * 4),
                ("gc", ctypes.c_double * 4), ("s_exp", ctypes.c_double * 6), ("s_coef", ctypes.c_double * 6),
                ("p_exp", ctypes.c_double * 6), ("p_coef", ctypes.c_double * 6)]


class RawDiatomic(ctypes.Structure):
    _fields_ = [("z1", ctypes.c_int), ("z2", ctypes.c_int), ("exponent", ctypes.c_double),
                ("factor", ctypes.c_double)]


def oracle_records(atoms, diat, embedded):
    """ctypes arrays for oracle_set_parameters; STO-6G from the embedded record of
    the same element, rescaled where the orbital exponent changed."""
    arr = (RawAtomic * len(atoms))()
    for i, z in enumerate(sorted(atoms)):
        a = atoms[z]
        r = arr[i]
        r.Z = z
        r.has_d = a["has_d"]
        for k, key in enumerate(RAW_KEYS):
            r.v[k] = a["v"][key]
        r.n_gauss = a["n_gauss"]
        for k in range(4):
            r.ga[k], r.gb[k], r.gc[k] = a["ga"][k], a["gb"][k], a["gc"][k]
        for l, (ename, cname) in enumerate([("s_exp", "s_coef"), ("p_exp", "p_coef")]):
            zeta = a["v"]["zetaS" if l == 0 else "zetaP"]
            if l == 1 and (z == 1 or zeta == 0):
                continue
            e, c = rescaled_sto6g(embedded[z], l, zeta)
            for k in range(6):
                getattr(r, ename)[k] = e[k]
                getattr(r, cname)[k] = c[k]
    darr = (RawDiatomic * max(1, len(diat)))()
    for i, d in enumerate(diat):
        darr[i].z1, darr[i].z2, darr[i].exponent, darr[i].factor = d["z1"], d["z2"], d["exponent"], d["factor"]
    return arr, len(atoms), darr, len(diat)


# ---------------------------------------------------------------------------
# DFTB
# ---------------------------------------------------------------------------
def _block(src, name):
    return re.split(name + r"\[\](?:\[\d+\])? = \{", src)[1].split("};")[0]


def _braced(blk):
    return [x for x in re.findall(r"\{([^{}]*)\}", blk)]


def dftb_embedded(set_name):
    """{'elems': {Z: dict}, 'pairs': {(Z1, Z2): dict}} of an embedded set, from dftb_tables.inc."""
    src = open(DFTB_INC).read()
    elems = [x.split(",") for x in _braced(_block(src, "kDftbElemRaw"))]
    pairs = [x.split(",") for x in _braced(_block(src, "kDftbPairRaw"))]
    table = [[float(v) for v in x.split(",")] for x in _braced(_block(src, "kDftbTable"))]
    spl = [[float(v) for v in x.split(",")] for x in _braced(_block(src, "kDftbSplineRaw"))]
    sets = [x.split(",") for x in _braced(_block(src, "kDftbSetRaw"))]
    s = next(t for t in sets if t[0].strip().strip('"') == set_name)
    e0, ne, p0, npair = (int(t) for t in s[1:])
    out = {"elems": {}, "pairs": {}}
    for e in elems[e0:e0 + ne]:
        f = [t.strip() for t in e]
        z = int(f[0])
        out["elems"][z] = {"Es": float(f[1]), "Ep": float(f[2]), "Ed": float(f[3]), "Us": float(f[4]),
                           "Up": float(f[5]), "Ud": float(f[6]), "fs": float(f[7]), "fp": float(f[8]),
                           "fd": float(f[9]), "hub": float(f[10]), "has_hub": int(f[11]), "wss": float(f[12]),
                           "wpp": float(f[13]), "has_spin": int(f[14]), "wsp": float(f[15]), "wps": float(f[16])}
    for p in pairs[p0:p0 + npair]:
        f = [t.strip() for t in p]
        z1, z2, rows, row0, nspl, sp0 = int(f[0]), int(f[1]), int(f[3]), int(f[4]), int(f[5]), int(f[12])
        out["pairs"][(z1, z2)] = {"grid": float(f[2]), "rows": table[row0:row0 + rows], "cutoff": float(f[6]),
                                  "a": (float(f[7]), float(f[8]), float(f[9])), "c4": float(f[10]),
                                  "c5": float(f[11]), "splines": spl[sp0:sp0 + nspl]}
    return out


KEEP = [19, 9, 18, 8, 15, 5, 16, 6]


def _num(x):
    return repr(float(x))


def _row20(kept):
    full = [0.0] * 20
    for c, v in zip(KEEP, kept):
        full[c] = v
    # runs of zeros as n*v tokens, the rest comma-separated
    toks, k = [], 0
    while k < 20:
        if full[k] == 0.0:
            j = k
            while j < 20 and full[j] == 0.0:
                j += 1
            toks.append("%d*0.0" % (j - k) if j - k > 1 else "0.0")
            k = j
        else:
            toks.append(_num(full[k]))
            k += 1
    return ", ".join(toks)


def skf_text(pair, atomic=None, mass=1.0):
    lines = ["%s, %d" % (_num(pair["grid"]), len(pair["rows"]))]
    if atomic is not None:
        e = atomic
        lines.append(" ".join(_num(x) for x in (e["Ed"], e["Ep"], e["Es"], 0.0, e["Ud"], e["Up"], e["Us"], e["fd"],
                                                e["fp"], e["fs"])))
    lines.append("%s, 19*0.0" % _num(mass))
    lines += [_row20(r) for r in pair["rows"]]
    lines += ["", "Spline", "%d %s" % (len(pair["splines"]), _num(pair["cutoff"])),
              " ".join(_num(x) for x in pair["a"])]
    for i, s in enumerate(pair["splines"]):
        t = " ".join(_num(x) for x in s)
        if i == len(pair["splines"]) - 1:
            t += " " + _num(pair["c4"]) + " " + _num(pair["c5"])
        lines.append(t)
    lines += ["", "<Documentation>", "  written from the embedded tables for a test", "</Documentation>"]
    return "\n".join(lines) + "\n"


def write_skf_directory(path, set_name, elements=None, hubbard=True, spin=True, variants=True, skip_pairs=()):
    """A Slater-Koster directory holding an embedded set.  variants: spell some
    files in lower case, without the dash, or as forwarding files."""
    d = dftb_embedded(set_name)
    os.makedirs(path, exist_ok=True)
    zs = sorted(z for z in d["elems"] if elements is None or z in elements)
    for z1 in zs:
        for z2 in zs:
            if (z1, z2) in skip_pairs:
                continue
            a, b = SYMBOL[z1], SYMBOL[z2]
            text = skf_text(d["pairs"][(z1, z2)], d["elems"][z1] if z1 == z2 else None)
            name = "%s-%s.skf" % (a, b)
            if variants and (z1, z2) == (8, 8):
                name = name.lower()
            elif variants and (z1, z2) == (7, 1):
                name = "%s%s.skf" % (a, b)
            if variants and (z1, z2) == (6, 1):
                # forwarding file: the content is the name of the file holding the data
                with open(os.path.join(path, "CH-data.skf"), "w") as f:
                    f.write(text)
                text = "CH-data.skf\n"
            with open(os.path.join(path, name), "w") as f:
                f.write(text)
    if hubbard:
        with open(os.path.join(path, "hubbard.dat"), "w") as f:
            for z in zs:
                if d["elems"][z]["has_hub"]:
                    f.write("%s %s\n" % (SYMBOL[z], _num(d["elems"][z]["hub"])))
    if spin:
        with open(os.path.join(path, "spin.dat"), "w") as f:
            f.write("# element W_ss W_sp W_ps W_pp W_sd W_pd W_dd W_ds W_dp\n")
            for z in zs:
                e = d["elems"][z]
                if e["has_spin"]:
                    f.write("%s %s %s %s %s 0.0 0.0 0.0 0.0 0.0\n" % (SYMBOL[z], _num(e["wss"]), _num(e["wsp"]),
                                                                      _num(e["wps"]), _num(e["wpp"])))
    return d
