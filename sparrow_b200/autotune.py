"""Autotuner of the batched SCF: picks, per molecule-size bin of 32 AOs, the
orbital update (exact / hybrid / rotation) and the Pulay subspace size that
minimise the SCF kernel's device time, and writes them as the library's
compiled-in defaults (sparrow_b200/csrc/tuned_table.h).

Run on the GPU the library will serve (then rebuild the library):

    python -m sparrow_b200.autotune [--out PATH] [--json PATH]

Method, per bin: a seeded mix of molecules whose AO counts fall in the bin
(alkanes C_nH_2n+2, water clusters (H2O)_n and polyenes C_2kH_2k+2, PM6),
enough to fill every SM several times; every candidate (3 orbital updates x
Pulay subspaces 4, 5, 6) runs the same batch (one warm-up, then the median of
`--reps` SCF stages timed with CUDA events).  A candidate must converge every
molecule to within 1e-8 Hartree of the first candidate's energies, or it is
not eligible.  Bins above the largest measured one inherit its choice.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MODES = ("exact", "hybrid", "rotation")
MODE_CODE = {"exact": 0, "hybrid": 1, "rotation": 2}
BINS = 16


def bin_molecules(k, count, seed):
    """Seeded molecules with 32k <= n_AO < 32k + 32 (n_AO >= 2)."""
    from sparrow_b200 import geometry
    rng = np.random.default_rng(seed + 101 * k)
    lo, hi = max(32 * k, 2), 32 * k + 31
    kinds = []
    for n in range(1, 80):  # alkanes: 6n + 2 AOs
        if lo <= 6 * n + 2 <= hi:
            kinds.append(("alkane", n))
    for n in range(1, 80):  # water clusters: 6n AOs
        if lo <= 6 * n <= hi:
            kinds.append(("water", n))
    for n in range(2, 60):  # polyenes: 10k + 2 AOs
        if lo <= 10 * n + 2 <= hi:
            kinds.append(("polyene", n))
    if not kinds:
        return []
    out = []
    for _ in range(count):
        kind, n = kinds[int(rng.integers(len(kinds)))]
        if kind == "alkane":
            Z, x = geometry.alkane(n, rng)
        elif kind == "water":
            Z, x = geometry.water_cluster(n, seed=int(rng.integers(1 << 30)))
        else:
            Z, x = geometry.polyene(n, rng)
        out.append((np.asarray(Z, dtype=np.int32), geometry.to_bohr(x)))
    return out


def measure_bin(mols, reps):
    import sparrow_b200
    b = sparrow_b200.Batch("PM6", mols, scc=1e-7, rmsd=1e-8, max_iter=100)
    rows, ref = [], None
    for mode in MODES:
        for diis in (4, 5, 6):
            b.set_tuning(mode, diis)
            b.run()
            e, _, it, conv = b.results()
            times = []
            for _ in range(reps):
                b.run()
                e, _, it, conv = b.results()
                times.append(float(b.stage_times()[2]))
            if ref is None:
                ref = e.copy()
            ok = bool(conv.all()) and float(np.max(np.abs(e - ref))) < 1e-8
            rows.append({"orbital_update": mode, "diis": diis, "scf_ms": float(np.median(times)),
                         "mean_iterations": float(it.mean()), "eligible": ok})
    del b
    return rows


def write_table(path, choice, measured, device):
    modes = [MODE_CODE[choice[k][0]] for k in range(BINS)]
    diis = [choice[k][1] for k in range(BINS)]
    lines = ["// SCF choices per molecule-size bin of 32 AOs (bin k: 32k .. 32k+31 AOs, the",
             "// last bin open), the defaults of ScfParams.  Written by the autotuner",
             "// (python -m sparrow_b200.autotune); regenerate it after changing the SCF",
             "// kernels.  Orbital update: 0 exact, 1 hybrid, 2 rotation.",
             "//",
             "// Measured on %s: SCF device ms of each bin's batch per candidate" % device,
             "// (orbital update / Pulay subspace), the chosen one marked *."]
    for k in sorted(measured):
        best = choice[k]
        cells = []
        for r in measured[k]["rows"]:
            tag = "%s/%d %.1f" % (r["orbital_update"][0], r["diis"], r["scf_ms"])
            if (r["orbital_update"], r["diis"]) == best:
                tag += "*"
            if not r["eligible"]:
                tag += "(x)"
            cells.append(tag)
        lines.append("//   bin %2d (%d molecules): %s" % (k, measured[k]["molecules"], ", ".join(cells)))
    lines += ["#pragma once",
              "#define SGB_TUNED_ORBITAL_UPDATE {%s}" % ", ".join(str(v) for v in modes),
              "#define SGB_TUNED_DIIS_SIZE {%s}" % ", ".join(str(v) for v in diis)]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--out", default=os.path.join(ROOT, "sparrow_b200", "csrc", "tuned_table.h"))
    p.add_argument("--json", default=None, help="also write the measurements as JSON")
    p.add_argument("--max-bin", type=int, default=9, help="largest bin measured (bins above inherit)")
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--seed", type=int, default=31)
    args = p.parse_args()
    sys.path.insert(0, ROOT)
    import torch
    device = torch.cuda.get_device_name(0)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    measured, choice = {}, {}
    t0 = time.time()
    for k in range(args.max_bin + 1):
        count = sms * (4 if k < 6 else 1)
        mols = bin_molecules(k, count, args.seed)
        if not mols:
            continue
        rows = measure_bin(mols, args.reps)
        ok = [r for r in rows if r["eligible"]]
        best = min(ok, key=lambda r: r["scf_ms"])
        choice[k] = (best["orbital_update"], best["diis"])
        measured[k] = {"molecules": len(mols), "rows": rows}
        print("bin %d: %s/%d %.2f ms (%d eligible)" % (k, best["orbital_update"], best["diis"], best["scf_ms"],
                                                       len(ok)), flush=True)
    last = max(choice)
    for k in range(BINS):
        if k not in choice:
            choice[k] = choice[min(last, max([j for j in choice if j <= k], default=last))]
    write_table(args.out, choice, measured, device)
    summary = {"device": device, "seconds": time.time() - t0,
               "table": {k: list(choice[k]) for k in range(BINS)}, "measured": measured}
    if args.json:
        with open(args.json, "w") as f:
            json.dump(summary, f)
    print(json.dumps({"device": device, "table": summary["table"], "seconds": summary["seconds"]}))


if __name__ == "__main__":
    main()
