"""Oracle energies and gradients of the large water clusters (H2O)_256 and
(H2O)_512 (1536 / 3072 AOs), PM6, rms(dP) 1e-8, seed 0 of the water-cluster
generator: the "vs the reference" column of the large-molecule path.

The oracle sums the energy with compensated (Neumaier) summation: a plain
running sum over the 2.4M / 9.4M density-matrix terms lost 1.6e-8 and 6.0e-7
Hartree at these sizes.

Run from the repository root (CPU only, single-threaded oracle; about 12 and
117 minutes):  python tests/golden/make_large_water_golden.py 256 512
Each size is written to tests/golden/large_water_pm6_<n>.json.
"""
import json
import os
import sys
import time

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", ".."))

from sparrow_b200 import geometry  # noqa: E402
from tests import oracle_lib as O  # noqa: E402


def main(sizes):
    for n in sizes:
        Z, xa = geometry.water_cluster(n, seed=0)
        x = geometry.to_bohr(xa)
        t0 = time.time()
        r = O.scf("PM6", Z, x, scc=1e-7, rmsd=1e-8)
        rec = {"method": "PM6", "waters": n, "seed": 0, "nao": r["nao"], "nocc": r["nocc"], "energy": r["energy"],
               "e_el": r["e_el"], "e_rep": r["e_rep"], "iterations": r["iterations"], "converged": r["converged"],
               "gradient": [round(v, 12) for v in r["gradient"].reshape(-1).tolist()],
               "oracle_seconds": round(time.time() - t0, 1)}
        out = os.path.join(os.path.dirname(__file__), "large_water_pm6_%d.json" % n)
        with open(out, "w") as f:
            json.dump(rec, f)
        print(n, rec["energy"], rec["iterations"], rec["oracle_seconds"], flush=True)


if __name__ == "__main__":
    main([int(a) for a in sys.argv[1:]] or [256, 512])
