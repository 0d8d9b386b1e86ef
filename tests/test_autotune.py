"""The autotuner's host logic (no GPU): the size bins of its workloads and
the table it writes."""
import re

import numpy as np

from sparrow_b200 import autotune


def _nao(Z):
    return int(sum(1 if z == 1 else 4 for z in Z))


def test_bin_workloads_fall_in_their_bins():
    for k in range(10):
        mols = autotune.bin_molecules(k, 12, seed=5)
        assert mols, k
        for Z, x in mols:
            n = _nao(Z)
            assert max(32 * k, 2) <= n <= 32 * k + 31, (k, n)
            assert x.shape == (len(Z), 3)


def test_written_table_parses(tmp_path):
    rows = [{"orbital_update": m, "diis": d, "scf_ms": 1.0 + i, "mean_iterations": 12.0, "eligible": True}
            for i, (m, d) in enumerate((m, d) for m in autotune.MODES for d in (4, 5, 6))]
    choice = {k: ("hybrid" if k < 3 else "exact", 6 if k < 5 else 5) for k in range(autotune.BINS)}
    out = tmp_path / "t.h"
    autotune.write_table(str(out), choice, {0: {"molecules": 10, "rows": rows}}, "test device")
    text = out.read_text()
    modes = re.search(r"#define SGB_TUNED_ORBITAL_UPDATE \{([^}]*)\}", text).group(1)
    diis = re.search(r"#define SGB_TUNED_DIIS_SIZE \{([^}]*)\}", text).group(1)
    modes = [int(v) for v in modes.split(",")]
    diis = [int(v) for v in diis.split(",")]
    assert len(modes) == len(diis) == autotune.BINS
    assert modes[:3] == [1, 1, 1] and modes[3] == 0 and diis[4] == 6 and diis[5] == 5
    assert "e/4 1.0*" not in text and "h/6" in text


def test_library_table_matches_header():
    import os
    import sparrow_b200
    text = open(os.path.join(os.path.dirname(autotune.__file__), "csrc", "tuned_table.h")).read()
    modes = [int(v) for v in re.search(r"ORBITAL_UPDATE \{([^}]*)\}", text).group(1).split(",")]
    names = {0: "exact", 1: "hybrid", 2: "rotation"}
    table = sparrow_b200.tuning_table()
    assert [names[m] for m in modes] == [t[1] for t in table]
