"""Benchmark: batched PM6 SCF solves/s on one B200.

Workload: 4096 saturated hydrocarbons C_nH_{2n+2}, n uniform in [2, 30]
(8-92 atoms, 14-182 AOs), seeded synthetic geometries (numpy PCG64, seed 1),
PM6, restricted SCF to |dE| < 1e-7 Eh and rms(dP) < 1e-8, FP64, energy and
nuclear gradient per molecule.  One step = one batched single point
(integrals -> SCF -> gradient) over all 4096 molecules.

Arms:
  default            the sm_100a engine through the C-ABI (libsparrow_b200.so)
  --impl reference   the reference's path restated on the CPU (the oracle,
                     oracle/liboracle_nddo.so), timed on this machine's cores

Output: one JSON line (rank 0).  `value` is device-timed throughput with the
inputs resident in HBM; `e2e` is the same metric through sg_batch_calculate
from host buffers (host setup, H2D copies, kernels, D2H of energies and
gradients); `roofline` is the dominant kernel (the persistent SCF kernel)
against the measured FP64 GEMM rate; `cpu_baseline` is the oracle on a
bounded random sample of the same molecules.  Side legs (rank 0): the plain
one-molecule-per-launch GPU form, the request server's p50/p99 latency, and
the large-molecule path on (H2O)_256/512/1024 in FP64 and mixed precision,
and DFTB3 + TD-DFTB excitations over 1024 polyenes; PM6 on one (H2O)_32
cluster (the plain single-point form against the oracle on one and on all
cores) and the batch with AM1.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_MOLECULES = 4096
SEED = 1
METHOD = "PM6"
SCC = 1e-7
RMSD = 1e-8
MAX_ITER = 100
CORE_CHARGE = {1: 1, 6: 4, 7: 5, 8: 6}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="sparrow_b200", choices=["sparrow_b200", "reference"])
    p.add_argument("--molecules", type=int, default=N_MOLECULES)
    p.add_argument("--method", default=METHOD)
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU time of the cpu_baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-serving", action="store_true", help="skip the request-server latency leg")
    p.add_argument("--no-large", action="store_true", help="skip the large-molecule (water cluster) leg")
    p.add_argument("--no-tddftb", action="store_true", help="skip the DFTB3 + TD-DFTB polyene leg")
    p.add_argument("--no-plain", action="store_true", help="skip the plain one-molecule-per-launch GPU leg")
    p.add_argument("--no-open-shell", action="store_true", help="skip the unrestricted (radical) leg")
    p.add_argument("--no-hessian", action="store_true", help="skip the semi-numerical Hessian leg")
    p.add_argument("--no-water32", action="store_true", help="skip the (H2O)_32 single-point leg")
    p.add_argument("--no-am1", action="store_true", help="skip the AM1 batch leg")
    p.add_argument("--large-sizes", default="256,512,1024", help="water counts of the large-molecule leg")
    p.add_argument("--serving-loads", default="500,1000,2000,4000,8000,16000,20000",
                   help="offered loads (req/s) of the serving leg")
    p.add_argument("--serving-seconds", type=float, default=2.0, help="arrival window per offered load")
    p.add_argument("--serving-slots", type=int, default=8, help="concurrent batches of the request server")
    return p.parse_args()


def molecules_for(rank, count, seed=SEED):
    from sparrow_b200 import geometry
    mols = geometry.alkane_batch(count, seed=seed + 1000 * rank)
    return [(z, geometry.to_bohr(x)) for z, x in mols]


# ----------------------------------------------------------------------------
# CPU side (the oracle): molecule-parallel over host processes
# ----------------------------------------------------------------------------
def _oracle_solve(args):
    method, Z, x = args
    from tests import oracle_lib
    t0 = time.perf_counter()
    r = oracle_lib.scf(method, Z, x, scc=SCC, rmsd=RMSD, max_iter=MAX_ITER, gradient=True)
    return time.perf_counter() - t0, r["energy"], r["iterations"], r["gradient"]


def cpu_rate(method, mols, target_seconds, procs, rng_seed=12345):
    """Oracle throughput (solves/s) on a random sample sized to ~target_seconds of wall time."""
    import multiprocessing as mp
    import numpy as np
    rng = np.random.default_rng(rng_seed)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        # calibrate on a few molecules
        calib = [mols[i] for i in rng.choice(len(mols), size=min(procs, 8), replace=False)]
        res = pool.map(_oracle_solve, [(method, z, x) for z, x in calib])
        per_mol = sum(r[0] for r in res) / len(res)
        count = int(max(procs, min(len(mols), target_seconds * procs / max(per_mol, 1e-3))))
        idx = rng.choice(len(mols), size=count, replace=False)
        sample = [mols[i] for i in idx]
        t0 = time.perf_counter()
        res = pool.map(_oracle_solve, [(method, z, x) for z, x in sample], chunksize=1)
        wall = time.perf_counter() - t0
    # (molecule index, oracle energy, oracle gradient) of the timed sample
    return count / wall, count, wall, [(int(i), r[1], r[3]) for i, r in zip(idx, res)]


def plain_gpu_rate(method, mols, target_seconds=8.0, max_count=512, rng_seed=777):
    """The plain GPU form: one molecule per launch sequence through the
    Calculator surface (set_structure / calculate), host buffers in and out,
    one molecule at a time, on a random sample of the batch."""
    import numpy as np
    import sparrow_b200
    rng = np.random.default_rng(rng_seed)
    order = rng.permutation(len(mols))[:max_count]
    calc = sparrow_b200.get_calculator(method)
    calc.settings["self_consistence_criterion"] = SCC
    calc.settings["density_rmsd_criterion"] = RMSD
    calc.settings["max_scf_iterations"] = MAX_ITER
    calc.set_required_properties(["energy", "gradients"])
    z, x = mols[order[0]]
    calc.set_structure(z, x)
    calc.calculate()  # warm-up: module load, pools
    count, t0 = 0, time.perf_counter()
    energies = []
    for i in order:
        z, x = mols[i]
        calc.set_structure(z, x)
        energies.append(calc.calculate().energy)
        count += 1
        if time.perf_counter() - t0 > target_seconds:
            break
    wall = time.perf_counter() - t0
    return count / wall, count, wall


def serving_mix(count, seed=5):
    """The serving request mix: alkanes C_nH_2n+2 (n ~ U[1,60]) or water
    clusters (H2O)_n (n ~ U[2,64]), 70 % PM6 and 30 % DFTB2 (mio-1-1)."""
    import numpy as np
    from sparrow_b200 import geometry
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        if rng.random() < 0.5:
            z, x = geometry.alkane(int(rng.integers(1, 61)), rng)
        else:
            z, x = geometry.water_cluster(int(rng.integers(2, 65)), seed=int(rng.integers(1 << 30)))
        out.append((np.ascontiguousarray(z, dtype=np.int32), np.ascontiguousarray(geometry.to_bohr(x)).reshape(-1),
                    "PM6" if rng.random() < 0.7 else "DFTB2"))
    return out


def serving_offline(pool):
    """Offline ceiling of the serving mix: the pool's requests as one batch
    per method (energy + gradient), device time of the launch sequence after
    a warm-up run."""
    import sparrow_b200
    by = {}
    for z, x, m in pool:
        by.setdefault(m, []).append((z, x.reshape(-1, 3)))
    dev_ms = 0.0
    wall_s = 0.0
    for m, mols in by.items():
        b = sparrow_b200.Batch(m, mols, scc=SCC, rmsd=RMSD, max_iter=MAX_ITER)
        b.run(gradients=True)
        t0 = time.perf_counter()
        b.run(gradients=True)
        b.results()
        wall_s += time.perf_counter() - t0
        dev_ms += float(sum(b.stage_times()))
        del b
    return {"requests": len(pool), "device_rps": len(pool) / (dev_ms * 1e-3), "wall_rps": len(pool) / wall_s,
            "methods": {m: len(v) for m, v in by.items()}}


def serving_leg(loads=(500, 1000, 2000, 4000, 8000, 16000, 20000), seconds=2.0, slots=8, plain_count=48, seed=5):
    """Open-loop Poisson arrivals into the request server at each offered load
    (req/s) for `seconds`; latency = completion - submission, timed by the
    server.  Beside it, the offline ceiling (the same mix as whole batches)
    and the plain form: the same requests one at a time through one
    Calculator (closed loop)."""
    import numpy as np
    import sparrow_b200
    pool = serving_mix(2048, seed)
    out = {"mix": "alkanes n~U[1,60] | (H2O)_n n~U[2,64], 70% PM6 / 30% DFTB2 (mio-1-1), "
                  "energy+gradient, 3-384 AOs", "slots": slots, "seconds_per_load": seconds, "loads": []}
    out["offline"] = serving_offline(pool)
    rng = np.random.default_rng(seed + 1)
    with sparrow_b200.Server(device_budget_gb=64.0, slots=slots, scc=SCC, rmsd=RMSD, max_iter=MAX_ITER) as srv:
        # warm-up: every code path and the arena pools
        for r in [srv.submit(m, z, x) for z, x, m in pool[:64]]:
            srv.wait(r)
        for lam in loads:
            n = int(lam * seconds)
            gaps = rng.exponential(1.0 / lam, size=n)
            picks = rng.integers(0, len(pool), size=n)
            ids = []
            t0 = time.perf_counter()
            t_next = t0
            for k in range(n):
                t_next += gaps[k]
                dt = t_next - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                z, x, m = pool[picks[k]]
                ids.append(srv.submit(m, z, x))
            t_sub = time.perf_counter() - t0
            lat = []
            it = []
            for r in ids:
                res = srv.wait(r)
                lat.append(res.latency_s)
                it.append(res.iterations)
            t_all = time.perf_counter() - t0
            st = srv.stats()
            lat = np.array(lat) * 1e3
            out["loads"].append({"offered_rps": lam, "requests": n, "achieved_rps": n / t_all,
                                 "submit_rps": n / t_sub, "p50_ms": float(np.percentile(lat, 50)),
                                 "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                                 "batches_so_far": st["batches"], "max_batch": st["max_batch"]})
    # plain form: one request at a time through the Calculator surface
    lat = []
    calcs = {}
    for k in range(plain_count):
        z, x, m = pool[k]
        c = calcs.get(m)
        if c is None:
            c = sparrow_b200.get_calculator(m)
            c.settings["self_consistence_criterion"] = SCC
            c.settings["density_rmsd_criterion"] = RMSD
            c.settings["max_scf_iterations"] = MAX_ITER
            c.set_required_properties(["energy", "gradients"])
            calcs[m] = c
        t0 = time.perf_counter()
        c.set_structure(z, x)
        c.calculate()
        lat.append(time.perf_counter() - t0)
    lat = np.array(lat[2:]) * 1e3
    out["plain_gpu"] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                        "throughput_rps": 1e3 / float(lat.mean()), "requests": int(lat.size)}
    return out


def cublas_bf16_product_ms(Np, reps=10):
    """Device ms of cuBLAS (through torch) for the split-BF16 product's shape:
    (Np x 4Np) times (4Np x Np)^T, BF16 in, FP32 accumulation (FP32 out where
    torch offers it, else BF16 out)."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(1)
    a = torch.randn((Np, 4 * Np), device="cuda", dtype=torch.bfloat16, generator=g)
    b = torch.randn((Np, 4 * Np), device="cuda", dtype=torch.bfloat16, generator=g)
    try:
        f = lambda: torch.mm(a, b.t(), out_dtype=torch.float32)  # noqa: E731
        f()
        out = "fp32"
    except (TypeError, RuntimeError):
        f = lambda: torch.mm(a, b.t())  # noqa: E731
        out = "bf16"
    for _ in range(3):
        f()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        f()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del a, b
    torch.cuda.empty_cache()
    return ms, out


def large_leg(sizes=(256, 512, 1024), seed=0):
    """Mixed-precision PM6 on large water clusters (the large-molecule path):
    per size the FP64 path and the split-BF16 path (energy + gradient), device
    ms of the SCF stage, wall ms of run + results, and the energy error of the
    mixed path against the FP64 GPU path and, where the oracle's fixture
    exists (tests/golden/large_water_pm6_<n>.json), of both against the
    oracle.  The purification products are timed on the device: the mixed
    path's tensor-core GEMM (this library's tcgen05 kernel) per product beside
    cuBLAS on the same shape, and the FP64 squares (cuBLAS DSYRK)."""
    import numpy as np
    import sparrow_b200
    from sparrow_b200 import geometry
    rows = []
    warm = True
    for n in sizes:
        Z, xa = geometry.water_cluster(n, seed=seed)
        x = geometry.to_bohr(xa)
        gold = None
        gp = os.path.join(ROOT, "tests", "golden", "large_water_pm6_%d.json" % n)
        if os.path.exists(gp):
            with open(gp) as f:
                gold = json.load(f)
        row = {"waters": n, "nao": 6 * n, "atoms": 3 * n}
        for path in ("large", "large_mixed"):
            reps = 2 if warm else 1  # the first run of the process pays cuBLAS module loading
            for _ in range(reps):
                b = sparrow_b200.Batch("PM6", [(Z, x)], scc=SCC, rmsd=RMSD, max_iter=MAX_ITER, scf_path=path)
                t0 = time.perf_counter()
                b.run(gradients=True)
                e, g, it, conv = b.results()
                wall = time.perf_counter() - t0
                st = b.stage_times()
                nm, ns, pcyc = b.scf_stats()
                pc = [int(v) for v in pcyc[0]]
                del b
            r = {"energy": float(e[0]), "converged": bool(conv[0]), "iterations": int(it[0]),
                 "mixed_iterations": int(nm[0]), "sp2_steps": int(ns[0]), "scf_ms": float(st[2]),
                 "total_device_ms": float(sum(st)), "wall_ms": wall * 1e3}
            if pc[1] > 0:
                r["tc_gemm_products"] = int(pc[1])
                r["tc_gemm_ms_per_product"] = pc[0] / pc[1] / 1e6
            if pc[3] > 0:
                r["fp64_dsyrk_products"] = int(pc[3])
                r["fp64_dsyrk_ms_per_product"] = pc[2] / pc[3] / 1e6
            if gold is not None:
                r["dE_vs_oracle"] = float(e[0]) - gold["energy"]
                r["max_dgrad_vs_oracle"] = float(np.max(np.abs(g[0].reshape(-1) - np.array(gold["gradient"]))))
            row[path] = r
        warm = False
        Np = (6 * n + 127) // 128 * 128
        cb_ms, cb_out = cublas_bf16_product_ms(Np)
        flops = 8.0 * Np ** 3
        rm = row["large_mixed"]
        row["split_bf16_product"] = {
            "shape": "(%d x %d) x (%d x %d)^T, BF16 in, FP32 accumulation" % (Np, 4 * Np, Np, 4 * Np),
            "flops": flops,
            "tc_gemm_ms": rm.get("tc_gemm_ms_per_product"),
            "tc_gemm_tflops": flops / rm["tc_gemm_ms_per_product"] / 1e9 if rm.get("tc_gemm_ms_per_product") else None,
            "cublas_ms": cb_ms, "cublas_out": cb_out, "cublas_tflops": flops / cb_ms / 1e9,
            "tc_over_cublas_time": rm["tc_gemm_ms_per_product"] / cb_ms if rm.get("tc_gemm_ms_per_product") else None}
        row["dE_mixed_vs_fp64"] = row["large_mixed"]["energy"] - row["large"]["energy"]
        row["speedup_mixed_over_fp64"] = row["large"]["total_device_ms"] / row["large_mixed"]["total_device_ms"]
        rows.append(row)
    return {"workload": "PM6 (H2O)_n, n in %s, seed %d, one molecule over the whole GPU, energy+gradient, "
                        "rms dP 1e-8" % (list(sizes), seed), "sizes": rows}


def tddftb_leg(count=1024, seed=6, nroots=8, cpu_seconds=10.0):
    """DFTB3 (3ob-3-1) ground state plus TD-DFTB for the lowest singlets over a
    batch of polyenes C_2kH_2k+2, k ~ U[5,40]: device ms of the SCF and of the
    excitations, molecules/s, Davidson outcome; the CPU oracle (dense Casida)
    on a bounded sample of the smallest molecules of the batch, with the
    largest excitation-energy difference of the GPU on that sample."""
    import numpy as np
    import sparrow_b200
    from sparrow_b200 import geometry
    mols = [(z, geometry.to_bohr(x)) for z, x in geometry.polyene_batch(count, seed=seed)]
    out = {"workload": "%d polyenes C_2kH_2k+2, k~U[5,40], seed %d, DFTB3 3ob-3-1, rms dP 1e-10, %d lowest singlets "
                       "(full TD-DFTB, Davidson residual 1e-10)" % (count, seed, nroots)}
    for rep in range(2):  # the first pass pays module loading
        b = sparrow_b200.Batch("DFTB3", mols, scc=1e-9, rmsd=1e-10, max_iter=300)
        b.record_event(0)
        b.run()
        b.record_event(1)
        e, _, it, conv = b.results()
        b.record_event(2)
        om, mu, st = b.excitations(nroots)
        b.record_event(3)
        scf_ms, td_ms = b.elapsed_ms(0, 1), b.elapsed_ms(2, 3)
    cyc = b.excitation_cycles().astype(float)
    out.update({"scf_ms": scf_ms, "tddftb_ms": td_ms, "molecules_per_s": count / ((scf_ms + td_ms) / 1e3),
                "scf_converged": int(conv.sum()), "mean_scf_iterations": float(it.mean()),
                "excitations_ok": int((st == 0).sum()),
                "tddftb_cycle_share": {"canonical_orbitals": float(cyc[:, 0].sum() / cyc.sum()),
                                       "transition_charges": float(cyc[:, 1].sum() / cyc.sum()),
                                       "davidson": float(cyc[:, 2].sum() / cyc.sum())}})
    # CPU oracle on a random sample across the whole k range, all host cores
    import multiprocessing as mp
    procs = host_cores()
    rng = np.random.default_rng(99)
    pick = rng.choice(count, size=min(count, procs), replace=False)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        t0 = time.perf_counter()
        res = pool.map(_oracle_tddftb, [(3, mols[i][0], mols[i][1], nroots) for i in pick], chunksize=1)
        wall = time.perf_counter() - t0
    dmax, mmax = 0.0, 0.0
    for i, (_, omr, dpr) in zip(pick, res):
        dmax = max(dmax, float(np.max(np.abs(omr - om[i][:len(omr)]))))
        for r_ in range(len(omr)):
            sgn = 1.0 if np.dot(dpr[r_], mu[i][r_]) >= 0 else -1.0
            mmax = max(mmax, float(np.max(np.abs(dpr[r_] - sgn * mu[i][r_]))))
    ks = sorted((len(mols[i][0]) - 2) // 4 for i in pick)
    out["cpu_baseline"] = {"value": len(pick) / wall, "unit": "molecules/s", "cores": procs, "kind": "port",
                           "cpu": cpu_info(),
                           "sample": "%d random polyenes of the batch (k = %s), oracle DFTB3 SCF + TD-DFTB (dense "
                                     "Casida up to 2000 transitions, matrix-free Davidson above), one per process, "
                                     "%.1f s wall" % (len(pick), ",".join(str(k) for k in ks), wall),
                           "max_abs_domega_gpu_vs_oracle_hartree": dmax,
                           "max_abs_dmu_gpu_vs_oracle_ebohr": mmax}
    return out


def _oracle_tddftb(args):
    order, Z, x, nroots = args
    from tests import oracle_lib as O
    t0 = time.perf_counter()
    r = O.dftb_tddftb(order, Z, x, nroots=nroots, scc=1e-9, rmsd=1e-10)
    return time.perf_counter() - t0, r["omega"], r["dipoles"]


def _oracle_plain(args):
    method, Z, x, reps = args
    from tests import oracle_lib as O
    out = []
    for _ in range(reps):
        t0 = time.perf_counter()
        r = O.scf(method, Z, x, scc=SCC, rmsd=RMSD, max_iter=MAX_ITER, gradient=True)
        out.append(time.perf_counter() - t0)
    return out, r["energy"], r["gradient"]


def water32_leg(gpu_calls=20):
    """PM6 energy + gradient of one (H2O)_32 cluster (96 atoms, 192 AOs; the
    4x4x2 jittered grid, seed 0), rms dP 1e-8: the plain GPU form (one
    Calculator.calculate per solve, host buffers in and out) on the batched
    kernel (one CTA) and on the whole-GPU large-molecule path, the oracle on
    one core (one solve after another) and on all cores (independent solves,
    one per process), with the GPU's energy and gradient errors."""
    import multiprocessing as mp
    import numpy as np
    import sparrow_b200
    from sparrow_b200 import geometry
    Z, xa = geometry.water_cluster(32, seed=0)
    x = geometry.to_bohr(xa)
    calc = sparrow_b200.get_calculator("PM6")
    calc.settings["self_consistence_criterion"] = SCC
    calc.settings["density_rmsd_criterion"] = RMSD
    calc.set_required_properties(["energy", "gradients"])
    calc.set_structure(Z, x)
    for _ in range(3):
        res = calc.calculate()
    lat = []
    for _ in range(gpu_calls):
        t0 = time.perf_counter()
        calc.set_structure(Z, x)
        res = calc.calculate()
        lat.append(time.perf_counter() - t0)
    lat = np.array(lat) * 1e3
    # the same solve on the whole-GPU large-molecule path (every SM on one
    # molecule; energy and gradient, no orbitals)
    calc_l = sparrow_b200.get_calculator("PM6")
    calc_l.settings["self_consistence_criterion"] = SCC
    calc_l.settings["density_rmsd_criterion"] = RMSD
    calc_l.settings["scf_path"] = "large"
    calc_l.set_required_properties(["energy", "gradients"])
    calc_l.set_structure(Z, x)
    for _ in range(3):
        res_l = calc_l.calculate()
    lat_l = []
    for _ in range(gpu_calls):
        t0 = time.perf_counter()
        calc_l.set_structure(Z, x)
        res_l = calc_l.calculate()
        lat_l.append(time.perf_counter() - t0)
    lat_l = np.array(lat_l) * 1e3
    procs = host_cores()
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        one = pool.map(_oracle_plain, [("PM6", Z, x, 3)])[0]
        t0 = time.perf_counter()
        allc = pool.map(_oracle_plain, [("PM6", Z, x, 1)] * procs)
        wall_all = time.perf_counter() - t0
    t1 = float(np.median(one[0]))
    return {"workload": "PM6 (H2O)_32, 96 atoms, 192 AOs, seed 0, energy+gradient, rms dP 1e-8",
            "gpu_plain": {"p50_ms": float(np.median(lat)), "p99_ms": float(np.percentile(lat, 99)),
                          "solves_per_s": 1e3 / float(np.median(lat)), "iterations": int(res.iterations)},
            "cpu_1core": {"seconds_per_solve": t1, "solves_per_s": 1.0 / t1, "kind": "port", "cores": 1,
                          "cpu": cpu_info()},
            "cpu_all_cores": {"solves_per_s": procs / wall_all, "cores": procs, "kind": "port",
                              "sample": "%d independent solves, one per process" % procs},
            "gpu_over_cpu_1core": t1 / (float(np.median(lat)) / 1e3),
            "abs_dE_hartree": abs(res.energy - one[1]),
            "max_abs_dgrad_hartree_per_bohr": float(np.max(np.abs(res.gradients - one[2]))),
            "gpu_large_path": {"p50_ms": float(np.median(lat_l)), "p99_ms": float(np.percentile(lat_l, 99)),
                               "solves_per_s": 1e3 / float(np.median(lat_l)), "iterations": int(res_l.iterations),
                               "gpu_over_cpu_1core": t1 / (float(np.median(lat_l)) / 1e3),
                               "abs_dE_hartree": abs(res_l.energy - one[1]),
                               "max_abs_dgrad_hartree_per_bohr": float(np.max(np.abs(res_l.gradients - one[2])))}}


def am1_leg(mols, steps=3, cpu_seconds=10.0):
    """The same 4096-alkane batch with AM1: device solves/s of the batched
    energy + gradient (CUDA events over `steps` runs), and the oracle on a
    random sample over all host cores with the GPU's largest errors on it."""
    import numpy as np
    import sparrow_b200
    b = sparrow_b200.Batch("AM1", mols, scc=SCC, rmsd=RMSD, max_iter=MAX_ITER)
    for _ in range(2):
        b.run(gradients=True)
        e, g, it, conv = b.results()
    b.record_event(0)
    for _ in range(steps):
        b.run(gradients=True)
        e, g, it, conv = b.results()
    b.record_event(1)
    ms = b.elapsed_ms(0, 1) / steps
    procs = host_cores()
    rate, count, wall, cpu_results = cpu_rate("AM1", mols, cpu_seconds, procs, rng_seed=4242)
    return {"workload": "%d alkanes C_nH_2n+2, n~U[2,30], AM1 energy+gradient, rms dP 1e-8" % len(mols),
            "value": len(mols) / (ms / 1e3), "unit": "solves/s", "ms_per_step": ms,
            "mean_scf_iterations": float(np.mean(it)), "not_converged": int((~conv).sum()),
            "cpu_baseline": {"value": rate, "unit": "solves/s", "cores": procs, "kind": "port", "cpu": cpu_info(),
                             "sample": "%d random molecules, molecule-parallel over %d processes, %.1f s wall" % (
                                 count, procs, wall),
                             "max_abs_dE_gpu_vs_oracle_hartree": float(max(abs(e[i] - eo) for i, eo, _ in cpu_results)),
                             "max_abs_dgrad_gpu_vs_oracle_hartree_per_bohr": float(
                                 max(np.max(np.abs(g[i] - go)) for i, _, go in cpu_results))},
            "device_over_cpu": (len(mols) / (ms / 1e3)) / rate}


def open_shell_leg(count=1024, seed=8, cpu_seconds=5.0):
    """Unrestricted SCF throughput: a batch of alkyl radicals (alkanes C_nH_2n+2,
    n ~ U[2,30], without their last hydrogen; doublets), energy+gradient, PM6
    (UHF) and DFTB2 mio-1-1 (spin-polarised): device ms and solves/s, with the
    CPU oracle on a bounded sample of the same radicals (PM6)."""
    import numpy as np
    import sparrow_b200
    from sparrow_b200 import geometry
    rad = [(np.asarray(z)[:-1], geometry.to_bohr(x)[:-1]) for z, x in geometry.alkane_batch(count, seed=seed)]
    out = {"workload": "%d alkyl radicals C_nH_2n+1 (n~U[2,30], seed %d), doublets, energy+gradient, rms dP 1e-8" % (
        count, seed)}
    energies = {}
    for method in ("PM6", "DFTB2"):
        for rep in range(2):  # the first pass pays module loading
            b = sparrow_b200.Batch(method, rad, multiplicities=[2] * count, scc=1e-7, rmsd=1e-8, max_iter=300)
            b.record_event(0)
            b.run(gradients=True)
            b.record_event(1)
            e, _, it, conv = b.results()
            ms = b.elapsed_ms(0, 1)
        energies[method] = e
        out[method] = {"device_ms": ms, "solves_per_s": count / (ms / 1e3), "converged": int(conv.sum()),
                       "mean_iterations": float(it.mean())}
    from tests import oracle_lib as O
    rng = np.random.default_rng(3)
    t0, done, dmax = time.perf_counter(), 0, 0.0
    for i in rng.permutation(count):
        if time.perf_counter() - t0 > cpu_seconds:
            break
        r = O.scf_uhf("PM6", rad[i][0], rad[i][1], 2, scc=1e-7, rmsd=1e-8)
        dmax = max(dmax, abs(r["energy"] - energies["PM6"][i]))
        done += 1
    wall = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": done / wall, "unit": "solves/s", "cores": 1, "kind": "port", "cpu": cpu_info(),
                           "sample": "%d random radicals of the batch, oracle PM6 UHF energy+gradient, %.1f s wall" % (
                               done, wall),
                           "max_abs_dE_gpu_vs_oracle_hartree": dmax}
    return out


def hessian_leg(cpu_step_seconds=30.0):
    """Semi-numerical Hessian (central differences of analytic gradients, 0.01
    bohr; the reference's only Hessian): the 28-atom structure of the
    reference's frequency tests and a C30H62 alkane, PM6.  GPU wall ms (all 6n
    displaced geometries as batches) against the CPU oracle doing the same
    displacements one after another (sft_1 only), and the lowest harmonic
    frequency of sft_1 against the reference's -125.561 cm^-1."""
    import json as _json
    import numpy as np
    import sparrow_b200
    from sparrow_b200 import geometry
    from tests import harmonic
    from tests import oracle_lib as O
    gold = _json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden",
                                        "hessian_known_answers.json")))
    st = gold["structures"]["sft_1"]
    sym = {"H": 1, "C": 6, "N": 7, "O": 8}
    Z = [sym[e] for e in st["elements"]]
    x = np.array(st["xyz_angstrom"]) * O.bohr_per_angstrom()
    out = {"workload": "PM6 Hessians: sft_1 (C10H14O4, 28 atoms, 168 displaced geometries) and C30H62 "
                       "(92 atoms, 552 displaced geometries)"}
    sparrow_b200.hessian("PM6", Z, x)  # module loading
    t0 = time.perf_counter()
    H, nc = sparrow_b200.hessian("PM6", Z, x, scc=1e-9, rmsd=1e-9)
    gpu_ms = (time.perf_counter() - t0) * 1e3
    f = harmonic.frequencies(Z, x, H)
    rng = np.random.default_rng(1)
    za, xa = geometry.alkane(30, rng)
    t0 = time.perf_counter()
    Hb, ncb = sparrow_b200.hessian("PM6", za, geometry.to_bohr(xa))
    big_ms = (time.perf_counter() - t0) * 1e3
    # the oracle: the same central differences, displacement after displacement, on a bounded share
    t0, done = time.perf_counter(), 0
    for k in range(3 * len(Z)):
        if time.perf_counter() - t0 > cpu_step_seconds:
            break
        for sgn in (1, -1):
            xs = x.copy().reshape(-1)
            xs[k] += 0.01 * sgn
            O.scf("PM6", Z, xs.reshape(-1, 3), scc=1e-9, rmsd=1e-9)
        done += 1
    wall = time.perf_counter() - t0
    cpu_full_s = wall / max(done, 1) * 3 * len(Z)
    out["sft_1"] = {"gpu_wall_ms": gpu_ms, "not_converged": nc, "lowest_frequency_cm": float(f[0]),
                    "reference_lowest_frequency_cm": -125.561,
                    "cpu_baseline": {"value": cpu_full_s, "unit": "s per Hessian", "cores": 1, "kind": "port", "cpu": cpu_info(),
                                     "sample": "%d of %d coordinates (both displacements) in %.1f s, scaled" % (
                                         done, 3 * len(Z), wall)},
                    "gpu_over_cpu_1core": cpu_full_s / (gpu_ms / 1e3)}
    out["C30H62"] = {"gpu_wall_ms": big_ms, "not_converged": ncb}
    return out


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_info():
    """The host CPU as the CPU baselines see it: model string, logical CPUs,
    CPUs this process may run on, physical cores, OMP_NUM_THREADS."""
    model, phys = None, set()
    try:
        pid = cid = None
        for line in open("/proc/cpuinfo"):
            k, _, v = line.partition(":")
            k, v = k.strip(), v.strip()
            if k == "model name" and model is None:
                model = v
            elif k == "physical id":
                pid = v
            elif k == "core id":
                cid = v
            elif not k and pid is not None:
                phys.add((pid, cid))
                pid = cid = None
        if pid is not None:
            phys.add((pid, cid))
    except OSError:
        pass
    return {"model": model, "logical_cpus": os.cpu_count(), "usable_cpus": host_cores(),
            "physical_cores": len(phys) or None, "OMP_NUM_THREADS": os.environ.get("OMP_NUM_THREADS")}


# ----------------------------------------------------------------------------
# roofline bookkeeping (algorithmic FLOPs per SCF iteration)
# ----------------------------------------------------------------------------
def scf_flops(mols, iterations, diis=6):
    """F_eig = 4N^3, F_dens = 2 N^2 n_occ, F_G = 12 nnz(2c2e) + 256 heavy atoms,
    F_DIIS = 2N^3 + m^2 N^2, per iteration, summed over molecules."""
    total = 0.0
    for (Z, _), it in zip(mols, iterations):
        heavy = int((Z > 1).sum())
        light = len(Z) - heavy
        N = 4 * heavy + light
        nocc = sum(CORE_CHARGE[int(z)] for z in Z) // 2
        nnz = 100 * heavy * (heavy - 1) // 2 + 10 * heavy * light + light * (light - 1) // 2
        per = 4 * N ** 3 + 2 * N * N * nocc + 12 * nnz + 256 * heavy + 2 * N ** 3 + diis * diis * N * N
        total += per * int(it)
    return total


def fp64_gemm_peak():
    """cuBLAS FP64 GEMM rate (TFLOP/s) measured here: the FP64 roofline denominator."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.path = None

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(prefix="sparrow_b200_clocks_", suffix=".csv")
            self.f = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, gpu_index=0):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                if int(parts[0]) != gpu_index:
                    continue
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        try:
            os.unlink(self.path)
        except OSError:
            pass
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def load_traffic():
    """Per-launch DRAM bytes of the SCF kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "scf_kernel_ncu.json")
    try:
        return json.load(open(path))
    except Exception:
        return None


# ----------------------------------------------------------------------------
def workload_config(args, world):
    """The workload description both arms print: the same keys and values."""
    return {"workload": "%d alkanes C_nH_2n+2, n~U[2,30] per GPU, %s energy+gradient, rms dP 1e-8" % (
        args.molecules, args.method), "molecules_per_gpu": args.molecules, "method": args.method,
        "replicas": world, "l2": "inputs larger than L2: the batch's integrals and matrices occupy ~8 GB"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    mols = molecules_for(0, args.molecules)
    procs = host_cores()
    rates = []
    for step in range(args.warmup + args.steps):
        rate, count, wall, _ = cpu_rate(args.method, mols, max(3.0, args.cpu_seconds / 2), procs,
                                        rng_seed=777 + step)
        if step >= args.warmup:
            rates.append((rate, count, wall))
    value = sum(r[0] for r in rates) / len(rates)
    sample = "%d-%d random molecules of the %d-alkane batch per step, oracle (C++ FP64 restatement), " \
             "molecule-parallel over %d processes" % (min(r[1] for r in rates), max(r[1] for r in rates),
                                                       args.molecules, procs)
    line = {
        "impl": "reference", "metric": "%s SCF solves/s (energy+gradient)" % args.method, "value": value,
        "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(r[2] for r in rates) / len(rates), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, no dataset)",
        "config": workload_config(args, world),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": procs, "kind": "port", "sample": sample,
                         "cpu": cpu_info()},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# replicas: one rank per GPU, molecules sharded by rank (seeded per rank), no
# data-path collective; the process group only carries the barriers and the
# max-over-ranks of the timings
# ----------------------------------------------------------------------------
def init_ranks(world, timeout_s=300):
    """torch.distributed process group for world > 1 (NCCL with GPUs, gloo without), else None."""
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as td
    td.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                          timeout=datetime.timedelta(seconds=timeout_s))
    return td


def reduce_max(dist, v):
    """Maximum of v over the ranks (v itself without a process group)."""
    if dist is None:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_engine(args, rank, world):
    import numpy as np
    import sparrow_b200

    mols = molecules_for(rank, args.molecules)
    # CPU baseline first: its process pool must start before this process touches the GPU
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        procs = host_cores()
        rate, count, wall, cpu_results = cpu_rate(args.method, mols, args.cpu_seconds, procs)
        cpu = {"value": rate, "unit": "solves/s", "cores": procs, "kind": "port", "cpu": cpu_info(),
               "sample": "%d random molecules of the batch, oracle (C++ FP64 restatement of the reference path), "
                         "molecule-parallel over %d processes, %.1f s wall" % (count, procs, wall)}

    dist = init_ranks(world)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        return reduce_max(dist, v)

    peak = None
    if rank == 0:
        try:
            peak = fp64_gemm_peak()
        except Exception:
            peak = None

    b = sparrow_b200.Batch(args.method, mols, scc=SCC, rmsd=RMSD, max_iter=MAX_ITER)
    for _ in range(args.warmup):
        b.run(gradients=True)
        e, g, it, conv = b.results()
    stage_sum = np.zeros(4)
    clocks = ClockSampler()
    barrier()
    clocks.start()
    b.record_event(0)
    for _ in range(args.steps):
        b.run(gradients=True)
        e, g, it, conv = b.results()
        stage_sum += b.stage_times()
    b.record_event(1)
    dev_ms = b.elapsed_ms(0, 1)
    clk = clocks.stop()
    barrier()
    dev_ms = max_over_ranks(dev_ms)
    launches = b.launches * args.steps
    n_total = args.molecules * world
    value = n_total * args.steps / (dev_ms / 1e3)
    not_conv = int((~conv).sum())
    if cpu is not None:
        # accuracy of the timed run against the oracle on the CPU sample
        cpu["max_abs_dE_gpu_vs_oracle_hartree"] = float(max(abs(e[i] - eo) for i, eo, _ in cpu_results))
        cpu["max_abs_dgrad_gpu_vs_oracle_hartree_per_bohr"] = float(
            max(np.max(np.abs(g[i] - go)) for i, _, go in cpu_results))

    # the tuned table in force, against the previous fixed choices (a Jacobi
    # start and occupied-virtual rotations, Pulay subspace 6) on the same batch
    tuning = None
    if rank == 0:
        b.set_tuning("rotation", 6)
        b.run()
        b.results()
        b.run()
        b.results()
        fixed_ms = float(b.stage_times()[2])
        b.set_tuning(None, None)
        b.run()
        b.results()
        b.run()
        b.results()
        tuned_ms = float(b.stage_times()[2])
        tuning = {"table": [{"first_ao": t[0], "orbital_update": t[1], "diis_size": t[2]}
                            for t in sparrow_b200.tuning_table()],
                  "scf_ms_tuned": tuned_ms, "scf_ms_fixed_rotation_diis6": fixed_ms,
                  "gain_over_fixed": fixed_ms / tuned_ms}

    # end to end from host buffers through the public batch call (flat host
    # arrays in the C-ABI's layout, prepared once; every step creates the
    # batch, uploads, computes and reads energies and gradients back)
    t_e2e = []
    h2d = d2h = 0
    fn_atoms, fZ, fX = sparrow_b200.flatten_molecules(mols)
    for step in range(args.steps + 1):
        barrier()
        t0 = time.perf_counter()
        e2, g2, it2, conv2 = sparrow_b200.batch_calculate_flat(args.method, fn_atoms, fZ, fX, scc=SCC, rmsd=RMSD,
                                                               max_iter=MAX_ITER, gradients=True)
        dt = time.perf_counter() - t0
        if step > 0:
            t_e2e.append(dt)
    t_e2e_max = max_over_ranks(sum(t_e2e))
    e2e_value = n_total * args.steps / t_e2e_max
    hb, db = b.transfer_bytes()
    b_bytes = sum(8 * 20 * (4 * int((z > 1).sum()) + int((z == 1).sum())) ** 2 for z, _ in mols)
    n_atoms_total = int(sum(len(z) for z, _ in mols))
    # inputs of one step: the setup upload measured by the batch; results: energies + gradients
    h2d = hb
    d2h = 8 * args.molecules + 8 * 3 * n_atoms_total + 40 * args.molecules

    # the plain one-molecule-per-launch GPU form on a sample of the same batch
    plain = None
    if rank == 0 and not args.no_plain:
        prate, pcount, pwall = plain_gpu_rate(args.method, mols)
        plain = {"value": prate, "unit": "solves/s",
                 "sample": "%d random molecules of the batch, one Calculator.calculate() each (host buffers, "
                           "energy+gradient), %.1f s wall" % (pcount, pwall),
                 "batched_device_over_plain": value / world / prate, "batched_e2e_over_plain": e2e_value / world / prate}


    def drop_caches():
        # each side leg starts from a device free of the previous legs' idle arenas
        import gc
        import torch
        gc.collect()
        sparrow_b200.lib().sg_release_cached_memory()
        torch.cuda.empty_cache()

    serving = None
    if rank == 0 and not args.no_serving:
        drop_caches()
        serving = serving_leg(loads=tuple(float(v) for v in args.serving_loads.split(",")),
                              seconds=args.serving_seconds, slots=args.serving_slots)

    large = None
    if rank == 0 and not args.no_large:
        drop_caches()
        large = large_leg(sizes=tuple(int(v) for v in args.large_sizes.split(",")))
    tddftb = None
    if rank == 0 and not args.no_tddftb:
        drop_caches()
        tddftb = tddftb_leg()
    open_shell = None
    if rank == 0 and not args.no_open_shell:
        drop_caches()
        open_shell = open_shell_leg()
    hessian = None
    if rank == 0 and not args.no_hessian:
        drop_caches()
        hessian = hessian_leg()
    water32 = None
    if rank == 0 and not args.no_water32:
        drop_caches()
        water32 = water32_leg()
    am1 = None
    if rank == 0 and not args.no_am1:
        drop_caches()
        am1 = am1_leg(mols)

    # roofline of the SCF kernel (average launch)
    scf_ms = stage_sum[2] / args.steps
    flops = scf_flops(mols, it)
    achieved = flops / (scf_ms / 1e3) / 1e12
    traffic = load_traffic()
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if peak else None,
            "traffic": traffic.get("dram_bytes_per_launch") if traffic else None,
            "kernel": "k_scf (persistent SCF: Fock build, DIIS, Jacobi eigensolver, density)",
            "peak_source": "FP64 cuBLAS GEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 entry)",
            "algorithmic_flops_per_launch": flops,
            "stage_ms": {"pair_integrals": stage_sum[0] / args.steps, "one_electron": stage_sum[1] / args.steps,
                         "scf": scf_ms, "gradient": stage_sum[3] / args.steps}}
    line = {
        "metric": "%s SCF solves/s (energy+gradient)" % args.method, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, no dataset)",
        "config": workload_config(args, world),
        "run": {"parallelism": "replicas x%d (molecules sharded, no collective)" % world,
                "batch_matrix_bytes": int(b_bytes), "mean_scf_iterations": float(np.mean(it)),
                "not_converged": not_conv},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": roof,
        "cpu_baseline": cpu,
        "plain_gpu": plain,
        "serving": serving,
        "large_molecules": large,
        "tddftb": tddftb,
        "open_shell": open_shell,
        "hessian": hessian,
        "tuning": tuning,
        "water32_pm6": water32,
        "am1": am1,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and "CUDA_VISIBLE_DEVICES" not in os.environ:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_engine(args, rank, world)


if __name__ == "__main__":
    main()
