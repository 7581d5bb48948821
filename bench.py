"""Benchmark: batched DC operating point of diode-clamped resistor meshes.

Workload (one step): the DC operating point (Simulator::run_dc: direct
Newton attempt, gmin stepping where it fails) of 4096 seeded meshes per GPU,
grid side drawn uniformly from 16..96 (257..9217 unknowns), resistors
lognormal around 1 kOhm (sigma 0.1), level-1 diodes (IS=1e-14, N=1) at 5% of
the nodes, 0-1 mA current sources at 2%, a 1 V corner source; Newton from a
zero guess, all instances in one kernel launch.  Metric: circuit-solves/s
(whole job).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank solves its own 4096 instances (weak
scaling, no collective on the data path); the time is the max over ranks.
--impl reference times the reference's own CPU code (oracle/_ref, built from
the reference sources) on this host's cores: one process pool kept for the
whole run, each step the DC operating point of 64 instances drawn evenly
over the size distribution.

Besides the headline, the line carries (at N = 1):
  setup / e2e_cold  circuit build + host ordering + plans + upload of the
                    batch, and one cold run through the public API;
  plain_dc          the same DC operating points one instance per launch;
  cpu_baseline /    the reference's solve_dc on the host cores, and its
  cpu_newton_only   NeoSolver refactorize + solve x the Newton iterations
                    alone (no per-instance symbolic phase);
  plain_vs_batched  transient of a 32-stage CMOS inverter chain, plain and
                    as Monte Carlo variants, with parity of sampled variants;
  adjoint           transient adjoint of driven 500-node RC trees, with
                    central-difference and .sens parity;
  bsim4_mc          BSIM4v7 Monte Carlo transient of a 200-MOSFET ring +
                    NAND circuit, batched and plain, with sampled parity;
  ac_sweep          batched complex refactor + solve of an AC sweep;
  power_grid        the single-topology AMD-LU refactor/solve case.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import tempfile
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "circuit-solves/s (batched DC operating point, diode-clamped meshes)"
UNIT = "circuit-solves/s"
WORKLOAD = "batched DC OP, 4096 diode-clamped R meshes per GPU, side U{16..96}, FP64"
L2_NOTE = "working set (LU values, several GB) larger than L2; no flush"
REF_PER_STEP = 64


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--count", type=int, default=4096, help="instances per GPU")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-sample", type=int, default=REF_PER_STEP,
                    help="instances in the CPU-baseline sample (0 = skip)")
    ap.add_argument("--plain-sample", type=int, default=24,
                    help="instances of the plain (one per launch) DC measurement (0 = skip)")
    ap.add_argument("--no-inverter", action="store_true",
                    help="skip the plain-vs-batched transient measurement")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the batched transient-adjoint section")
    ap.add_argument("--adjoint-batch", type=int, default=256,
                    help="instances of the transient-adjoint section")
    ap.add_argument("--no-power-grid", action="store_true",
                    help="skip the single large power-grid refactor/solve section")
    ap.add_argument("--grid-side", type=int, default=300,
                    help="side of the power-grid mesh of that section")
    ap.add_argument("--inverter-batch", type=int, default=1184,
                    help="instances of the batched inverter-chain transient")
    ap.add_argument("--bsim4-batch", type=int, default=2048,
                    help="Monte Carlo instances of the BSIM4v7 ring + NAND transient (0 = skip)")
    ap.add_argument("--ac-points", type=int, default=1024,
                    help="frequency points of the batched AC sweep section (0 = skip)")
    ap.add_argument("--row-maps", action="store_true",
                    help="refactor destinations from per-warp row maps instead of the update maps")
    ap.add_argument("--ac-side", type=int, default=64,
                    help="side of the RC mesh of the AC sweep section")
    return ap.parse_args()


# --- workload ------------------------------------------------------------------

def make_meshes(count, seed, rank):
    from neospice_b200 import sharding, workloads
    return workloads.diode_mesh_batch(count, seed=sharding.rank_seed(seed, rank))


def stratified_sample(sides, k, offset=0):
    """k instances spread evenly over the size distribution: the instances
    sorted by grid side, every (count/k)-th of them from `offset` (mod the
    stride).  Returned largest first, the order the host pool runs them in
    (longest jobs first keeps the pool's tail short)."""
    import numpy as np
    count = len(sides)
    k = min(k, count)
    stride = max(1, count // k)
    order = np.argsort(np.asarray(sides), kind="stable")
    pick = [int(order[(offset % stride) + i * stride]) for i in range(k)]
    return sorted(pick, key=lambda i: -int(sides[i]))


def common_config(a):
    """The `config` both arms print (the same workload, word for word)."""
    return {"workload": WORKLOAD, "instances_per_gpu": a.count, "seed": a.seed, "l2": L2_NOTE}


# --- reference CPU path (oracle/_ref), one process per core ----------------------

def _ref_warm(_):
    import oracle
    oracle.ref()
    return os.getpid()


def _ref_worker(mesh):
    import oracle
    t0 = time.perf_counter()
    sol, iters, _ = oracle.ref_mesh_dc(mesh)
    return sol, iters, time.perf_counter() - t0


def _ref_newton_worker(job):
    """The reference NeoSolver on one mesh: numeric() (ordering + first
    factor) on the first Newton matrix, then `iters` x (refactorize + solve)
    -- the linear algebra of the Newton iterations that the GPU kernel
    replaces, without the per-instance symbolic phase.  Returns (numeric
    seconds, loop seconds)."""
    import oracle
    mesh, iters = job
    cp, ri, vals, rhs = oracle.ref_mesh_initjct(mesh)
    s = oracle.RefSolver(len(cp) - 1, cp, ri)
    t0 = time.perf_counter()
    if s.numeric(vals) != 0:
        raise RuntimeError("reference numeric() failed")
    t1 = time.perf_counter()
    for _ in range(iters):
        s.refactorize(vals)
        s.solve(rhs)
    return t1 - t0, time.perf_counter() - t1


def _ref_tran_worker(job):
    import oracle
    desc, tstep, tstop = job
    t0 = time.perf_counter()
    tr, vr, info = oracle.ref_sim(desc, 1, tstep, tstop)
    return tr, vr, info, time.perf_counter() - t0


class RefPool:
    """One pool of host processes (spawn-started: the reference keeps
    per-process globals, so it is not run threaded) kept for a whole
    measurement; the pool's start-up and the loading of the reference
    library happen before any timed region."""

    def __init__(self, processes):
        import multiprocessing as mp
        self.processes = processes
        self.pool = mp.get_context("spawn").Pool(processes)
        self.pool.map(_ref_warm, range(processes), chunksize=1)

    def map(self, fn, jobs):
        """fn over jobs (results in order) and the wall seconds taken."""
        t0 = time.perf_counter()
        res = list(self.pool.imap(fn, jobs, chunksize=1))
        return res, time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# --- clocks -------------------------------------------------------------------------

class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        # the raw samples: NSG_CLOCKS_DIR if set, else the system's temp dir
        out = os.environ.get("NSG_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = pathlib.Path(out) / f"clocks_rank{index}.csv"

    def start(self):
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes per launch of the Newton kernel from the committed ncu
    summary, scaled to this workload (see profiles/)."""
    p = ROOT / "profiles" / "newton_dc_kernel_traffic.json"
    if not p.exists():
        return None
    return json.loads(p.read_text())


# --- our arm ---------------------------------------------------------------------

def run_ours(a, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from neospice_b200.circuit import DcBatch

    meshes = make_meshes(a.count, a.seed, rank)

    # Cold: circuit build, host ordering (once per sparsity pattern), plans and
    # upload, then one run through the public API with host buffers.
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    circuits = [m.build() for m in meshes]
    t1 = time.perf_counter()
    batch = DcBatch(circuits, symbolic=DcBatch.PER_PATTERN)
    if a.row_maps:
        batch.set_row_maps(True)
    t2 = time.perf_counter()
    params_h = torch.from_numpy(batch.params()).pin_memory()
    nsol = int(batch.solution_offsets[-1])
    sol_h = torch.empty(nsol, dtype=torch.float64).pin_memory()
    d_params = torch.empty(params_h.numel(), dtype=torch.float64, device="cuda")
    d_sol = torch.empty(nsol, dtype=torch.float64, device="cuda")
    d_status = torch.empty(batch.count, dtype=torch.int32, device="cuda")
    d_iters = torch.empty(batch.count, dtype=torch.int32, device="cuda")
    t3 = time.perf_counter()
    d_params.copy_(params_h, non_blocking=True)
    batch.run(d_params, d_sol, d_status, d_iters)
    sol_h.copy_(d_sol, non_blocking=True)
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    reorders_cold = batch.reorders()
    st = batch.instance_stats()

    for _ in range(a.warmup):
        batch.run(d_params, d_sol, d_status, d_iters)
    torch.cuda.synchronize()
    reorders_warm = batch.reorders()

    def barrier():
        if world > 1:
            dist.barrier()

    # Device-timed region: inputs resident in HBM; the instances' working set
    # (several GB of LU values) is far larger than L2.
    clocks = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        batch.run(d_params, d_sol, d_status, d_iters)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    sec = e0.elapsed_time(e1) / 1000.0
    reorders_timed = batch.reorders() - reorders_warm

    status = d_status.cpu().numpy()
    iters = d_iters.cpu().numpy()

    # End to end through the public API: pinned host parameters in, host
    # solutions out, every step.
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(a.steps):
        d_params.copy_(params_h, non_blocking=True)
        batch.run(d_params, d_sol, d_status, d_iters)
        sol_h.copy_(d_sol, non_blocking=True)
    f1.record()
    torch.cuda.synchronize()
    barrier()
    sec_e2e = f0.elapsed_time(f1) / 1000.0

    from neospice_b200 import sharding
    sec, sec_e2e, cold = sharding.max_over_ranks([sec, sec_e2e, t4 - t0])

    if rank == 0:
        solves = world * a.count * a.steps
        value = solves / sec
        e2e = solves / sec_e2e
        # Algorithmic bytes / flops of one launch (one DC of every instance):
        # per Newton iteration, refactor + solve + assembly compulsory bytes.
        it = iters.astype(np.float64)
        n, nnz, nlu, upd = (st[k].astype(np.float64) for k in ("n", "nnz", "nnz_lu", "updates"))
        per_iter = (8 * nnz + 8 * nlu + 4 * (nlu + n) + 8 * n) + (12 * nlu + 16 * n) + (8 * nnz + 8 * n)
        bytes_launch = float((it * per_iter).sum())
        flops_launch = float((it * (2 * upd + n)).sum())
        launch_s = sec / a.steps
        peak, peak_kind = measured_peaks()
        achieved = bytes_launch / launch_s / 1e9
        traffic = ncu_traffic()
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(1e3 * sec / a.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded meshes)",
            "config": common_config(a),
            "workload_stats": {
                "unknowns_total": int(n.sum()), "lu_entries_total": int(nlu.sum()),
                "refactor_updates_total": int(upd.sum()),
                "newton_iterations_mean": float(it.mean()),
                "converged": int((status == 0).sum()),
                "symbolic": "host Markowitz ordering once per sparsity pattern, "
                            "GPU pivot re-validation per instance",
                "parallelism": f"dp{world} (independent instances)",
                "reorders": {"cold_run": reorders_cold, "warmup": reorders_warm - reorders_cold,
                             "timed": reorders_timed}},
            "e2e": {"value": round(e2e, 3), "unit": UNIT,
                    "h2d_bytes_per_step": int(params_h.numel() * 8),
                    "d2h_bytes_per_step": int(nsol * 8)},
            "setup": {"circuit_build_s": round(t1 - t0, 3), "batch_create_s": round(t2 - t1, 3),
                      "setup_s": round(t2 - t0, 3), "cold_run_s": round(t4 - t3, 3),
                      "what": "batch_create = host ordering once per sparsity pattern, "
                              "plans, upload"},
            "e2e_cold": {"value": round(world * a.count / cold, 3), "unit": UNIT,
                         "seconds": round(cold, 3),
                         "what": "one fresh batch: circuit build + setup + H2D + first run "
                                 "(incl. its host re-orders) + D2H"},
            "gpu_launches": a.steps,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 5),
                         "traffic": (traffic or {}).get("bytes_per_launch"),
                         "kernel": "newton_dc_kernel",
                         "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)"
                                         if peak_kind == "measured" else
                                         "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"),
                         "algorithmic_bytes_per_launch": bytes_launch,
                         "fp64_gflops": round(flops_launch / launch_s / 1e9, 2)},
            "clocks": clk,
        }
        if a.plain_sample > 0 and world == 1:
            try:
                line["plain_dc"] = plain_dc(meshes, a.plain_sample, value)
            except Exception as exc:
                line["plain_dc"] = {"error": str(exc)}
        pool = None
        if a.cpu_sample > 0:
            import oracle
            if oracle.have_ref():
                pool = RefPool(os.cpu_count() or 1)
                line.update(cpu_legs(pool, meshes, batch, d_sol, iters, a.cpu_sample))
        if not a.no_inverter and world == 1:
            try:
                line["plain_vs_batched"] = inverter_plain_vs_batched(a.inverter_batch, pool)
            except Exception as exc:
                line["plain_vs_batched"] = {"error": str(exc)}
        if a.bsim4_batch > 0 and world == 1:
            try:
                line["bsim4_mc"] = bsim4_mc_transient(a.bsim4_batch, pool)
            except Exception as exc:
                line["bsim4_mc"] = {"error": str(exc)}
        if pool is not None:
            pool.close()
        if not a.no_adjoint and world == 1:
            try:
                line["adjoint"] = adjoint_rc_tree(a.adjoint_batch)
            except Exception as exc:
                line["adjoint"] = {"error": str(exc)}
            try:
                line["adjoint"]["parity"] = adjoint_parity()
            except Exception as exc:
                line["adjoint"]["parity"] = {"error": str(exc)}
        if a.ac_points > 0 and world == 1:
            try:
                line["ac_sweep"] = ac_sweep(a.ac_side, a.ac_points)
            except Exception as exc:
                line["ac_sweep"] = {"error": str(exc)}
        if not a.no_power_grid and world == 1:
            try:
                line["power_grid"] = power_grid_refactor(a.grid_side, a.steps, a.warmup)
            except Exception as exc:
                line["power_grid"] = {"error": str(exc)}
        print(json.dumps(line), flush=True)

    del batch
    if world > 1:
        dist.destroy_process_group()


def cpu_legs(pool, meshes, batch, d_sol, iters, k):
    """The reference on a stratified sample of k instances, over all host
    cores: its solve_dc (cpu_baseline, and parity of our solutions), and its
    NeoSolver refactorize + solve repeated for each instance's Newton
    iterations (cpu_newton_only)."""
    import numpy as np
    sides = [m.side for m in meshes]
    idx = stratified_sample(sides, k, 0)
    res, wall = pool.map(_ref_worker, [meshes[i] for i in idx])
    gpu = batch.split(d_sol)
    worst = 0.0
    for (sol, _, _), i in zip(res, idx):
        err = np.abs(gpu[i] - sol) / np.maximum(np.abs(sol), 1e-3)
        worst = max(worst, float(err.max()))
    nres, nwall = pool.map(_ref_newton_worker, [(meshes[i], int(iters[i])) for i in idx])
    sample = (f"{len(idx)} of the {len(meshes)} instances, evenly spread over the sorted grid "
              f"sides, largest first; one process per core; {cpu_model()}")
    return {
        "cpu_baseline": {"value": round(len(idx) / wall, 4), "unit": UNIT,
                         "cores": pool.processes, "kind": "reference",
                         "sample": "reference solve_dc, " + sample},
        "cpu_newton_only": {
            "value": round(len(idx) / nwall, 4), "unit": UNIT, "cores": pool.processes,
            "what": "reference NeoSolver refactorize + solve x each instance's Newton "
                    "iterations (the GPU's iteration counts, equal to the reference's), "
                    "after one untimed numeric(); no device loads, no symbolic phase",
            "numeric_core_s": round(sum(r[0] for r in nres), 3),
            "loop_core_s": round(sum(r[1] for r in nres), 3),
            "solve_dc_core_s": round(sum(r[2] for r in res), 3)},
        "parity": {"checked": len(idx), "max_rel_err_vs_reference": worst,
                   "iterations_equal": bool(all(int(iters[i]) == r[1]
                                                for r, i in zip(res, idx)))},
    }


def plain_dc(meshes, k, batched_value):
    """The plain path of the same DC operating points: one instance per
    launch (a one-circuit DcBatch each), a stratified sample of k instances,
    each timed with CUDA events after one warm-up run."""
    import torch
    from neospice_b200.circuit import DcBatch
    idx = stratified_sample([m.side for m in meshes], k, 1)
    total = 0.0
    for i in idx:
        b = DcBatch([meshes[i].build()], symbolic=DcBatch.PER_PATTERN)
        b.run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.run()
        e1.record()
        torch.cuda.synchronize()
        total += e0.elapsed_time(e1) / 1e3
        del b
    value = len(idx) / total
    return {"value": round(value, 3), "unit": UNIT, "instances": len(idx),
            "seconds": round(total, 4), "batched_over_plain": round(batched_value / value, 2),
            "what": "one instance per launch, stratified sample of the same meshes"}


# --- plain vs batched transient (32-stage CMOS inverter chain) ---------------------

INV_PULSE = (0.0, 1.8, 0.0, 1e-10, 1e-10, 1e-9, 2e-9)

# FP64 operations per Newton iteration of one instance of the BSIM4v7 ring +
# NAND circuit (DADD + DMUL + 2 DFMA thread instructions of the transient
# kernel counted by ncu over every launch of 592 instances, .tran 1p 0.2n,
# divided by their 275,593 Newton iterations), and B200's nominal FP64 rate.
B4_FLOPS_PER_ITER = 6.41e5
FP64_NOMINAL_FLOPS = 37e12


def _tran_parity(ours, ref):
    """Timepoints, voltages and Newton iterations of one of our transients
    against the reference's."""
    import numpy as np
    tr, vr, info = ref
    same_pts = len(tr) == len(ours["time"])
    err = float(np.max(np.abs(ours["values"] - vr) / np.maximum(np.abs(vr), 1e-3))) \
        if same_pts else None
    return {"timepoints_equal": bool(same_pts and np.allclose(tr, ours["time"], rtol=1e-12, atol=0)),
            "max_rel_err_vs_reference": err,
            "iterations_equal": info["iterations"] == ours["newton_iters"],
            "iterations_rel_diff": abs(info["iterations"] - ours["newton_iters"]) /
                                   max(1, info["iterations"])}


def inverter_plain_vs_batched(batch_count, pool=None, parity_variants=8):
    """Transient of a 32-stage level-1 CMOS inverter chain (10 fF per stage,
    VDD 1.8 V, PULSE 0->1.8 V 100p/100p 1n/2n, .tran 1p 20n): the plain path
    (one instance per launch) and the batched path (batch_count Monte Carlo
    variants in one launch), each timed through TranBatch.run (device
    clock), with parity against the reference's solve_transient for the
    nominal instance and `parity_variants` evenly spaced variants."""
    import numpy as np
    import torch
    from neospice_b200 import workloads as W
    from neospice_b200.circuit import TranBatch

    nominal = W.inverter_chain(32, pulse=INV_PULSE)
    probes = np.arange(nominal.num_nodes, dtype=np.int32)

    def timed(nls, reps):
        b = TranBatch([n.build() for n in nls], 1e-12, 20e-9, probes, max_points=21000)
        b.run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            b.run()
        e1.record()
        torch.cuda.synchronize()
        return b, e0.elapsed_time(e1) / 1000.0 / reps

    bp, t_plain = timed([nominal], 2)
    rp = bp.results()[0]
    mc = [W.inverter_chain_mc(np.random.default_rng([7, i])) for i in range(batch_count)]
    bb, t_batch = timed(mc, 1)
    rb = bb.results()
    ok = sum(r["status"] == 0 for r in rb)
    out = {
        "workload": "transient, 32-stage CMOS inverter chain (MOS1), PULSE input, .tran 1p 20n; "
                    f"batched = {batch_count} Monte Carlo variants (VTO sigma 30 mV, KP 5%)",
        "plain": {"value": round(1.0 / t_plain, 4), "unit": "circuit-solves/s",
                  "seconds_per_solve": round(t_plain, 4), "points": len(rp["time"]),
                  "newton_iterations": rp["newton_iters"]},
        "batched": {"value": round(batch_count / t_batch, 3), "unit": "circuit-solves/s",
                    "instances": batch_count, "seconds": round(t_batch, 4), "ok": ok},
        "ratio": round((batch_count / t_batch) * t_plain, 2),
    }
    try:
        import oracle
        sys.path.insert(0, str(ROOT / "tests"))
        import netlists
        if oracle.have_ref():
            t0 = time.perf_counter()
            ref_nom = oracle.ref_sim(netlists.ref_desc(nominal), 1, 1e-12, 20e-9)
            t_ref = time.perf_counter() - t0
            out["parity"] = _tran_parity(rp, ref_nom)
            out["cpu_reference_1core"] = {"value": round(1.0 / t_ref, 4), "unit": "circuit-solves/s"}
            if pool is not None and parity_variants > 0:
                pick = sorted({int(round(x)) for x in
                               np.linspace(0, batch_count - 1, parity_variants)})
                res, wall = pool.map(_ref_tran_worker,
                                     [(netlists.ref_desc(mc[i]), 1e-12, 20e-9) for i in pick])
                checks = [_tran_parity(rb[i], (r[0], r[1], r[2])) for i, r in zip(pick, res)]
                errs = [c["max_rel_err_vs_reference"] for c in checks]
                out["batched"]["parity"] = {
                    "variants_checked": pick,
                    "timepoints_equal": all(c["timepoints_equal"] for c in checks),
                    "max_rel_err_vs_reference": None if None in errs else max(errs),
                    "iterations_equal": all(c["iterations_equal"] for c in checks),
                    "tolerance": "1e-9 relative voltages (1e-3 V floor), identical timepoints "
                                 "and iteration counts"}
                out["cpu_reference_pool"] = {
                    "value": round(len(pick) / wall, 4), "unit": "circuit-solves/s",
                    "cores": pool.processes, "sample": f"{len(pick)} Monte Carlo variants"}
    except Exception as exc:  # reported, not raised: the GPU numbers stand alone
        out["parity"] = {"error": str(exc)}
    return out


# --- BSIM4v7 Monte Carlo transient (ring oscillator + NAND chain) -------------------

B4_PROBES = [0, 1, 2, 7, 13, 26, 27, 99, 100]


def bsim4_mc_transient(count, pool=None, parity_instances=4, tstep=1e-12, tstop=5e-9):
    """Batched Monte Carlo transient of the 200-MOSFET BSIM4v7 circuit
    (workloads.bsim4_ring_nand: 25-stage ring oscillator + 25 NAND2 gates
    each followed by an inverter, default LEVEL=14 cards, L 90n, W_n 200n,
    W_p 400n, per-device DELVTO sigma 30 mV and TOXE +-3 %, VDD ramped to
    1.2 V in 50 ps), .tran 1p 5n, `count` instances in one launch with
    per-instance timestep control; the plain path (one instance per launch);
    parity of evenly spaced instances against the reference's
    solve_transient (timepoints, probe voltages, Newton iterations)."""
    import numpy as np
    import torch
    from neospice_b200 import workloads as W
    from neospice_b200.circuit import TranBatch

    probes = np.array(B4_PROBES, np.int32)
    nls = [W.bsim4_ring_nand(np.random.default_rng([33, i])) for i in range(count)]
    t0 = time.perf_counter()
    circuits = [nl.build() for nl in nls]
    b = TranBatch(circuits, tstep, tstop, probes, max_points=6000)
    t_setup = time.perf_counter() - t0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    ev[0].record()
    b.run()
    ev[1].record()
    torch.cuda.synchronize()
    t_batch = ev[0].elapsed_time(ev[1]) / 1e3
    res = b.results()
    ok = sum(r["status"] == 0 for r in res)
    bp = TranBatch([nls[0].build()], tstep, tstop, probes, max_points=6000)
    bp.run()
    torch.cuda.synchronize()
    ev[2].record()
    bp.run()
    ev[3].record()
    torch.cuda.synchronize()
    t_plain = ev[2].elapsed_time(ev[3]) / 1e3
    iters = np.array([r["newton_iters"] for r in res], np.float64)
    out = {
        "workload": f"BSIM4v7 Monte Carlo transient, {count} instances of a 200-MOSFET circuit "
                    "(25-stage ring oscillator + 25 NAND2 + 25 INV, default LEVEL=14 cards, "
                    "DELVTO sigma 30 mV, TOXE +-3 %, n = 102), .tran 1p 5n, FP64",
        "batched": {"value": round(count / t_batch, 3), "unit": "circuit-solves/s",
                    "instances": count, "seconds": round(t_batch, 4), "ok": int(ok),
                    "setup_s": round(t_setup, 3),
                    "points_mean": float(np.mean([len(r["time"]) for r in res])),
                    "newton_iters_mean": float(iters.mean()),
                    "device_loads_per_s": round(200.0 * float(iters.sum()) / t_batch, 1),
                    "fp64_gflops": round(B4_FLOPS_PER_ITER * float(iters.sum()) / t_batch / 1e9, 1),
                    "fp64_frac_of_nominal": round(B4_FLOPS_PER_ITER * float(iters.sum()) / t_batch
                                                  / FP64_NOMINAL_FLOPS, 4),
                    "fp64_note": "FP64 operations per Newton iteration of this circuit (DADD + "
                                 "DMUL + 2 DFMA thread instructions counted by ncu on 592 "
                                 "instances, .tran 1p 0.2n: 6.41e5) x iterations / time; peak = "
                                 "nominal 37 TFLOP/s (no measured FP64 peak)"},
        "plain": {"value": round(1.0 / t_plain, 4), "unit": "circuit-solves/s",
                  "seconds_per_solve": round(t_plain, 4)},
        "batched_over_plain": round((count / t_batch) * t_plain, 2),
    }
    try:
        import oracle
        sys.path.insert(0, str(ROOT / "tests"))
        import netlists
        if oracle.have_ref() and pool is not None and parity_instances > 0:
            pick = sorted({int(round(x)) for x in np.linspace(0, count - 1, parity_instances)})
            ref, wall = pool.map(_ref_tran_worker,
                                 [(netlists.ref_desc(nls[i]), tstep, tstop) for i in pick])
            checks = [_tran_parity({"time": res[i]["time"], "values": res[i]["values"],
                                    "newton_iters": res[i]["newton_iters"]},
                                   (r[0], r[1][:, B4_PROBES], r[2])) for i, r in zip(pick, ref)]
            errs = [c["max_rel_err_vs_reference"] for c in checks]
            worst = None if None in errs else max(errs)
            out["parity"] = {"instances_checked": pick,
                             "timepoints_equal": all(c["timepoints_equal"] for c in checks),
                             "max_rel_err_vs_reference": worst,
                             "iterations_equal": all(c["iterations_equal"] for c in checks),
                             "iterations_max_rel_diff": max(c["iterations_rel_diff"] for c in checks),
                             "within_tolerance": bool(worst is not None and worst <= 1e-3 and
                                                      all(c["timepoints_equal"] for c in checks)),
                             "tolerance": "Newton tolerances: 1e-3 relative voltages (1e-3 V "
                                          "floor), identical timepoints; the GPU's exp/log/pow "
                                          "round differently from the host C library in a few "
                                          "percent of BSIM4 load outputs, so 1e-9 is not "
                                          "attainable for BSIM4 transients"}
            per = [r[3] for r in ref]
            out["cpu_reference"] = {
                "value": round(pool.processes / float(np.mean(per)), 4), "unit": "circuit-solves/s",
                "cores": pool.processes, "seconds_per_solve_1core": round(float(np.mean(per)), 3),
                "sample": f"{len(pick)} of the Monte Carlo instances, reference solve_transient; "
                          "value = cores / mean seconds per solve"}
    except Exception as exc:
        out["parity"] = {"error": str(exc)}
    return out


# --- batched transient adjoint (RC trees driven by CMOS inverters) -------------------

ADJ_TIGHT = dict(reltol=1e-9, vntol=1e-12, abstol=1e-15, max_iter=200)


def _adjoint_targets(results, max_points, seed=91):
    """Seeded synthetic targets: an exponential fall with a per-instance
    time constant, sampled at each instance's own timepoints."""
    import numpy as np
    rng = np.random.default_rng(seed)
    tg = np.zeros(len(results) * max_points)
    for i, r in enumerate(results):
        tau = 2e-10 * np.exp(0.2 * rng.standard_normal())
        tg[i * max_points:i * max_points + len(r["time"])] = 1.8 * np.exp(-r["time"] / tau)
    return tg


def adjoint_rc_tree(count, nodes=500, every=32):
    """Gradients of sum_n (v_far(t_n) - target(t_n))^2 over .tran 1p 2n of
    `count` seeded 500-node RC trees (R lognormal around 50 Ohm, C around
    2 fF, sigma 0.2) each driven by a level-1 CMOS inverter, with respect to
    every R and C and the drivers' W, L and VTO: the recorded forward run,
    then the discrete adjoint with a checkpoint every `every` steps.  Both
    timed with CUDA events; grads/s counts full gradient vectors."""
    import numpy as np
    import torch
    from neospice_b200 import workloads as W
    from neospice_b200.circuit import TranBatch

    nls = [W.rc_tree_driven(np.random.default_rng([90, i]), nodes) for i in range(count)]
    far = nodes - 1
    max_points = 4096
    b = TranBatch([nl.build() for nl in nls], 1e-12, 2e-9, np.full(1, far, np.int32),
                  max_points=max_points)
    b.record(True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    ev[0].record()
    b.run()
    ev[1].record()
    torch.cuda.synchronize()
    res = b.results()
    d_tg = torch.from_numpy(_adjoint_targets(res, max_points)).cuda()
    ev[1].record()
    g, loss, st = b.adjoint(np.full(count, far), d_tg, 1.0, every)
    ev[2].record()
    torch.cuda.synchronize()
    t_fwd = ev[0].elapsed_time(ev[1]) / 1e3
    t_adj = ev[1].elapsed_time(ev[2]) / 1e3
    ok = int((st.cpu().numpy() == 0).sum())
    n_params = sum(1 for d in nls[0].devices if d[0] in ("R", "C")) + 6
    steps = [len(r["time"]) - 1 for r in res]
    return {
        "workload": f"transient adjoint, {count} x {nodes}-node RC tree driven by a MOS1 inverter, "
                    f".tran 1p 2n, loss = sum (v_far - target)^2, grads w.r.t. every R, C and the "
                    f"drivers' W/L/VTO ({n_params} per instance), checkpoint every {every} steps",
        "grads_per_s": round(count / (t_fwd + t_adj), 3), "unit": "gradients/s",
        "forward_s": round(t_fwd, 4), "adjoint_s": round(t_adj, 4), "ok": ok,
        "steps_mean": float(np.mean(steps)),
        "newton_iters_mean": float(np.mean([r["newton_iters"] for r in res])),
        "loss_mean": float(loss.mean()),
    }


def adjoint_parity(nodes=500, instances=2, per_instance=24, every=32, h_rels=(1e-6, 1e-4)):
    """Parity of the adjoint section at its own size: instances 0 and 1 of
    the benchmarked batch (same seeds, same targets), a seeded sample of
    `per_instance` parameters each (the drivers' W, L, VTO and R / C of the
    tree), gradient against central differences of the same discrete
    transient (Newton to reltol 1e-9 in the re-solves), all in one batch:
    per instance one unperturbed copy and a +h and a -h copy per parameter
    and step.  Tolerance 1e-6 relative plus the loss's rounding floor
    5e-12 L / 2h.  At h = 1e-6 relative that floor is a few 1e-6 of the
    gradient (the loss is a sum of 2,000 squared errors), so the quotient
    cannot resolve 1e-6; at h = 1e-4 the floor drops 100-fold and the
    truncation error stays near h^2, and a quotient counts as resolved when
    its floor is below a tenth of the 1e-6 tolerance.  Also instance 0's DC
    gradient of v_far against the reference's .sens (resistors and sources,
    one-sided FD with a 1e-4 step: 5e-3 relative)."""
    import numpy as np
    import torch
    from neospice_b200 import workloads as W
    from neospice_b200.circuit import DcBatch, TranBatch

    far = nodes - 1
    max_points = 4096
    base = [W.rc_tree_driven(np.random.default_rng([90, i]), nodes) for i in range(instances)]
    sel = []
    for i, nl in enumerate(base):
        nl.build()
        pidx = nl.param_index
        kinds = [d[0] for d in nl.devices]
        mos = [pidx[k] + o for k, kd in enumerate(kinds) if kd == "M" for o in (0, 1, 2)]
        rs = [pidx[k] for k, kd in enumerate(kinds) if kd == "R"]
        cs = [pidx[k] for k, kd in enumerate(kinds) if kd == "C"]
        rng = np.random.default_rng([92, i])
        rest = per_instance - len(mos)
        pick = list(rng.choice(rs, rest // 2, replace=False)) + \
            list(rng.choice(cs, rest - rest // 2, replace=False))
        sel.append(mos + [int(x) for x in pick])
    copies = []     # (instance, parameter index or None, sign, step index)
    for i in range(instances):
        copies.append((i, None, 0, -1))
        for p in sel[i]:
            for hk in range(len(h_rels)):
                copies += [(i, p, +1, hk), (i, p, -1, hk)]
    b = TranBatch([base[c[0]].build() for c in copies], 1e-12, 2e-9, np.full(1, far, np.int32),
                  max_points=max_points)
    b.record(True)
    b.run()
    torch.cuda.synchronize()
    res = b.results()
    first = {c[0]: k for k, c in enumerate(copies) if c[1] is None}
    same = all(len(res[k]["time"]) == len(res[first[c[0]]]["time"]) for k, c in enumerate(copies))
    # the benchmark's targets for instances 0..instances-1, then per copy
    tg_inst = _adjoint_targets([res[first[i]] for i in range(instances)], max_points)
    tg = np.concatenate([tg_inst[c[0] * max_points:(c[0] + 1) * max_points] for c in copies])
    off, pdc, ptr = b.params()
    hs = {}
    for k, (i, p, sgn, hk) in enumerate(copies):
        if p is None:
            continue
        h = abs(pdc[off[k] + p]) * h_rels[hk]
        hs[(i, p, hk)] = h
        pdc[off[k] + p] += sgn * h
        ptr[off[k] + p] += sgn * h
    b.set_adjoint_options(**ADJ_TIGHT)
    dev = lambda x: torch.from_numpy(x).cuda()
    g, loss, st = b.adjoint(np.full(len(copies), far), dev(tg), 1.0, every, dev(pdc), dev(ptr))
    torch.cuda.synchronize()
    g, loss, st = g.cpu().numpy(), loss.cpu().numpy(), st.cpu().numpy()
    steps = []
    for hk, h_rel in enumerate(h_rels):
        worst, worst_all, within, resolved = 0.0, 0.0, 0, 0
        for i in range(instances):
            k0 = first[i]
            for p in sel[i]:
                kp = copies.index((i, p, +1, hk))
                km = copies.index((i, p, -1, hk))
                h = hs[(i, p, hk)]
                fd = (loss[kp] - loss[km]) / (2 * h)
                ga = g[off[k0] + p]
                floor = 5e-12 * loss[k0] / (2 * h)
                within += int(abs(ga - fd) <= 1e-6 * abs(fd) + floor)
                worst_all = max(worst_all, abs(ga - fd) / abs(fd))
                if floor < 1e-7 * abs(fd):
                    resolved += 1
                    worst = max(worst, abs(ga - fd) / abs(fd))
        steps.append({"h_rel": h_rel, "within_tolerance": within, "resolved": resolved,
                      "max_rel_err_resolved": worst, "max_rel_err": worst_all})
    out = {"instances": instances, "parameters_checked": instances * per_instance,
           "status_ok": bool((st == 0).all()), "schedules_equal": bool(same),
           "within_tolerance": min(x["within_tolerance"] for x in steps),
           "steps": steps,
           "tolerance": "1e-6 relative + 5e-12 L / 2h (central FD); resolved: floor below "
                        "1e-7 |fd|"}
    # DC gradient of v_far against the reference's .sens
    try:
        import oracle
        sys.path.insert(0, str(ROOT / "tests"))
        import netlists
        if oracle.have_ref():
            nl = base[0]
            db = DcBatch([nl.build()], symbolic=DcBatch.PER_INSTANCE)
            sols, dst, _ = db.run()
            cot = torch.zeros_like(sols)
            cot[far] = 1.0
            gd, gst = db.adjoint(sols, cot)
            torch.cuda.synchronize()
            gd = gd.cpu().numpy()
            pidx = nl.param_index
            kinds = [d[0] for d in nl.devices]
            order = ([pidx[k] for k, kd in enumerate(kinds) if kd == "R"] +
                     [pidx[k] for k, kd in enumerate(kinds) if kd in ("V", "VPULSE")] +
                     [pidx[k] for k, kd in enumerate(kinds) if kd in ("I", "IPULSE")])
            sref, _ = oracle.ref_sim_sens(netlists.ref_desc(nl), far)
            ours = gd[np.array(order, np.int64)]
            scale = float(np.max(np.abs(sref)))
            dev_err = np.abs(ours - sref) - (5e-3 * np.abs(sref) + 1e-6 * scale)
            out["dc_sens"] = {"entries": len(sref), "status_ok": int(dst.sum()) == 0 and
                              int(gst.sum()) == 0, "all_within": bool((dev_err <= 0).all()),
                              "max_abs_diff": float(np.max(np.abs(ours - sref))),
                              "max_abs_sens": scale,
                              "tolerance": "5e-3 relative + 1e-6 x max |sens|"}
    except Exception as exc:
        out["dc_sens"] = {"error": str(exc)}
    return out


# --- batched AC sweep (complex refactor + solve) -----------------------------------

def ac_sweep(side, points, ref_sample=16):
    """AC sweep of a side x side RC mesh (workloads.rc_mesh, n = side^2 + 1
    + 1): the pivots of the first frequency point ordered on the host
    (NeoSolver::numeric_complex), then all `points` log-spaced frequency
    points (1 kHz .. 100 GHz) refactored (factor_complex) and solved
    (solve_complex) in one batch on the GPU, timed with CUDA events; the
    reference's NeoSolver refactorize_complex + solve_complex per point on
    one host core over `ref_sample` points, with bitwise parity of those
    points' solutions."""
    import numpy as np
    import torch
    from neospice_b200 import workloads as W
    from neospice_b200.solver import Batch, Topology, _interleave

    nl = W.rc_mesh(np.random.default_rng(2027), side)
    n, cp, ri, g, c, b = W.ac_system(nl)
    freqs = np.logspace(3, 11, points)
    omegas = 2 * np.pi * freqs
    ax = np.empty((points, 2 * len(ri)))
    ax[:, 0::2] = g[None, :]
    ax[:, 1::2] = omegas[:, None] * c[None, :]
    t0 = time.perf_counter()
    topo = Topology.order_complex(n, cp, ri, ax[0])
    t_sym = time.perf_counter() - t0
    info = topo.info()
    batch = Batch([topo] * points)
    d_ax = torch.from_numpy(ax.ravel()).cuda()
    bz = _interleave(b)
    d_b = torch.from_numpy(np.tile(bz, points)).cuda()
    d_x = torch.empty_like(d_b)
    d_lu, st = batch.refactor_complex(d_ax)
    d_x.copy_(d_b)
    batch.solve_complex(d_lu, d_x)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    reps = 3
    ev[0].record()
    for _ in range(reps):
        batch.refactor_complex(d_ax, d_lu, st)
    ev[1].record()
    for _ in range(reps):
        d_x.copy_(d_b)
        batch.solve_complex(d_lu, d_x)
    ev[2].record()
    torch.cuda.synchronize()
    t_ref = ev[0].elapsed_time(ev[1]) / 1e3 / reps
    t_sol = ev[1].elapsed_time(ev[2]) / 1e3 / reps
    ok = int((st.cpu().numpy() == 0).sum())
    x = d_x.cpu().numpy()
    nnz, nlu, upd = len(ri), info["nnz_lu"], info["updates"]
    # compulsory bytes per point: complex A in, complex LU out, index stream,
    # then the sweeps (complex LU and vectors)
    b_ref = 16 * nnz + 16 * nlu + 4 * (nlu + n) + 16 * n
    b_sol = 24 * nlu + 32 * n
    peak, peak_kind = measured_peaks()
    out = {
        "workload": f"AC sweep of a {side}x{side} RC mesh (n={n}), {points} log-spaced frequency "
                    "points 1 kHz..100 GHz, complex FP64: one host ordering, then every point "
                    "refactored (fixed pivots) and solved in one batch",
        "value": round(points / (t_ref + t_sol), 2), "unit": "frequency points/s",
        "refactor_ms": round(1e3 * t_ref, 3), "solve_ms": round(1e3 * t_sol, 3), "ok": ok,
        "host_symbolic_s": round(t_sym, 4), "nnz": nnz, "nnz_lu": nlu,
        "complex_updates_per_point": upd,
        "refactor_gbs": round(points * b_ref / t_ref / 1e9, 2),
        "refactor_frac_hbm": round(points * b_ref / t_ref / 1e9 / peak, 5),
        "refactor_fp64_gflops": round(points * 8.0 * upd / t_ref / 1e9, 2),
        "solve_gbs": round(points * b_sol / t_sol / 1e9, 2), "peak_gbs": peak,
        "peak_source": peak_kind,
    }
    try:
        import oracle
        if oracle.have_ref():
            rs = oracle.RefSolver(n, cp, ri)
            rs.numeric_complex(ax[0])
            pick = sorted({int(round(v)) for v in np.linspace(1, points - 1, ref_sample)})
            worst_equal = True
            t0 = time.perf_counter()
            sols = []
            for k in pick:
                rs.refactorize_complex(ax[k])
                sols.append(rs.solve_complex(b))
            t_cpu = (time.perf_counter() - t0) / len(pick)
            for k, xr in zip(pick, sols):
                v = 2 * int(batch.vector_offsets[k])
                xk = x[v:v + 2 * n]
                worst_equal &= bool(np.array_equal(xk[0::2], xr.real) and
                                    np.array_equal(xk[1::2], xr.imag))
            out["cpu_reference_1core"] = {"value": round(1.0 / t_cpu, 2), "unit": "frequency points/s",
                                          "sample": f"{len(pick)} points, refactorize_complex + "
                                                    "solve_complex"}
            out["parity"] = {"points_checked": len(pick), "bitwise_equal": worst_equal}
    except Exception as exc:
        out["parity"] = {"error": str(exc)}
    return out


# --- one large topology: power-grid refactor and solve ------------------------------

def power_grid_refactor(side, reps, warmup):
    """The large-single-topology case at a reduced size: a side x side RC
    power grid (0.1 Ohm lognormal sigma 0.05 mesh, 1 pF per node, VDD pads
    on a pitch-50 lattice, side^2/100 PWL loads), linear, so the AMD-LU
    engine (as the reference's make_solver picks it).  Times the grid-wide
    fixed-pivot replay refactor and the forward/backward sweeps of the
    transient matrix (conductances + C/h with h = 10 ps) with CUDA events,
    against the reference's AmdLuSolver refactorize + solve on one core."""
    import numpy as np
    import torch
    from neospice_b200 import workloads as W
    from neospice_b200.solver import Batch, Topology

    nl = W.power_grid(np.random.default_rng(2026), side, 50, max(1, side * side // 100))
    c = nl.build()
    cp, ri = c.pattern()
    g, _ = c.initial_matrix(0.0)
    n = len(cp) - 1
    # transient companion matrix: each 1 pF cap adds C/h to its node's diagonal
    tran = g.copy()
    caps = {d[1] for d in nl.devices if d[0] == "C"}
    for j in caps:
        for p in range(cp[j], cp[j + 1]):
            if ri[p] == j:
                tran[p] += 1e-12 / 1e-11
    t0 = time.perf_counter()
    topo = Topology.order(n, cp, ri, tran, solver="amdlu")
    t_symbolic = time.perf_counter() - t0
    info = topo.info()
    batch = Batch([topo])
    batch.set_schedule(2)
    d_a = torch.from_numpy(tran).cuda()
    rhs = np.random.default_rng(5).standard_normal(n)
    d_b = torch.from_numpy(rhs).cuda()
    d_x = torch.empty_like(d_b)
    for _ in range(max(warmup, 1)):
        st, _ = batch.refactor(d_a)
        d_x.copy_(d_b)
        batch.solve(d_x)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    for _ in range(reps):
        batch.refactor(d_a, d_status=st)
    ev[1].record()
    for _ in range(reps):
        d_x.copy_(d_b)
        batch.solve(d_x)
    ev[2].record()
    torch.cuda.synchronize()
    t_ref = ev[0].elapsed_time(ev[1]) / 1e3 / reps
    t_sol = ev[1].elapsed_time(ev[2]) / 1e3 / reps
    x = d_x.cpu().numpy()
    nnz, nlu, upd = len(ri), info["nnz_lu"], info["updates"]
    # the device update map holds uint16 positions when every LU column is
    # shorter than 65,537 rows, else int32
    map_b = 2 if int(np.bincount(topo.export()[3]).max()) <= 65536 else 4
    b_ref = 8 * nnz + 8 * nlu + map_b * upd + 4 * (nlu + n) + 8 * n
    b_sol = 12 * nlu + 16 * n
    peak, peak_kind = measured_peaks()
    out = {
        "workload": f"power grid {side}x{side} (n={n}), {len([d for d in nl.devices if d[0] == 'V'])} "
                    f"pads, AMD-LU replay refactor + solve of the transient matrix, grid-wide schedule",
        "status": int(st.cpu()[0]), "nnz": nnz, "nnz_lu": nlu, "updates": upd,
        "host_symbolic_s": round(t_symbolic, 3),
        "refactor_ms": round(1e3 * t_ref, 4), "solve_ms": round(1e3 * t_sol, 4),
        "refactor_gbs": round(b_ref / t_ref / 1e9, 2), "solve_gbs": round(b_sol / t_sol / 1e9, 2),
        "refactor_gflops": round((2 * upd + n) / t_ref / 1e9, 2),
        "refactor_frac_hbm": round(b_ref / t_ref / 1e9 / peak, 5),
        "solves_per_s": round(1.0 / (t_ref + t_sol), 2), "peak_gbs": peak,
        "peak_source": peak_kind,
    }
    try:
        import oracle
        if oracle.have_ref():
            ref = oracle.RefAmdLu(n, cp, ri)
            ref.numeric(tran)
            t0 = time.perf_counter()
            ref.refactorize(tran)
            xr = ref.solve(rhs)
            t_cpu = time.perf_counter() - t0
            out["cpu_reference_1core"] = {"refactor_plus_solve_ms": round(1e3 * t_cpu, 3),
                                          "solves_per_s": round(1.0 / t_cpu, 3)}
            out["parity"] = {"bitwise_equal": bool(np.array_equal(x, xr)),
                             "max_rel_err": float(np.max(np.abs(x - xr) /
                                                         np.maximum(np.abs(xr), 1e-30)))}
    except Exception as exc:
        out["parity"] = {"error": str(exc)}
    return out


# --- reference arm -----------------------------------------------------------------

def run_reference(a, rank):
    """The reference's solve_dc on this host's cores: one process pool for
    the whole run (started, and the library loaded in every process, before
    the first step); each step the DC operating points of REF_PER_STEP
    instances spread evenly over the size distribution (a different sample
    each step), largest first."""
    if rank != 0:
        return
    import oracle
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference library oracle/_ref/libnsref.so not built"}))
        return
    meshes = make_meshes(a.count, a.seed, 0)
    sides = [m.side for m in meshes]
    procs = os.cpu_count() or 1
    per_step = max(REF_PER_STEP, procs)
    pool = RefPool(procs)
    try:
        for w in range(a.warmup):
            pool.map(_ref_worker, [meshes[i] for i in stratified_sample(sides, procs, 7 + w)])
        solves, wall = 0, 0.0
        for s in range(a.steps):
            idx = stratified_sample(sides, per_step, s)
            _, t = pool.map(_ref_worker, [meshes[i] for i in idx])
            solves += len(idx)
            wall += t
    finally:
        pool.close()
    value = solves / wall
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(1e3 * wall / a.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded meshes)", "impl": "reference",
        "config": common_config(a),
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": procs, "kind": "reference",
                         "sample": f"{per_step} instances per step, evenly spread over the sorted "
                                   f"grid sides (a different sample each step), largest first; "
                                   f"reference solve_dc, one process per core, {cpu_model()}"},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    a = _args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank)
    else:
        run_ours(a, rank, world, local_rank)


if __name__ == "__main__":
    main()
