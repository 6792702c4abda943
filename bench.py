"""Benchmark of the B200 time-marching path: FP64 node-RK4-steps/s on the 256^3 Taylor-Green workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload tgv256|sphere48|spheres16|tgv128]

A step is one RK4 step (Solver::marchTimeStep) over the whole grid. Each rank runs an independent replica
(the single-grid path does not shard), so value = ranks x nodes x K / max-over-ranks device time. The
ensemble leg shards its members over the ranks (longest first, by node count) with no collective on the
data path; its time is the slowest rank's.
Timing: CUDA events on the solver's own stream around K graph-launched steps after W warm-up steps; the
resident fields (2.7 GB) are far larger than L2, so no flush is needed between steps.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "3d-ns-fsi_b200"))

import numpy as np  # noqa: E402

WORKLOADS = {
    "tgv256": dict(case="tgv256", desc="Taylor-Green vortex, periodic 256^3, M0=0.1, Re=1600, CFL 0.5, FP64"),
    "sphere48": dict(case="sphere48", desc="single sphere 48^3, inflow/outflow x, periodic y/z, M0=0.3, Re_D=100"),
    "spheres16": dict(case="spheres16", desc="16 spheres, 256x128x128, inflow/outflow x, periodic y/z, M0=0.3, "
                                             "Re_D=200 on the mean diameter"),
    "tgv128": dict(case="tgv128", desc="Taylor-Green vortex, periodic 128^3 (profiling size), FP64"),
}
BYTES_PER_NODE_STEP = 680  # algorithmic HBM bytes per node per RK4 step (stage-fused scheme)
STAGE_BYTES = [120, 200, 200, 160]


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(workload):
    """DRAM bytes (read + write) of the stage-kernel launches of one step of this workload, from the
    committed ncu summary profiles/k_stage_ws_<workload>_dram.md (its line `dram_bytes_per_launch: s1, s2, s3,
    s4`, one capture of the four stage launches of one step), as the mean per launch; None if absent."""
    p = os.path.join(ROOT, "profiles", "k_stage_ws_%s_dram.md" % workload)
    try:
        for line in open(p):
            if line.startswith("dram_bytes_per_launch:"):
                v = [float(x) for x in line.split(":")[1].split(",")]
                return {"per_launch": sum(v) / len(v), "per_stage": v, "source": os.path.relpath(p, ROOT)}
    except (OSError, ValueError):
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 1 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def host_model():
    """The host CPU's model name (first /proc/cpuinfo entry), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(case_path, nodes):
    """Serial CPU reference timed on this host: the reference build (oracle/_ref) if present, else the
    oracle port. Sample: one RK4 step of the same workload at full size."""
    from oracle import pyoracle as po
    if po.ref_available():
        r = po.time_reference(case_path, 0, 1)
        return {"value": r["node_steps_per_s"], "unit": "node-RK4-steps/s", "cores": 1, "kind": "reference",
                "sample": "1 RK4 step of the full workload grid (%d nodes), serial reference build, %.1f s" %
                          (nodes, r["seconds"]),
                "host_cores_present": os.cpu_count(), "host_model": host_model()}
    o = po.Oracle(open(case_path).read())
    sec = o.march(1)
    o.close()
    return {"value": nodes / sec, "unit": "node-RK4-steps/s", "cores": 1, "kind": "port",
            "sample": "1 RK4 step of the full workload grid (%d nodes), serial oracle port, %.1f s" % (nodes, sec),
            "host_cores_present": os.cpu_count(), "host_model": host_model()}


TUNE_CACHE = os.path.join(ROOT, "3d-ns-fsi_b200", "tuning", "stage_tiles.jsonl")


def reduce_over_ranks(x, dist, op="max"):
    """x reduced (max or sum) over all ranks of the process group (x itself without one)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x, dist):
    return reduce_over_ranks(x, dist, "max")


def shard_members(nodes, world):
    """The members each of `world` ranks advances: longest-processing-time-first over the members' node
    counts (ties by index), each rank's list in member order."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    for m in sorted(range(len(nodes)), key=lambda m: (-nodes[m], m)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(m)
        load[r] += nodes[m]
    return [sorted(p) for p in parts]


def ensemble_leg(steps, device, nsfsi, sequential=True, rank=0, world=1, dist=None):
    """Batched ensemble (64 seeded single-sphere flows on 5 grid shapes) against the same 64 runs made one
    after another on the plain path. Both timed on the device (CUDA events), setup excluded, alternating. With several
    ranks every rank advances its shard of the members (one graph per step for its shard) and the slowest
    rank's time counts; every rank must call this (it holds collectives)."""
    allCfgs = nsfsi.ensemble_configs(n=64, steps=steps)
    allNodes = [int(c.NI * c.NJ * c.NK) for c in allCfgs]
    mine = shard_members(allNodes, world)[rank]
    cfgs = [allCfgs[m] for m in mine]
    nodes = [allNodes[m] for m in mine]
    os.makedirs(os.path.dirname(TUNE_CACHE), exist_ok=True)

    def sync(x):
        # Members whose flow becomes non-finite keep marching, as the reference does (Mesh::checkFinity
        # prints and continues); the reference's own algorithm diverges on the same members.
        try:
            x.sync()
            return 0
        except nsfsi.NsfError as e:
            if e.code != 3:
                raise
            return 1

    # The ensemble run and the pass over the plain solves alternate, ENS_REPEATS times, so both see the same
    # thermal and power-cap history; the medians are compared (every run advances the same flows by `steps`).
    ens_runs, seq_runs = [], []
    nonfinite = 0
    with nsfsi.Ensemble(cfgs, device=device, tune_cache=TUNE_CACHE) as ens:
        tile, lps, items = ens.info()
        ens.march(3)
        sync(ens)
        solvers = [nsfsi.Solver(c, device=device) for c in cfgs] if sequential else []
        try:
            for s in solvers:
                s.march(3)
                sync(s)
            for r in range(ENS_REPEATS):
                ens_runs.append(ens.march_timed(steps))
                sync(ens)
                if sequential:
                    t = 0.0
                    for s in solvers:
                        t += s.march_timed(steps)
                        bad = sync(s)
                        if r == 0:
                            nonfinite += bad  # after the first `steps` steps, as the configurations state
                    seq_runs.append(t)
        finally:
            for s in solvers:
                s.close()
    ens_ms = statistics.median(ens_runs)
    seq_ms = statistics.median(seq_runs) if sequential else 0.0
    # the slowest rank's times; non-finite members summed over the ranks
    ens_ms = max_over_ranks(ens_ms, dist)
    seq_ms = max_over_ranks(seq_ms, dist)
    nonfinite = int(reduce_over_ranks(nonfinite, dist, "sum"))
    work = sum(allNodes) * steps
    return {"workload": "64 single-sphere flows, shapes 32^3/48^3/64^3/96x64x64/128x64x64, M U[0.2,0.4], "
                        "Re_D U[50,300], D U[0.15,0.25]", "members": len(allCfgs), "nodes": sum(allNodes),
            "ranks": world, "members_per_rank": len(cfgs),
            "steps": steps, "value": work / (ens_ms / 1e3), "unit": "node-RK4-steps/s",
            "sequential_value": work / (seq_ms / 1e3) if sequential else None,
            "speedup_vs_sequential": seq_ms / ens_ms if sequential else None,
            "ms": ens_ms, "sequential_ms": seq_ms if sequential else None, "tile": ["32x8", "16x16"][tile], "launches_per_step": lps,
            "stage_work_items": items, "nonfinite_members": nonfinite, "repeats": len(ens_runs),
            "ms_repeats": [round(x, 2) for x in ens_runs], "sequential_ms_repeats": [round(x, 2) for x in seq_runs]}


def adjoint_leg(device, nsfsi, reps=3, steps=200):
    """Discrete adjoint on a 64^3 channel with a sphere (200 RK4 steps, J = the sphere's x-force averaged
    over the last 50 steps): wall time of the synchronous forward and backward calls (host overhead
    included) with the default tape limit (the forward run records every step's snapshot set when they fit
    in half the free device memory) and with checkpointing only (20 slots), against one plain forward
    solve; with 20 slots and a segment tape of two segments' sets; the finite-difference agreement along
    two seeded directions (h = 1e-6) and the device time of one adjoint step by phase."""
    cfg = nsfsi.config_load(nsfsi.case_path("adj64"))
    cfg.stop_time_level = steps
    navg = max(1, min(50, steps // 4))
    def timed(s):
        s.adj_forward()
        s.adj_backward()  # captures the adjoint step graphs
        fwd, bwd = [], []
        for _ in range(reps):
            t0 = time.perf_counter()
            J = s.adj_forward()
            t1 = time.perf_counter()
            gi, gu = s.adj_backward()
            t2 = time.perf_counter()
            fwd.append(t1 - t0)
            bwd.append(t2 - t1)
        return J, gi, gu, float(np.median(fwd)), float(np.median(bwd))

    with nsfsi.Solver(cfg, device=device) as s:  # binomial checkpointing only (20 slots), for comparison
        s.adj_configure(navg, 20)
        s.adj_tape_limit(0)
        _, _, _, cf, cb = timed(s)
    with nsfsi.Solver(cfg, device=device) as s:
        u0 = s.download(range(5))
        s.adj_configure(navg, 20)
        J, gi, gu, f, b = timed(s)
        tape_bytes = s.adj_tape_bytes()
        phases = s.adj_profile_step(steps // 2)
        rng = np.random.default_rng(2024)
        scale = np.maximum(np.abs(u0).max(axis=1), 1e-3)[:, None]
        errs = []
        for _ in range(2):
            du = rng.standard_normal(u0.shape) * scale
            di = rng.standard_normal(gi.shape)
            ad = float((gu * du).sum() + (gi * di).sum())
            h = 1e-6
            fd = (s.adj_forward(u0 + h * du, 1 + h * di) - s.adj_forward(u0 - h * du, 1 - h * di)) / (2 * h)
            errs.append(abs(fd - ad) / abs(ad))
    # 20 slots and a tape of two segments' sets (a state every ceil(steps / 21) steps; the backward run
    # records each segment's sets from its state)
    seg = {}
    if tape_bytes:
        set_bytes = tape_bytes // steps
        seg_steps = -(-steps // 21)
        with nsfsi.Solver(cfg, device=device) as s:
            s.adj_configure(navg, 20)
            s.adj_tape_limit(2 * seg_steps * set_bytes)
            _, sgi, sgu, sf, sb = timed(s)
            seg_bytes, seg_len = s.adj_segment_tape()
            seg = {"snapshots": 20, "segment_steps": seg_len, "segment_tape_bytes": seg_bytes,
                   "forward_ms": sf * 1e3, "backward_ms": sb * 1e3,
                   "same_gradient_as_tape": bool(np.array_equal(sgi, gi) and np.array_equal(sgu, gu))}
    # one plain forward solve of the same case and length (the solver's step graph, no checkpoints), timed
    # after a warm-up run: wall time of the synchronous march + sync, and device time
    plain_wall, plain_dev = [], []
    with nsfsi.Solver(cfg, device=device) as p:
        p.march(steps)
        p.sync()
        for _ in range(reps):
            t0 = time.perf_counter()
            p.march(steps)
            p.sync()
            plain_wall.append(time.perf_counter() - t0)
            plain_dev.append(p.march_timed(steps) / 1e3)
    pf = float(np.median(plain_wall))
    return {"workload": "adj64: 64^3 channel, sphere D=0.2 at (0.4,0.5,0.5), M 0.3, Re_D 100 (Re 1666.7 per unit "
                        "length on the speed of sound), %d RK4 steps, J over the last %d" % (steps, navg),
            "mode": "tape" if tape_bytes else "checkpoints", "tape_bytes": tape_bytes,
            "J": J, "forward_ms": f * 1e3, "backward_ms": b * 1e3, "backward_over_forward": b / f,
            "plain_forward_ms": pf * 1e3, "plain_forward_device_ms": float(np.median(plain_dev)) * 1e3,
            "backward_over_plain_forward": b / pf, "gradient_over_plain_forward": (f + b) / pf,
            "checkpointed": {"snapshots": 20, "forward_ms": cf * 1e3, "backward_ms": cb * 1e3,
                             "gradient_over_plain_forward": (cf + cb) / pf},
            "segment_tape": dict(seg, gradient_over_plain_forward=(seg["forward_ms"] + seg["backward_ms"]) / 1e3 / pf)
            if seg else None,
            "fd_step": 1e-6, "fd_rel_err_max": max(errs), "fd_directions": len(errs),
            "adjoint_step_phase_ms": {k: round(v, 4) for k, v in phases.items()}}


SAVE_FIELDS = (("save_density", [0]), ("save_momentum", [1, 2, 3]), ("save_energy", [4]),
               ("save_velocity", [5, 6, 7]), ("save_pressure", [8]), ("save_temperature", [9]),
               ("save_viscosity", [10]), ("save_thermal_cond", [11]))


def snapshot_leg(cfg, device, nsfsi, steps=60, every=20):
    """Cost of snapshot output inside the march: the host loop of Simulation::run (march one step, read
    t/dt/timeLevel) with a snapshot of the fields the case saves every `every` steps, as
    OutputManager::storeCurrentSolution takes them. Modes: no snapshot; a synchronous download of all twelve
    fields into pageable memory (what a host mirror of every field costs); a synchronous download of the saved
    fields into a page-locked buffer; nsf_download_async of the saved fields into two reused page-locked buffers (the snapshot writer's
    scheme, without the file formatting, which runs on the writer's thread). Host wall clock per step, each
    mode run twice and the second run kept (the first allocates staging buffers)."""
    import ctypes
    L = nsfsi.lib()
    saved = [f for name, fs in SAVE_FIELDS if getattr(cfg, name) for f in fs]
    mask = sum(1 << f for f in saved)
    s = nsfsi.Solver(cfg, device=device)
    N, nf = s.N, len(saved)
    dp = ctypes.POINTER(ctypes.c_double)
    bufs = []
    for _ in range(2):
        p = ctypes.c_void_p()
        s._check(L.nsf_host_alloc(8 * nf * N, ctypes.byref(p)))
        bufs.append(p)
    host_all = np.empty((12, N))

    def run(mode):
        tickets = [0, 0]
        s.march(3)
        s.sync()
        t0 = time.perf_counter()
        for q in range(1, steps + 1):
            s.march(1)
            s.time()
            if q % every:
                continue
            if mode == "sync_all":
                s._check(L.nsf_download(s.h, 0xFFF, host_all.ctypes.data_as(dp)))
            elif mode == "sync_saved":
                s._check(L.nsf_download(s.h, mask, ctypes.cast(bufs[0], dp)))
            elif mode == "async":
                b = (q // every) & 1
                if tickets[b]:
                    s._check(L.nsf_download_wait(s.h, tickets[b]))
                t = ctypes.c_uint64()
                s._check(L.nsf_download_async(s.h, mask, ctypes.cast(bufs[b], dp), ctypes.byref(t)))
                tickets[b] = t.value
        for t in tickets:
            if t:
                s._check(L.nsf_download_wait(s.h, t))
        return (time.perf_counter() - t0) * 1e3 / steps

    try:
        ms = {}
        for mode in ("none", "sync_all", "sync_saved", "async"):
            run(mode)
            ms[mode] = run(mode)
        # one snapshot's trip to the host with nothing else queued: the bound on how often snapshots hide
        s.sync()
        t = ctypes.c_uint64()
        t0 = time.perf_counter()
        s._check(L.nsf_download_async(s.h, mask, ctypes.cast(bufs[0], dp), ctypes.byref(t)))
        s._check(L.nsf_download_wait(s.h, t.value))
        trip_ms = (time.perf_counter() - t0) * 1e3
    finally:
        s.close()
        for p in bufs:
            L.nsf_host_free(p)
    n_snap = steps // every
    return {"steps": steps, "every": every, "fields_saved": nf, "bytes_per_snapshot": 8 * nf * N,
            "async_trip_ms": round(trip_ms, 3), "async_trip_gbs": round(8 * nf * N / trip_ms / 1e6, 2),
            "ms_per_step": {k: round(v, 4) for k, v in ms.items()},
            "ms_per_snapshot_over_none": {k: round((ms[k] - ms["none"]) * steps / n_snap, 3)
                                          for k in ("sync_all", "sync_saved", "async")},
            "timing": "host wall clock; march 1 + t/dt/timeLevel read per step, snapshot every `every` steps"}


def case_file(workload):
    return os.path.join(ROOT, "3d-ns-fsi_b200", "cases", WORKLOADS[workload]["case"] + ".cfg")


def case_grid(path):
    """NI, NJ, NK of a case file, read as text (the reference arm loads nothing of the product)."""
    import re
    text = open(path).read()
    return [int(re.search(r"^\s*%s\s*=\s*(\d+)" % k, text, re.M).group(1)) for k in ("NI", "NJ", "NK")]


def arm_config(workload, grid, world):
    """The `config` object of the JSON line, the same for both arms."""
    return {"workload": workload, "desc": WORKLOADS[workload]["desc"], "grid": grid,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "resident fields 2.7 GB >> 126 MB L2; no flush" if workload == "tgv256" else
                  "resident fields larger than the 126 MB L2; no flush"}


ENS_REPEATS = 3           # alternating ensemble runs and passes over the plain solves; medians compared
E2E_REPEATS = 3           # end-to-end runs (upload, K steps, download); the median is reported
REF_ARM_BUDGET_S = 330.0   # the reference arm's whole run (warm-up and timed steps) stays within minutes
REF_RATE_ESTIMATE = 1.5e6  # node-RK4-steps/s of the serial reference build on one host core


def run_reference_arm(args, rank, world):
    """The reference solver itself (oracle/_ref/ref_runner: the reference's own src/*.cpp compiled unmodified)
    on the host cores: W warm-up steps, then K timed calls of Solver::marchTimeStep on the full workload
    grid. The reference is serial (no threads), so it runs on one core; under torchrun rank 0 alone runs.
    Nothing of the product (library, kernels, Python package) is loaded in this arm."""
    if rank != 0:
        return
    case = case_file(args.workload)
    grid = case_grid(case)
    nodes = grid[0] * grid[1] * grid[2]
    ref_runner = os.path.join(ROOT, "oracle", "_ref", "ref_runner")
    if not os.path.exists(ref_runner):
        print(json.dumps({"impl": "reference", "unavailable": "the reference build oracle/_ref/ref_runner is absent "
                          "(build it with oracle/Makefile.ref from the reference sources)"}), flush=True)
        return
    # whole requested run if it fits the budget, else as many timed steps as fit (stated in the line)
    est = nodes / REF_RATE_ESTIMATE
    k = args.steps
    if (args.warmup + k) * est > REF_ARM_BUDGET_S:
        k = max(1, int(REF_ARM_BUDGET_S / est) - args.warmup)
    out = subprocess.run([ref_runner, case, tempfile.gettempdir(), "--time", str(args.warmup), str(k)], check=True,
                         capture_output=True, text=True).stdout
    r = json.loads(out.strip().splitlines()[-1])
    value, sec = float(r["node_steps_per_s"]), float(r["seconds"])
    sample = "%d warm-up and %d timed RK4 steps of the full %s grid (%d nodes), serial reference build, 1 core of %d" % (
        args.warmup, k, args.workload, nodes, os.cpu_count())
    if k != args.steps:
        sample += "; %d of the requested %d steps fit the arm's time budget" % (k, args.steps)
    line = {"impl": "reference", "metric": "node-RK4-steps/s (FP64)", "value": value, "unit": "node-RK4-steps/s",
            "n_gpus": 0, "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * sec / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": arm_config(args.workload, grid, world),
            "cpu_baseline": {"value": value, "unit": "node-RK4-steps/s", "cores": 1, "kind": "reference",
                             "sample": sample, "host_model": host_model()},
            "e2e": {"value": value, "unit": "node-RK4-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def arg_parser():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--repeats", type=int, default=10, help="repeats of the K-step timed region (median reported)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tgv256", choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--ensemble-steps", type=int, default=200, help="RK4 steps of the ensemble leg (0: skip)")
    ap.add_argument("--ensemble-only", action="store_true", help="run only the ensemble leg (profiling)")
    ap.add_argument("--no-seq", action="store_true", help="ensemble leg without the sequential comparison")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the discrete-adjoint leg")
    ap.add_argument("--no-snapshots", action="store_true", help="skip the snapshot-output leg")
    ap.add_argument("--adjoint-only", action="store_true", help="run only the discrete-adjoint leg (profiling)")
    ap.add_argument("--adjoint-steps", type=int, default=200, help="RK4 steps of the adjoint leg")
    return ap


def main():
    args = arg_parser().parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import nsfsi
    if args.ensemble_only:
        leg = ensemble_leg(args.ensemble_steps, local, nsfsi, sequential=not args.no_seq, rank=rank, world=world,
                           dist=dist)
        if rank == 0:
            print(json.dumps(leg), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.adjoint_only:
        print(json.dumps(adjoint_leg(local, nsfsi, steps=args.adjoint_steps)), flush=True)
        return
    wl = WORKLOADS[args.workload]
    case = nsfsi.case_path(wl["case"])
    cfg = nsfsi.config_load(case)
    nodes = int(cfg.NI * cfg.NJ * cfg.NK)

    nonfinite = [False]

    def sync(x):
        # a flow that goes non-finite keeps marching, as the reference does (Mesh::checkFinity prints and
        # continues); the kernels and their timing do not depend on the values
        try:
            x.sync()
        except nsfsi.NsfError as e:
            if e.code != 3:
                raise
            nonfinite[0] = True

    s = nsfsi.Solver(cfg, device=local)
    s.march(args.warmup)
    sync(s)
    import torch
    if dist:
        dist.barrier()
    # The timed region (exactly K graph-launched steps between two events) is repeated R times; the line
    # reports the median, and the clock sampler runs across all repeats.
    reps_ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.repeats):
            reps_ms.append(s.march_timed(args.steps))
        sync(s)
    ms = statistics.median(reps_ms)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * nodes * args.steps / (ms / 1e3)
    interior = int((cfg.NI - 2) * (cfg.NJ - 2) * (cfg.NK - 2))  # nodes whose RHS is computed
    launches = s.launches_per_step()

    # dominant kernel: the four stage kernels timed by event nodes inside replays of a graph of consecutive
    # steps (nsf_profile_steps), straight after the timed region; their share of those replays' step time,
    # applied to the timed region's ms_per_step, is the stage kernels' time per step (it cannot exceed the
    # step), and the roofline's achieved bandwidth follows from it
    with ClockSampler(local) as clkp:
        stage_ms, step_ms = s.profile_steps(max(args.steps, 50))
    share = float(stage_ms.sum() / step_ms)
    stage_step_ms = share * ms / args.steps
    achieved = BYTES_PER_NODE_STEP * nodes / (stage_step_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    traffic = profile_traffic(args.workload)
    s.close()

    # end to end through the C ABI with host buffers: pinned upload of the initial state, K steps with
    # the per-step t/dt/timeLevel read-back Simulation::run needs, pinned download of the final state
    # (every rank runs its replica; the slowest rank's wall time counts)
    e2e = None
    if not args.no_e2e:
        s2 = nsfsi.Solver(cfg, device=local)
        u0 = s2.download(range(5))
        pin_in = torch.empty((5, nodes), dtype=torch.float64, pin_memory=True)
        pin_in.numpy()[:] = u0
        pin_out = torch.empty((5, nodes), dtype=torch.float64, pin_memory=True)
        import ctypes
        dp = ctypes.POINTER(ctypes.c_double)
        L = nsfsi.lib()
        s2.march(args.warmup)
        sync(s2)
        runs = []  # (wall, upload, steps, download) seconds; the run is repeated and the median kept
        for _ in range(E2E_REPEATS):
            t0 = time.perf_counter()
            s2._check(L.nsf_upload_conserved(s2.h, ctypes.cast(pin_in.data_ptr(), dp)))
            t1 = time.perf_counter()
            for _ in range(args.steps):
                s2.march(1)
                s2.time()
            t2 = time.perf_counter()
            s2._check(L.nsf_download(s2.h, 31, ctypes.cast(pin_out.data_ptr(), dp)))
            t3 = time.perf_counter()
            runs.append((t3 - t0, t1 - t0, t2 - t1, t3 - t2))
        s2.close()
        runs.sort()
        wall, up, st, down = runs[len(runs) // 2]
        if dist:
            t = torch.tensor([wall], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            wall = float(t.item())
        e2e = {"value": world * nodes * args.steps / wall, "unit": "node-RK4-steps/s",
               "h2d_bytes_per_step": 5 * 8 * nodes / args.steps,
               "d2h_bytes_per_step": (5 * 8 * nodes + 24 * args.steps) / args.steps,
               "repeats": len(runs), "wall_ms_repeats": [round(r[0] * 1e3, 2) for r in runs],
               "median_run_ms": {"upload": round(up * 1e3, 2), "steps": round(st * 1e3, 2),
                                 "download": round(down * 1e3, 2)},
               "timing": "host wall clock around upload + K x (march 1, read t/dt/timeLevel) + download; "
                         "median of the repeats"}

    snaps = None
    if not args.no_snapshots and args.workload == "tgv256" and rank == 0:
        snaps = snapshot_leg(cfg, local, nsfsi)

    ens = None
    if args.ensemble_steps > 0 and args.workload == "tgv256":  # every rank takes its shard
        ens = ensemble_leg(args.ensemble_steps, local, nsfsi, sequential=not args.no_seq, rank=rank, world=world,
                           dist=dist)
    if rank == 0:
        line = {
            "metric": "node-RK4-steps/s (FP64)", "value": value, "unit": "node-RK4-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "interior_value": world * interior * args.steps / (ms / 1e3),
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": arm_config(args.workload, [int(cfg.NI), int(cfg.NJ), int(cfg.NK)], world),
            "e2e": e2e,
            "nonfinite": nonfinite[0],
            "gpu_launches": launches * args.steps,
            "clocks": clk.summary(),
            "repeats": args.repeats, "ms_per_step_repeats": [round(x / args.steps, 5) for x in reps_ms],
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         # DRAM bytes per stage-kernel launch (mean of the four stages) from the committed ncu
                         # capture of this workload, next to the algorithmic bytes per launch
                         "traffic": traffic["per_launch"] if traffic else None,
                         "traffic_source": traffic["source"] if traffic else None,
                         "algorithmic_bytes_per_launch": BYTES_PER_NODE_STEP * nodes / 4,
                         "kernel": "k_stage_ws (4 launches per step)", "stage_ms_per_step": round(stage_step_ms, 4),
                         "stage_share": round(share, 4), "stage_ms_profiled": [round(x, 4) for x in stage_ms],
                         "algorithmic_bytes_per_node_step": BYTES_PER_NODE_STEP, "peak_kind": peak_kind,
                         "frac_of_8000": achieved / 8000.0, "profile_step_ms": round(step_ms, 4),
                         # whole step (edge and control launches included): node-steps/s per GPU against
                         # the node-steps/s the peak bandwidth allows at 680 B per node-step
                         "step_frac": value / world / (peak * 1e9 / BYTES_PER_NODE_STEP),
                         "profile_clocks": clkp.summary()},
        }
        if snaps is not None:
            line["snapshots"] = snaps
        if ens is not None:
            line["ensemble"] = ens
        if not args.no_adjoint and args.workload == "tgv256":
            line["adjoint"] = adjoint_leg(local, nsfsi, steps=args.adjoint_steps)
        if world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(case, nodes)
            except Exception as e:  # noqa: BLE001
                line["cpu_baseline"] = {"value": None, "error": str(e)}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
