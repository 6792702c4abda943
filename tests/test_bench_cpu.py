"""bench.py keeps its output contract, checked on the CPU: the main arm run in-process against a stand-in
solver module (fixed device times, no device), the CPU-baseline helper on a small case, and the reference
arm on the 48^3 sphere workload for one step."""
import json
import os
import subprocess
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

STAGE_MS = [0.7, 0.72, 0.72, 0.8]
STEP_MS = 3.1


def fake_nsfsi():
    """A module with the solver API bench.py's main arm calls, reporting fixed times."""
    m = types.ModuleType("nsfsi")

    class NsfError(RuntimeError):
        code = 0

    class Cfg:
        NI = NJ = NK = 256

    class Solver:
        def __init__(self, cfg, device=0):
            pass

        def march(self, n):
            pass

        def sync(self):
            pass

        def march_timed(self, n):
            return STEP_MS * n

        def launches_per_step(self):
            return 19

        def profile_steps(self, n):
            return np.array(STAGE_MS), STEP_MS + 0.05

        def close(self):
            pass

    m.NsfError, m.Solver = NsfError, Solver
    m.case_path = lambda name: name
    m.config_load = lambda path: Cfg()
    return m


def test_main_arm_line_keeps_the_contract(monkeypatch, capsys):
    monkeypatch.setitem(sys.modules, "nsfsi", fake_nsfsi())
    monkeypatch.setattr(sys, "argv", ["bench.py", "--steps", "10", "--warmup", "3", "--no-e2e", "--ensemble-steps",
                                      "0", "--no-adjoint", "--no-cpu-baseline", "--no-snapshots"])
    bench.main()
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    nodes = 256 ** 3
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "clocks", "roofline"):
        assert key in line, key
    assert line["n_gpus"] == 1 and line["steps"] == 10 and line["warmup"] == 3
    assert line["higher_is_better"] is True and line["scaling"] == "weak" and line["dtype"] == "f64"
    assert line["config"]["workload"] == "tgv256"
    assert line["value"] == pytest.approx(nodes * 10 / (STEP_MS * 10 / 1e3))
    assert line["ms_per_step"] == pytest.approx(STEP_MS)
    assert line["interior_value"] == pytest.approx(254 ** 3 * 10 / (STEP_MS * 10 / 1e3))
    assert line["gpu_launches"] == 190
    assert set(line["clocks"]) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    r = line["roofline"]
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in r, key
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    share = sum(STAGE_MS) / (STEP_MS + 0.05)
    assert r["stage_share"] == pytest.approx(share, abs=1e-4)
    assert r["achieved"] == pytest.approx(680 * nodes / (share * STEP_MS / 1e3) / 1e9)
    assert r["stage_ms_per_step"] <= line["ms_per_step"]
    assert line["repeats"] == 10 and len(line["ms_per_step_repeats"]) == 10
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    assert r["step_frac"] == pytest.approx(line["value"] / (r["peak"] * 1e9 / 680))
    assert line["e2e"] is None  # --no-e2e


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref/ref_runner absent")
def test_cpu_baseline_describes_its_sample():
    case = os.path.join(ROOT, "tests", "golden", "cases", "tgv_small.cfg")
    b = bench.cpu_baseline(case, 14 * 12 * 13)
    assert b["kind"] == "reference" and b["cores"] == 1 and b["unit"] == "node-RK4-steps/s"
    assert b["value"] > 0 and "RK4 step" in b["sample"]
    assert b["host_cores_present"] >= 1 and "host_model" in b


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref/ref_runner absent")
def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "sphere48", "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300,
                         check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "node-RK4-steps/s"
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["steps"] == 1 and line["warmup"] == 3
    assert line["config"] == bench.arm_config("sphere48", [48, 48, 48], 1)


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref/ref_runner absent")
def test_reference_arm_loads_nothing_of_the_product():
    """The reference arm, run in a fresh process with the product's Python package made unimportable, maps
    no product library into the process."""
    script = (
        "import json, sys\n"
        "sys.modules['nsfsi'] = None\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'sphere48', '--steps', '2', '--warmup', '3']\n"
        "import bench\n"
        "bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'libnsfsi_mapped': 'libnsfsi' in maps, 'liboracle_mapped': 'liboracle' in maps}))\n")
    out = subprocess.run([sys.executable, "-c", script], cwd=ROOT, capture_output=True, text=True, timeout=300,
                         check=True).stdout.strip().splitlines()
    line, maps = json.loads(out[-2]), json.loads(out[-1])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 3
    assert maps == {"libnsfsi_mapped": False, "liboracle_mapped": False}


def test_reference_arm_budget_bounds_the_timed_steps():
    """A requested run longer than the arm's time budget is cut to the steps that fit, and says so."""
    nodes = 256 ** 3
    est = nodes / bench.REF_RATE_ESTIMATE
    assert (5 + 20) * est <= bench.REF_ARM_BUDGET_S  # the round-end command (20 steps, 5 warm-up) runs whole
    assert (5 + 200) * est > bench.REF_ARM_BUDGET_S


def test_case_grid_reads_the_case_text():
    assert bench.case_grid(bench.case_file("tgv256")) == [256, 256, 256]
    assert bench.case_grid(bench.case_file("spheres16")) == [256, 128, 128]


def test_profile_commands_parse():
    """Every bench.py command a profile summary names still parses with bench.py's options."""
    import glob
    import re
    import shlex
    cmds = set()
    for path in glob.glob(os.path.join(ROOT, "profiles", "*.md")):
        text = open(path).read().replace("\\\n", " ")
        cmds.update(m.strip() for m in re.findall(r"python bench\.py([^`\n]*)", text))
    assert cmds
    for c in cmds:
        bench.arg_parser().parse_args(shlex.split(c))


def test_roofline_traffic_comes_from_the_committed_capture():
    """roofline.traffic is the mean DRAM bytes per stage launch of the committed 256^3 capture: four launches,
    each within 5 % of its stage's algorithmic bytes (120 / 200 / 200 / 160 B per node), the step within 2 %."""
    t = bench.profile_traffic("tgv256")
    assert t is not None and t["source"] == os.path.join("profiles", "k_stage_ws_tgv256_dram.md")
    nodes = 256 ** 3
    alg = [120 * nodes, 200 * nodes, 200 * nodes, 160 * nodes]
    assert len(t["per_stage"]) == 4
    for got, want in zip(t["per_stage"], alg):
        assert abs(got / want - 1) < 0.05
    assert abs(sum(t["per_stage"]) / (bench.BYTES_PER_NODE_STEP * nodes) - 1) < 0.02
    assert t["per_launch"] == pytest.approx(sum(t["per_stage"]) / 4)


def test_ensemble_leg_alternates_and_compares_medians():
    """The ensemble leg alternates ensemble runs with passes over the plain solves (ENS_REPEATS of each, on a
    stand-in module whose device times drift run by run) and compares the medians; the non-finite members are
    counted once, after the first pass."""
    calls = []

    class Cfg:
        def __init__(self, n):
            self.NI = self.NJ = self.NK = n

    class NsfError(RuntimeError):
        def __init__(self, code):
            self.code = code

    ens_ms = iter([100.0, 90.0, 95.0])

    class Ensemble:
        def __init__(self, cfgs, device=0, tune_cache=None):
            self.n = len(cfgs)

        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

        def info(self):
            return 0, 10, 7

        def march(self, n):
            pass

        def sync(self):
            pass

        def march_timed(self, n):
            calls.append("ens")
            return next(ens_ms)

    seq_ms = {0: 2.0, 1: 3.0, 2: 2.5}

    class Solver:
        passes = 0

        def __init__(self, cfg, device=0):
            self.cfg = cfg
            self.runs = 0

        def march(self, n):
            pass

        def sync(self):
            if self.cfg.NI == 8 and self.runs > 0:  # one member goes non-finite
                raise NsfError(3)

        def march_timed(self, n):
            calls.append("seq")
            t = seq_ms[self.runs] * self.cfg.NI
            self.runs += 1
            return t

        def close(self):
            pass

    m = types.ModuleType("nsfsi")
    m.NsfError, m.Solver, m.Ensemble = NsfError, Solver, Ensemble
    m.ensemble_configs = lambda n, steps: [Cfg(8), Cfg(16)]
    out = bench.ensemble_leg(20, 0, m)
    assert calls == ["ens", "seq", "seq"] * 3
    assert out["repeats"] == 3 and out["ms_repeats"] == [100.0, 90.0, 95.0]
    assert out["sequential_ms_repeats"] == [2.0 * 24, 3.0 * 24, 2.5 * 24]
    assert out["ms"] == 95.0 and out["sequential_ms"] == 2.5 * 24
    assert out["speedup_vs_sequential"] == pytest.approx(2.5 * 24 / 95.0)
    assert out["nonfinite_members"] == 1
    assert out["value"] == pytest.approx((8 ** 3 + 16 ** 3) * 20 / 0.095)
