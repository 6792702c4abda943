"""Regenerates the golden fixtures under tests/golden/ from the reference solver itself.

Run in a container that has the reference sources (the build recipe oracle/Makefile.ref compiles them
into oracle/_ref/ref_runner):

    make -f oracle/Makefile.ref && python tests/golden/make_golden.py

For every case file in tests/golden/cases/ it runs the unmodified reference (through oracle/ref_harness.cpp)
and stores, in <case>.npz: node types, per-body ghost lists (i, j, k, body-intercept point, image point)
and filter-node lists, the initial dt, the per-step history (t, dt used, dt next, five change norms) and
all twelve fields (rho, rho_u, rho_v, rho_w, rho_E, u, v, w, p, T, mu, kappa) at the listed steps and
at the last step run (an end_time case stops where Simulation::run stops, so later listed steps are
replaced by that final step).
For the 48^3 sphere workload and the 16-sphere 256x128x128 workload it stores a fixed node subsample of the
fields instead of whole arrays (the 16-sphere run stops after its last listed step).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import pyoracle as po  # noqa: E402

# case name -> (config path, steps at which all fields are stored, subsample stride or None)
CASES = {
    "sphere_small": ("tests/golden/cases/sphere_small.cfg", [7, 30], None),
    "tgv_small": ("tests/golden/cases/tgv_small.cfg", [25], None),
    "two_spheres": ("tests/golden/cases/two_spheres.cfg", [20], None),
    "close_spheres": ("tests/golden/cases/close_spheres.cfg", [6, 20], None),
    "cylinder_sym": ("tests/golden/cases/cylinder_sym.cfg", [4, 60], None),
    "shipped_small": ("tests/golden/cases/shipped_small.cfg", [40], None),
    "sphere48": ("3d-ns-fsi_b200/cases/sphere48.cfg", [100], 13),
    "spheres16": ("3d-ns-fsi_b200/cases/spheres16.cfg", [2], 509),
}


def make(name):
    cfg, dumps, stride = CASES[name]
    out = po.run_reference(os.path.join(ROOT, cfg), [0] + dumps, final=True)
    s = po.read_ref_setup(out)
    rec = dict(shape=np.array(s["shape"]), geometry=s["geometry"], types=s["types"], dt0=np.array(s["dt0"]),
               history=po.read_ref_history(out), dumps=np.array(dumps), nbodies=np.array(len(s["bodies"])))
    for b, (g, f) in enumerate(s["bodies"]):
        rec["ghosts_%d" % b] = g
        rec["filter_%d" % b] = f
    fin = po.read_ref_fields(out, "final")
    rec["final_level"] = np.array(fin["level"])
    dumps = [d for d in dumps if d < fin["level"]] + [fin["level"]]
    rec["dumps"] = np.array(dumps)
    for d in dumps:
        fl = fin if d == fin["level"] else po.read_ref_fields(out, d)
        f = fl["fields"]
        if stride:
            idx = np.arange(0, f.shape[1], stride)
            rec["sample_idx"] = idx
            f = f[:, idx]
        rec["fields_%d" % d] = f
        rec["t_%d" % d] = np.array(fl["t"])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
    print(name, "ok", os.path.getsize(os.path.join(HERE, name + ".npz")))


# VTK / times.dat / norm files written by the reference's own OutputManager at the end of a run
# (ref_runner --vtk), gzipped into tests/golden/vtk_<case>/.
VTK_CASES = {"sphere_small": ("tests/golden/cases/sphere_small.cfg", 30)}


def make_vtk(name):
    import gzip
    import shutil
    import subprocess
    import tempfile
    cfg, steps = VTK_CASES[name]
    out = tempfile.mkdtemp(prefix="nsf_vtk_")
    subprocess.run([po.REF_RUNNER, os.path.join(ROOT, cfg), out, "--dump", str(steps), "--vtk"], check=True,
                   stdout=subprocess.DEVNULL)
    dst = os.path.join(HERE, "vtk_" + name)
    os.makedirs(dst, exist_ok=True)
    for f in sorted(os.listdir(os.path.join(out, "output"))):
        with open(os.path.join(out, "output", f), "rb") as src, gzip.open(os.path.join(dst, f + ".gz"), "wb") as g:
            shutil.copyfileobj(src, g)
    print("vtk_" + name, "ok", sorted(os.listdir(dst)))


if __name__ == "__main__":
    if not po.ref_available():
        sys.exit("oracle/_ref/ref_runner is not built; run make -f oracle/Makefile.ref first")
    for n in (sys.argv[1:] or list(CASES) + ["vtk_" + v for v in VTK_CASES]):
        make_vtk(n[4:]) if n.startswith("vtk_") else make(n)
