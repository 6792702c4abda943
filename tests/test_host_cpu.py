"""The C++ host layer (3d-ns-fsi_b200/host/nsfsi_host.hpp): the reference-style classes over the C ABI.

* The VTK writer (OutputManager mirror) must produce, for the reference's own field values, exactly the
  bytes the reference's OutputManager wrote (golden files made by tests/golden/make_golden.py through
  ref_runner --vtk).
* The drop-in driver program (host/main.cpp -> bin/nsfsi_main) must link and fail loudly without a GPU.
"""
import gzip
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "3d-ns-fsi_b200")
GOLD = os.path.join(ROOT, "tests", "golden")


def build_check(tmp):
    exe = os.path.join(tmp, "vtk_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "host"),
                    os.path.join(ROOT, "tests", "host", "vtk_check.cpp"), "-o", exe, "-L", os.path.join(PKG, "lib"),
                    "-lnsfsi", "-Wl,-rpath," + os.path.join(PKG, "lib"), "-pthread"], check=True)
    return exe


@pytest.mark.parametrize("mode", ["mirrors", "packed", "writer"])
def test_vtk_writer_matches_reference_bytes(mode):
    """The VTK text from the Mesh mirrors, from packed saved fields only (the snapshot download's layout) and
    from the snapshot writer's worker thread, each byte for byte against the reference's own file."""
    g = np.load(os.path.join(GOLD, "sphere_small.npz"))
    lvl = int(g["final_level"])
    fields = g["fields_%d" % lvl]
    t = float(g["t_%d" % lvl])
    ref = gzip.open(os.path.join(GOLD, "vtk_sphere_small", "out.vtk.0.gz")).read()
    with tempfile.TemporaryDirectory() as tmp:
        exe = build_check(tmp)
        fb = os.path.join(tmp, "fields.bin")
        np.ascontiguousarray(fields, dtype=np.float64).tofile(fb)
        out = os.path.join(tmp, "out.vtk")
        r = subprocess.run([exe, os.path.join(ROOT, "tests/golden/cases/sphere_small.cfg"), fb, repr(t), out, mode],
                           capture_output=True, text=True)
        assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
        if mode == "writer":
            assert "refused: NSF_ERR_" in r.stdout
        mine = open(out, "rb").read()
    assert mine == ref


def test_driver_program_fails_loudly_without_gpu():
    exe = os.path.join(PKG, "bin", "nsfsi_main")
    assert os.path.exists(exe)
    with tempfile.TemporaryDirectory() as tmp:
        r = subprocess.run([exe, os.path.join(ROOT, "tests/golden/cases/sphere_small.cfg"), os.path.join(tmp, "out")],
                           capture_output=True, text=True, cwd=tmp)
    assert r.returncode == 1
    assert "nsf_create" in r.stderr


def test_driver_program_rejects_bad_config():
    exe = os.path.join(PKG, "bin", "nsfsi_main")
    with tempfile.TemporaryDirectory() as tmp:
        bad = os.path.join(tmp, "ConfigFile")
        open(bad, "w").write("NI = 1.5\n")
        r = subprocess.run([exe], capture_output=True, text=True, cwd=tmp)
    assert r.returncode == 255  # main returns -1 on errorOccurred, as the reference's main does
