"""The drop-in driver (bin/nsfsi_main: ConfigSettings -> Simulation::run over the C ABI) on a B200 against
the output the reference's own OutputManager wrote for the same case (tests/golden/vtk_sphere_small)."""
import gzip
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "3d-ns-fsi_b200")
GOLD = os.path.join(ROOT, "tests", "golden", "vtk_sphere_small")


def numbers(text):
    """(non-numeric lines, numeric values) of a text file."""
    words, vals = [], []
    for line in text.splitlines():
        toks = line.split()
        try:
            vals.extend(float(x) for x in toks)
        except ValueError:
            words.append(line)
    return words, np.array(vals)


@pytest.mark.gpu
def test_driver_program_writes_the_reference_output():
    cfg = open(os.path.join(ROOT, "tests/golden/cases/sphere_small.cfg")).read()
    assert "saveFinal = false" in cfg
    cfg = cfg.replace("saveFinal = false", "saveFinal = true")
    with tempfile.TemporaryDirectory() as tmp:
        open(os.path.join(tmp, "ConfigFile"), "w").write(cfg)
        r = subprocess.run([os.path.join(PKG, "bin", "nsfsi_main")], capture_output=True, text=True, cwd=tmp,
                           timeout=300)
        assert r.returncode == 0, r.stderr
        assert "Time level: n = 30" in r.stdout
        for name in sorted(os.listdir(GOLD)):
            ref = gzip.open(os.path.join(GOLD, name)).read().decode()
            mine = open(os.path.join(tmp, "output", name[:-3])).read()
            wr, vr = numbers(ref)
            wm, vm = numbers(mine)
            assert wm == wr, name
            assert vm.shape == vr.shape, name
            # values are printed with 6 significant digits; the fields agree to ~1e-12, so a printed value
            # can differ from the reference's by at most one unit in its last digit, and a value the
            # reference holds as exactly zero (a symmetric velocity component) can carry ~1e-18 round-off
            tol = 1.0001e-5 * np.abs(vr) + 1e-12
            bad = np.abs(vm - vr) > tol
            assert not bad.any(), (name, vm[bad][:5], vr[bad][:5])
