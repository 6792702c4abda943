"""Snapshot downloads that overlap the march (nsf_download_async) and the snapshot writer of the C++ host layer.

* A download of conserved fields only (a direct copy from the field buffers) equals the same fields through the
  snapshot kernel.
* An asynchronous snapshot holds, bit for bit, what a synchronous nsf_download returns at the same time level,
  for any field subset, at level 0 (stored initial values of solid inactive nodes) and later, with more
  downloads in flight than staging buffers and steps marched while they travel.
* The drop-in driver, saving every field at every step, writes each out.vtk.N with exactly the bytes that the
  synchronous writer (OutputManager::writeVtk from Mesh mirrors) writes for the fields downloaded at that step.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

import nsfsi
from test_host_cpu import build_check

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "3d-ns-fsi_b200")
CASE = os.path.join(ROOT, "tests", "golden", "cases", "sphere_small.cfg")

ERR_ARG, ERR_STATE = 6, 7


def tgv(n, steps):
    """The periodic Taylor-Green case of tgv128.cfg on an n^3 grid, filtered every 5 steps."""
    text = open(nsfsi.case_path("tgv128")).read()
    for ax in "IJK":
        text = text.replace("N%s = 128" % ax, "N%s = %d" % (ax, n))
    text = text.replace("stopTimeLevel = 200", "stopTimeLevel = %d" % steps)
    text = text.replace("filterIntervals = [50, 200, 1000]", "filterIntervals = [5, 5, 5]")
    return nsfsi.config_parse(text)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sphere_small", "tgv48"])
def test_async_snapshots_equal_sync_downloads(case):
    cfg = nsfsi.config_load(CASE) if case == "sphere_small" else tgv(48, 40)
    # (level, fields) of each snapshot; two at level 7 back to back; five in flight over two staging buffers
    plan = [(0, range(12)), (3, [0, 4, 8]), (7, range(5)), (7, range(5, 12)), (12, [1, 2, 3, 9])]
    with nsfsi.Solver(cfg) as a, nsfsi.Solver(cfg) as b:
        snaps, want, lv = [], [], 0
        for level, fields in plan:
            a.march(level - lv)
            b.march(level - lv)
            lv = level
            snaps.append(a.download_async(fields))
            want.append(b.download(fields))
        a.march(5)  # later steps run while the copies land
        for s, w in zip(snaps, want):
            got = s.wait()
            assert got.shape == w.shape
            np.testing.assert_array_equal(got, w)
            assert s.done()
        # the march after the snapshots is unaffected
        b.march(5)
        np.testing.assert_array_equal(a.download(), b.download())


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sphere_small", "tgv40"])
def test_conserved_downloads_equal_snapshot_kernel(case):
    """A download of conserved fields only is a strided copy straight from the current buffers (on a 40^3
    grid the device rows are padded to 48 doubles); it equals, bit for bit, the same fields of a download
    that goes through the snapshot kernel, for every subset packing, at level 0 and after steps whose buffer
    roles rotate."""
    cfg = nsfsi.config_load(CASE) if case == "sphere_small" else tgv(40, 40)
    with nsfsi.Solver(cfg) as s:
        for steps in (0, 1, 2, 5):
            s.march(steps)
            full = s.download()  # all twelve fields: the snapshot kernel
            for fields in ([0], [4], [0, 4], [1, 2, 3], [0, 1, 2, 3, 4], [2, 4]):
                np.testing.assert_array_equal(s.download(fields), full[fields])


@pytest.mark.gpu
def test_async_download_refusals():
    cfg = nsfsi.config_load(CASE)
    L = nsfsi.lib()
    with nsfsi.Solver(cfg) as s:
        t = ctypes.c_uint64()
        pageable = np.empty(s.N)
        assert L.nsf_download_async(s.h, 1, nsfsi._dp(pageable), ctypes.byref(t)) == ERR_ARG
        assert "page-locked" in L.nsf_last_error(s.h).decode()
        snap = s.download_async([0])
        assert L.nsf_download_async(s.h, 0, snap._ptr(), ctypes.byref(t)) == ERR_ARG
        assert L.nsf_download_wait(s.h, snap.ticket + 1) == ERR_ARG
        assert L.nsf_download_wait(s.h, 0) == ERR_ARG
        np.testing.assert_array_equal(snap.wait(), s.download([0]))
    with nsfsi.Ensemble([cfg, cfg]) as ens:
        m = ctypes.c_void_p()
        assert L.nsf_ensemble_member(ens.h, 0, ctypes.byref(m)) == 0
        buf = ctypes.c_void_p()
        assert L.nsf_host_alloc(8 * s.N, ctypes.byref(buf)) == 0
        try:
            p = ctypes.cast(buf, ctypes.POINTER(ctypes.c_double))
            assert L.nsf_download_async(m, 1, p, ctypes.byref(t)) == ERR_STATE
        finally:
            assert L.nsf_host_free(buf) == 0


@pytest.mark.gpu
def test_driver_snapshots_match_the_synchronous_writer():
    text = open(CASE).read()
    for key in ("Momentum", "Energy", "Viscosity", "ThermalCond", "IC", "Final", "Intervals"):
        assert "save%s = false" % key in text
        text = text.replace("save%s = false" % key, "save%s = true" % key)
    text = text.replace("savePeriod = 5.", "savePeriod = 0.")
    cfg = nsfsi.config_parse(text)
    assert cfg.save_intervals and cfg.save_ic and cfg.save_final and cfg.save_period == 0
    with tempfile.TemporaryDirectory() as tmp:
        open(os.path.join(tmp, "ConfigFile"), "w").write(text)
        r = subprocess.run([os.path.join(PKG, "bin", "nsfsi_main")], capture_output=True, text=True, cwd=tmp,
                           timeout=300)
        assert r.returncode == 0, r.stderr
        # the same run through the synchronous path: IC, every step (savePeriod 0 saves each), final
        states = []
        with nsfsi.Solver(cfg) as s:
            t, lv, dt = s.time()
            states.append((t, s.download()))
            while lv < cfg.stop_time_level:
                s.march(1)
                t, lv, dt = s.time()
                states.append((t, s.download()))
            states.append((t, s.download()))
        outs = sorted(int(x.split(".")[-1]) for x in os.listdir(os.path.join(tmp, "output")) if x.startswith("out.vtk."))
        assert outs == list(range(len(states)))
        times = [float(x) for x in open(os.path.join(tmp, "output", "times.dat")).read().split()]
        assert len(times) == len(states)
        exe = build_check(tmp)
        cfgfile = os.path.join(tmp, "ConfigFile")
        for q, (t, fields) in enumerate(states):
            fb = os.path.join(tmp, "fields.bin")
            np.ascontiguousarray(fields).tofile(fb)
            ref = os.path.join(tmp, "sync.vtk")
            subprocess.run([exe, cfgfile, fb, repr(t), ref, "mirrors"], check=True)
            assert open(os.path.join(tmp, "output", "out.vtk.%d" % q), "rb").read() == open(ref, "rb").read(), q
