"""x-slab decomposition of one grid (nsf_slab_group_*): a grid split into 2-4 slabs along i, run as one
group on one device (halo planes exchanged after every stage, the x faces' periodic copies between the end
slabs, dt maxima and change norms reduced over the slabs), must reproduce the single-grid solve node for
node -- all twelve fields and the dt sequence bit for bit, the change norms to rounding."""
import os

import numpy as np
import pytest

import nsfsi
from sweep_cases import random_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = os.path.join(ROOT, "tests", "golden", "cases")


def no_bodies(name):
    text = open(os.path.join(CASES, name + ".cfg")).read()
    return "\n".join(line for line in text.splitlines() if "spheres =" not in line and "cylinders =" not in line)


def compare(text, nslabs, steps):
    with nsfsi.Solver(text) as s:
        s.march(steps)
        s.sync()
        ref = s.download()
        t, lv, dt = s.time()
        h = s.history()
    with nsfsi.SlabGroup(text, nslabs) as g:
        n, first, lps = g.info()
        assert n == nslabs and first[0] == 0
        g.march(steps)
        g.sync()
        got = g.download()
        assert np.array_equal(got, ref), [float(np.abs(a - b).max()) for a, b in zip(got, ref)]
        for p in range(nslabs):
            sl = g.slab(p)
            assert sl.time() == (t, lv, dt)
            hs = sl.history()
            assert np.array_equal(hs[:, :2], h[:, :2])
            assert float(np.abs(hs[:, 2:] - h[:, 2:]).max()) <= 1e-12 * float(np.abs(h[:, 2:]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("nslabs", [2, 3])
def test_taylor_green_periodic_slabs(nslabs):
    compare(open(os.path.join(CASES, "tgv_small.cfg")).read(), nslabs, 25)


@pytest.mark.gpu
@pytest.mark.parametrize("nslabs", [2, 4])
def test_channel_inlet_outlet_slabs(nslabs):
    """Inflow / outflow in x (the end slabs own the faces), periodic y / z, global density-filter steps."""
    compare(no_bodies("sphere_small"), nslabs, 30)


@pytest.mark.gpu
def test_symmetry_faces_slabs():
    compare(no_bodies("cylinder_sym"), 3, 20)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 4, 5, 11, 17])
def test_random_cases_slabs(seed):
    text = random_case(seed)
    if "spheres =" in text or "cylinders =" in text:
        text = "\n".join(line for line in text.splitlines() if "spheres =" not in line and "cylinders =" not in line)
    cfg = nsfsi.config_parse(text)
    if cfg.NI - 2 < 4:
        pytest.skip("too few planes for two slabs")
    compare(text, 2, 8)


@pytest.mark.gpu
def test_taylor_green_256_four_slabs():
    """The benchmark workload split into four slabs, three RK4 steps, against the single-grid solve."""
    compare(open(nsfsi.case_path("tgv256")).read(), 4, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("nslabs", [2, 3])
def test_nccl_path_on_one_gpu(nslabs):
    """A group created for several processes, here one (world = 1), with every plane moved by NCCL (send and
    receive to itself) and the partials all-gathered: the same fields, t and dt as the single-grid solve."""
    text = open(os.path.join(CASES, "tgv_small.cfg")).read()
    steps = 12
    with nsfsi.Solver(text) as s:
        s.march(steps)
        s.sync()
        ref = s.download()
        t, lv, dt = s.time()
    nid = nsfsi.slab_nccl_id()
    with nsfsi.SlabGroup(text, nslabs, 0, rank=0, world=1, nccl_id=nid, flags=nsfsi.SLAB_NCCL_ALL) as g:
        n, first, lps = g.info()
        assert n == nslabs
        g.march(steps)
        g.sync()
        got = g.download()
        assert np.array_equal(got, ref), [float(np.abs(a - b).max()) for a, b in zip(got, ref)]
        for p in range(nslabs):
            assert g.slab(p).time() == (t, lv, dt)
