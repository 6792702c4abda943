"""GPU parity on seeded random cases (tests/sweep_cases.py, both families): boundary combinations, bodies,
stop criteria, filter schedules and flow parameters beyond the fixed parity cases, each run for a few RK4 steps through the C ABI and by the CPU
oracle (which the CPU sweep pins bit for bit to the reference). Node classification must agree exactly and
every field within 1e-10 of its family's magnitude (test_parity_gpu.field_errors); a flow that goes
non-finite in the oracle must be reported non-finite by the device path. The cases the device setup
refuses with NSF_ERR_GEOMETRY, and only those: an image point whose surrounding box reaches past the last
node (the reference clamps the box index to n and reads out of range there), an image-point cell holding
another body's ghost node (the reference's ghost lookup throws), and a filter node of one body that a later
body made solid. Bodies that reach each other's ghost or filter nodes otherwise run, one after another in
the reference's body order, and must match the oracle like any other case."""
import math
import re

import numpy as np
import pytest

import nsfsi
from oracle import pyoracle as po
from sweep_cases import N_CASES, STEPS, random_case, wide_case
from test_parity_gpu import FIELD_TOL, field_errors


def image_point_past_last_node(o, shape):
    """Whether an image point of the oracle's ghost lists has a surrounding box index (ceil(x / d) + offset,
    as getSurroundingNodesBox forms it, src/SmallVectors.h:108) below 0 or at n or beyond on some axis."""
    geo = o.geometry()
    for ghosts, _, _ in o.bodies():
        for ip in ghosts[:, 6:9]:
            if not np.isfinite(ip).all():  # a ghost node without a normal: no box at all
                return True
            for a in range(3):
                raw = math.ceil(ip[a] / geo[a]) + geo[3 + a]
                if not raw >= 0 or raw >= shape[a]:
                    return True
    return False


def surrounding_box(geo, shape, ip):
    """Lower and upper node index per axis of an image point's cell (ceil(x / d) + offset, kept in 1..n)."""
    lo = []
    for a in range(3):
        nx = min(max(int(math.ceil(ip[a] / geo[a]) + geo[3 + a]), 1), shape[a])
        lo.append(nx - 1)
    return lo


def bodies_refused(o, shape):
    """The two cases of immersed bodies the device setup refuses: an image-point cell holding another body's
    ghost node (the reference's ghost lookup throws there) and a filter node of one body that a later body
    made solid. Bodies that otherwise reach each other's nodes run, in the reference's body order."""
    bodies = o.bodies()
    if len(bodies) < 2:
        return False
    sI, sJ = shape[1] * shape[2], shape[2]
    types = o.node_types()
    ghost_sets = [{int(g[0]) * sI + int(g[1]) * sJ + int(g[2]) for g in ghosts} for ghosts, _, _ in bodies]
    for _, filt, _ in bodies:
        if any(types[int(f)] != 0 for f in filt):
            return True
    geo = o.geometry()
    for q, (ghosts, _, _) in enumerate(bodies):
        for g in ghosts:
            lo = surrounding_box(geo, shape, g[6:9])
            for di in (0, 1):
                for dj in (0, 1):
                    for dk in (0, 1):
                        n = (lo[0] + di) * sI + (lo[1] + dj) * sJ + lo[2] + dk
                        if any(n in gs for r, gs in enumerate(ghost_sets) if r != q) and n not in ghost_sets[q]:
                            return True
    return False


def check_case(text):
    """One case through the oracle and the device path. The oracle marches STEPS steps, or for an end_time
    case until t reaches t_end (Simulation::run's stopping check; the last dt is shortened to land on it)."""
    shape = [int(re.search(r"^N%s = (\d+)$" % c, text, re.M).group(1)) for c in "IJK"]
    end_time = 'stopCriterion = "end_time"' in text
    t_end = float(re.search(r"^t_end = (\S+)$", text, re.M).group(1))
    o = po.Oracle(text)
    try:
        refused = image_point_past_last_node(o, shape) or bodies_refused(o, shape)
        if refused:  # the device path must refuse the case at setup
            with pytest.raises(nsfsi.NsfError) as e:
                nsfsi.Solver(text).close()
            assert e.value.code == 4  # NSF_ERR_GEOMETRY
            return
        types = o.node_types()
        level = 0
        while level < STEPS and not (end_time and o.t >= t_end):
            o.march(1)
            level += 1
        ref = o.fields()
        t_ref = o.t
    finally:
        o.close()
    with nsfsi.Solver(text) as s:
        assert np.array_equal(s.node_types(), types)
        s.march(level)
        try:
            s.sync()
            finite = True
        except nsfsi.NsfError as e:
            assert e.code == 3, e  # NSF_ERR_NONFINITE
            finite = False
        if not np.isfinite(ref).all():
            assert not finite
            return
        assert finite
        t, lv, _ = s.time()
        assert lv == level and abs(t - t_ref) <= 1e-12 * abs(t_ref)
        e = field_errors(s.download(), ref)
        assert (e <= FIELD_TOL).all(), dict(zip(nsfsi.FIELDS, e))


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(N_CASES))
def test_gpu_matches_oracle_random_case(seed):
    check_case(random_case(seed))


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(N_CASES))
def test_gpu_matches_oracle_wide_case(seed):
    """Cylinders along any periodic axis, stagnation starts, filter-interval changes, end_time stops."""
    o = po.Oracle(wide_case(seed))
    dt0 = o.dt
    o.close()
    check_case(wide_case(seed, dt0))
