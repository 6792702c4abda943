"""GPU parity on seeded random cases (tests/sweep_cases.py): boundary combinations, bodies and flow
parameters beyond the fixed parity cases, each run for a few RK4 steps through the C ABI and by the CPU
oracle (which the CPU sweep pins bit for bit to the reference). Node classification must agree exactly and
every field within 1e-10 of its family's magnitude (test_parity_gpu.field_errors); a flow that goes
non-finite in the oracle must be reported non-finite by the device path. A case with an image point whose
surrounding box reaches past the last node (the reference clamps the box index to n and reads out of range
there) must be refused at setup with NSF_ERR_GEOMETRY, and only such a case."""
import math
import re

import numpy as np
import pytest

import nsfsi
from oracle import pyoracle as po
from sweep_cases import N_CASES, STEPS, random_case
from test_parity_gpu import FIELD_TOL, field_errors


def image_point_past_last_node(o, shape):
    """Whether an image point of the oracle's ghost lists has a surrounding box index (ceil(x / d) + offset,
    as getSurroundingNodesBox forms it, src/SmallVectors.h:108) below 0 or at n or beyond on some axis."""
    geo = o.geometry()
    for ghosts, _, _ in o.bodies():
        for ip in ghosts[:, 6:9]:
            for a in range(3):
                raw = math.ceil(ip[a] / geo[a]) + geo[3 + a]
                if not raw >= 0 or raw >= shape[a]:
                    return True
    return False


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(N_CASES))
def test_gpu_matches_oracle_random_case(seed):
    text = random_case(seed)
    shape = [int(re.search(r"^N%s = (\d+)$" % c, text, re.M).group(1)) for c in "IJK"]
    o = po.Oracle(text)
    try:
        refused = image_point_past_last_node(o, shape)
        types = o.node_types()
        o.march(STEPS)
        ref = o.fields()
        t_ref = o.t
    finally:
        o.close()
    if refused:
        with pytest.raises(nsfsi.NsfError) as e:
            nsfsi.Solver(text).close()
        assert e.value.code == 4  # NSF_ERR_GEOMETRY
        return
    with nsfsi.Solver(text) as s:
        assert np.array_equal(s.node_types(), types)
        s.march(STEPS)
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
        assert lv == STEPS and abs(t - t_ref) <= 1e-12 * abs(t_ref)
        e = field_errors(s.download(), ref)
        assert (e <= FIELD_TOL).all(), dict(zip(nsfsi.FIELDS, e))
