"""The stage kernel's bounded waits: when a wait runs out, the kernel gives up cleanly and the host is told.

The test switch of nsf_debug_wait_limit makes the kernel's producer issue none of its epilogue loads,
so the column warps' waits for them can never be satisfied, and shortens every wait to a few thousand
polls. Nothing faults or hangs: each wait ends after its poll limit, raises the block's abort flag
(which ends the other waits), and the producer waits, bounded, for the copies it did issue. The step's
results are invalid, nsf_sync reports NSF_ERR_TIMEOUT, and a fresh solver on the same device then runs
normally and matches the reference."""
import os

import numpy as np
import pytest

import nsfsi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASE = os.path.join(ROOT, "tests", "golden", "cases", "sphere_small.cfg")
TIMEOUT = 5  # NSF_ERR_TIMEOUT


@pytest.mark.gpu
@pytest.mark.parametrize("steps", [1, 3])
def test_withheld_loads_time_out_and_are_reported(steps):
    s = nsfsi.Solver(CASE)
    try:
        s.debug_wait_limit(polls=4096, withhold_epilogue=True)
        s.march(steps)
        with pytest.raises(nsfsi.NsfError) as e:
            s.sync()
        assert e.value.code == TIMEOUT, e.value
        # the flag is sticky: later calls keep reporting it
        with pytest.raises(nsfsi.NsfError) as e:
            s.sync()
        assert e.value.code == TIMEOUT
    finally:
        s.close()
    # a fresh solver on the same device is unaffected and matches the reference's own fields
    g = np.load(os.path.join(ROOT, "tests", "golden", "sphere_small.npz"))
    with nsfsi.Solver(CASE) as s2:
        d = int(g["dumps"][0])
        s2.march(d)
        s2.sync()
        got, ref = s2.download(), g["fields_%d" % d]
        err = max(float(np.abs(got[f] - ref[f]).max() / max(np.abs(ref[f]).max(), 1e-6)) for f in range(12))
        assert err <= 1e-10, err

