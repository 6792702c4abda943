"""GPU parity at the benchmark workloads' stated step counts, against fixtures of the reference itself
(tests/golden/make_long_golden.py):

* the 256^3 Taylor-Green workload after 200 RK4 steps (the reference's own fields),
* the 64-member batched-ensemble workload after 200 RK4 steps per member (the reference's own fields; a
  member whose flow becomes non-finite in the reference must become non-finite at the same step here,
  and match at the step before),
* the 16-sphere 256x128x128 workload after 10, 50, 100 and 150 RK4 steps (its flow stays finite until step
  168) against the oracle in its extended-precision image-point mode (why: test_parity_gpu.py).

Each comparison covers a fixed seeded node subsample of all twelve fields at the 1e-10 field tolerance of
the other parity tests (scale: the field family's largest magnitude over the whole grid), plus per-field
checks over every node (sum |f|, sqrt(sum f^2), max |f|) within the bounds that tolerance implies, t, and
the dt history."""
import os

import numpy as np
import pytest

import nsfsi
from test_parity_gpu import DT_TOL, FAMILY, FIELD_TOL, SCALE_FLOOR, TIME_TOL

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def family_scale(checks):
    """Per field: the largest |f| over every node of its family (momenta, velocities share one scale)."""
    mx = checks[:, 2]
    return np.array([max(max(mx[g] for g in FAMILY.get(f, (f,))), SCALE_FLOOR) for f in range(len(mx))])


def full_checks(f):
    return np.stack([np.abs(f).sum(axis=1), np.sqrt((f * f).sum(axis=1)), np.abs(f).max(axis=1)], axis=1)


def assert_matches(fields, idx, ref_sample, ref_checks, what):
    """fields: (12, N) downloaded from the device."""
    scale = family_scale(ref_checks)
    err = np.abs(fields[:, idx] - ref_sample).max(axis=1) / scale
    assert (err <= FIELD_TOL).all(), (what, dict(zip(nsfsi.FIELDS, err)))
    n = fields.shape[1]
    c = full_checks(fields)
    bound = FIELD_TOL * scale[:, None] * np.array([n, np.sqrt(n), 1.0])[None, :]
    assert (np.abs(c - ref_checks) <= bound).all(), (what, np.abs(c - ref_checks) / bound)


@pytest.mark.gpu
def test_tgv256_200_steps_match_reference():
    g = np.load(os.path.join(GOLD, "tgv256_200.npz"))
    with nsfsi.Solver(nsfsi.case_path("tgv256")) as s:
        s.march(200)
        s.sync()
        t, level, dt = s.time()
        assert level == 200
        assert abs(t - float(g["t"])) <= TIME_TOL * float(g["t"])
        assert abs(dt / float(g["dt_next"]) - 1) <= DT_TOL
        h = s.history()
        assert len(h) == 200
        assert float(np.abs(h[:, 1] / g["history"][:, 1] - 1).max()) <= DT_TOL
        assert_matches(s.download(), g["sample_idx"], g["fields"], g["checks"], "tgv256 step 200")


def first_nonfinite_step(h):
    """The first step (1-based) after which a change norm is not finite, or -1."""
    bad = np.flatnonzero(~np.isfinite(h).all(axis=1))
    return int(bad[0]) + 1 if len(bad) else -1


@pytest.mark.gpu
def test_ensemble64_200_steps_match_reference():
    g = np.load(os.path.join(GOLD, "ensemble64_200.npz"))
    steps = int(g["steps"])
    cfgs = nsfsi.ensemble_configs(n=int(g["members"]), steps=steps)
    levels = {m: int(g["level_%d" % m]) for m in range(len(cfgs))}
    diverging = [m for m in levels if int(g["nonfinite_%d" % m]) > 0]
    assert diverging  # the workload holds flows that the reference's own algorithm does not keep finite
    with nsfsi.Ensemble(cfgs) as ens:
        done = 0
        for lv in sorted(set(levels.values())):
            ens.march(lv - done)
            done = lv
            try:
                ens.sync()
            except nsfsi.NsfError as e:
                assert e.code == 3, e  # non-finite members march on, as the reference does
            for m in (m for m in levels if levels[m] == lv):
                mem = ens.member(m)
                t, level, _ = mem.time()
                assert level == lv, (m, level, lv)
                assert abs(t - float(g["t_%d" % m])) <= TIME_TOL * float(g["t_%d" % m]), m
                assert_matches(mem.download(), g["idx_%d" % m], g["fields_%d" % m], g["checks_%d" % m],
                               "member %d step %d" % (m, lv))
        assert done <= steps
        ens.march(steps - done)
        try:
            ens.sync()
        except nsfsi.NsfError as e:
            assert e.code == 3, e
        for m in range(len(cfgs)):
            h = ens.member(m).history()
            rh = g["history_%d" % m]
            assert len(h) == steps
            assert first_nonfinite_step(h[:, 2:]) == int(g["nonfinite_%d" % m]), m
            lv = levels[m]
            assert float(np.abs(h[:lv, 1] / rh[:lv, 1] - 1).max()) <= DT_TOL, m


@pytest.mark.gpu
def test_spheres16_150_steps_match_oracle():
    g = np.load(os.path.join(GOLD, "spheres16_150.npz"))
    idx = g["sample_idx"]
    with nsfsi.Solver(nsfsi.case_path("spheres16")) as s:
        done = 0
        for lv in g["levels"]:
            lv = int(lv)
            s.march(lv - done)
            done = lv
            s.sync()
            t, level, _ = s.time()
            assert level == lv and abs(t - float(g["t_%d" % lv])) <= TIME_TOL * float(g["t_%d" % lv])
            assert_matches(s.download(), idx, g["fields_%d" % lv], g["checks_%d" % lv], "spheres16 step %d" % lv)
        h = s.history()
        assert float(np.abs(h[:, 1] / g["history"][: len(h), 1] - 1).max()) <= DT_TOL
    # the reference's raw double-precision image-point solve stays within its rounding band of the oracle
    for lv in g["levels"]:
        assert (g["raw_vs_exact_%d" % int(lv)] <= 1e-8).all()
