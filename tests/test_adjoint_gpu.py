"""Discrete adjoint (nsf_adj_configure / nsf_adj_forward / nsf_adj_backward): the gradient of the
time-averaged x-force on the immersed sphere with respect to the level-0 conserved field and the x-inlet's
velocity-profile factor, checked against central finite differences of the forward run along seeded random
directions, plus the properties of the checkpointing schedule (the result does not depend on the number of
snapshots; a second backward run after one forward run gives the same gradient)."""
import numpy as np
import pytest

import nsfsi
from oracle import pyoracle as po

FD_STEP = 1e-6   # finite-difference step along each direction
FD_TOL = 1e-6    # |adjoint - central difference| relative to the derivative (see fd_error)


def solver(case, steps=None):
    c = nsfsi.config_load(nsfsi.case_path(case))
    if steps is not None:
        c.stop_time_level = steps
    return nsfsi.Solver(c)


def fd_check(s, u0, gi, gu, du, di, h):
    """(adjoint directional derivative, central difference, size of the derivative's terms) along (du, di).

    The directional derivative of a random direction is a sum of about a million terms of random sign; the
    last value, the 2-norm of those terms, is the derivative's expected size, which the sum itself can fall
    far below when the terms happen to cancel (a seeded direction is not chosen to avoid that)."""
    ad = (0.0 if du is None else float((gu * du).sum())) + (0.0 if di is None else float((gi * di).sum()))
    terms = np.sqrt((0.0 if du is None else float(((gu * du) ** 2).sum()))
                    + (0.0 if di is None else float(((gi * di) ** 2).sum())))
    up = None if du is None else u0 + h * du
    um = None if du is None else u0 - h * du
    ip = None if di is None else 1 + h * di
    im = None if di is None else 1 - h * di
    fd = (s.adj_forward(up, ip) - s.adj_forward(um, im)) / (2 * h)
    return ad, fd, terms


def fd_error(ad, fd, terms):
    """|adjoint - central difference| relative to the larger of |derivative| and its terms' 2-norm."""
    return abs(fd - ad) / max(abs(ad), terms)


def seeded_directions(s, u0, count, seed):
    """count directions: the first three quarters perturb the level-0 field (each variable scaled by its
    largest magnitude) together with the inflow profile, the rest the inflow profile alone (amplitude 10)."""
    rng = np.random.default_rng(seed)
    c = s.cfg
    scale = np.maximum(np.abs(u0).max(axis=1), 1e-3)[:, None]
    out = []
    for d in range(count):
        di = rng.standard_normal((int(c.NJ), int(c.NK)))
        if d < 3 * count // 4:
            out.append((rng.standard_normal(u0.shape) * scale, di))
        else:
            out.append((None, 10 * di))
    return out


@pytest.mark.gpu
def test_adjoint_matches_finite_differences_64():
    """64^3 channel with a sphere, 200 RK4 steps, J averaged over the last 50, 20 snapshots."""
    with solver("adj64") as s:
        u0 = s.download(range(5))
        s.adj_configure(50, 20)
        s.adj_forward()
        gi, gu = s.adj_backward()
        assert np.isfinite(gu).all() and np.isfinite(gi).all()
        assert np.abs(gi).max() > 0 and np.abs(gu).max() > 0
        worst = 0.0
        for du, di in seeded_directions(s, u0, 16, seed=2024):
            ad, fd, terms = fd_check(s, u0, gi, gu, du, di, FD_STEP)
            rel = fd_error(ad, fd, terms)
            worst = max(worst, rel)
            assert rel <= FD_TOL, (ad, fd, terms, rel)
        print("worst relative error over 16 directions: %.2e" % worst)


@pytest.mark.gpu
def test_adjoint_short_run_tight():
    """32^3, 12 steps (no density-filter step is reached; the near-body filter runs every step), J over
    the last 4 steps, 3 snapshots so that the schedule recurses: the gradient matches the central
    difference at h = 1e-5 to 1e-8 in every direction, including single-node perturbations at the nodes of
    largest sensitivity, up to the central difference's own rounding floor (16 eps |J| / h: a single node
    moves J by little more than its last bits)."""
    h = 1e-5
    with solver("adj32", steps=12) as s:
        u0 = s.download(range(5))
        s.adj_configure(4, 3)
        s.adj_tape_limit(0)  # checkpoints, so that the schedule recurses
        J = s.adj_forward()
        assert s.adj_tape_bytes() == 0
        gi, gu = s.adj_backward()
        floor = 16 * np.finfo(float).eps * abs(J) / h
        dirs = seeded_directions(s, u0, 4, seed=7)
        # single nodes: the largest-gradient node of each variable
        for f in range(5):
            du = np.zeros_like(u0)
            n = int(np.abs(gu[f]).argmax())
            du[f, n] = max(abs(u0[f, n]), 1e-2)
            dirs.append((du, None))
        for du, di in dirs:
            ad, fd, terms = fd_check(s, u0, gi, gu, du, di, h)
            assert abs(fd - ad) <= 1e-8 * max(abs(ad), terms) + floor, (ad, fd, terms, floor)


@pytest.mark.gpu
def test_adjoint_schedule_does_not_change_the_gradient():
    """The recomputation is deterministic and the adjoint kernels run in the same order whatever the
    checkpointing schedule, so the gradient is bit-identical for 1, 4 and 40 snapshots (40 > steps: no
    recomputation) and for the tape (every step's snapshot set recorded by the forward run, no
    recomputation at all), and a second backward run after one forward run repeats it."""
    ref = None
    set_bytes = None
    for snaps in ("tape", 40, 4, 1, "segments"):
        with solver("adj32", steps=30) as s:
            s.adj_configure(10, {"tape": 20, "segments": 3}.get(snaps, snaps))
            if snaps == "segments":  # 3 + 1 slots: segments of 8 steps (the last of 6), a ring of two
                s.adj_tape_limit(16 * set_bytes)
            elif snaps != "tape":
                s.adj_tape_limit(0)
            s.adj_forward()
            assert (s.adj_tape_bytes() > 0) == (snaps == "tape"), snaps
            if snaps == "tape":
                set_bytes = s.adj_tape_bytes() // 30
            assert s.adj_segment_tape() == ((16 * set_bytes, 8) if snaps == "segments" else (0, 0)), snaps
            gi, gu = s.adj_backward()
            gi2, gu2 = s.adj_backward()
            assert np.array_equal(gi, gi2) and np.array_equal(gu, gu2)
            if ref is None:
                ref = (gi, gu)
            else:
                assert np.array_equal(gi, ref[0]) and np.array_equal(gu, ref[1]), snaps


@pytest.mark.gpu
def test_adjoint_tape_limit():
    """The tape is recorded when every step's snapshot set fits the limit, and not when it does not; a
    limit below a recorded tape releases it. Below the whole run's tape, the forward run stores a state
    every ceil(12 / (3 + 1)) = 3 steps and leaves a segment tape of two segments' sets (or one) for the
    backward run; with no segment's sets under the limit it checkpoints binomially. Same gradient in every
    mode."""
    with solver("adj32", steps=12) as s:
        s.adj_configure(4, 3)
        s.adj_forward()
        full = s.adj_tape_bytes()
        assert full > 0 and full % 12 == 0 and s.adj_segment_tape() == (0, 0)
        gi, gu = s.adj_backward()
        s.adj_tape_limit(full - 1)
        assert s.adj_tape_bytes() == 0
        s.adj_forward()
        assert s.adj_tape_bytes() == 0
        assert s.adj_segment_tape() == (full // 2, 3)
        gi2, gu2 = s.adj_backward()
        assert np.array_equal(gi, gi2) and np.array_equal(gu, gu2)
        gi2, gu2 = s.adj_backward()  # a second backward run from the same checkpoints
        assert np.array_equal(gi, gi2) and np.array_equal(gu, gu2)
        s.adj_tape_limit(full // 4)  # one segment's sets
        s.adj_forward()
        assert s.adj_segment_tape() == (full // 4, 3)
        gi2, gu2 = s.adj_backward()
        assert np.array_equal(gi, gi2) and np.array_equal(gu, gu2)
        s.adj_tape_limit(full // 4 - 1)  # releases the segment tape: binomial checkpointing
        assert s.adj_segment_tape() == (0, 0)
        s.adj_forward()
        assert s.adj_tape_bytes() == 0 and s.adj_segment_tape() == (0, 0)
        gi2, gu2 = s.adj_backward()
        assert np.array_equal(gi, gi2) and np.array_equal(gu, gu2)
        s.adj_tape_limit(full)
        s.adj_forward()
        assert s.adj_tape_bytes() == full
        gi3, gu3 = s.adj_backward()
        assert np.array_equal(gi, gi3) and np.array_equal(gu, gu3)


@pytest.mark.gpu
def test_adjoint_dt_is_frozen_from_the_plain_run():
    """The frozen dt sequence is the plain solver's dt history for the same run."""
    with solver("adj32", steps=30) as s:
        s.adj_configure(10, 4)
        s.adj_forward()
        dts = s.adj_dt()
    with solver("adj32", steps=30) as p:
        p.march(30)
        p.sync()
        hist = p.history()
    assert np.array_equal(dts, hist[:, 1])


@pytest.mark.gpu
def test_adjoint_rejects_unsupported_cases():
    """An end-time stop criterion (no fixed step count) and symmetry y faces are refused."""
    c = nsfsi.config_load(nsfsi.case_path("adj32"))
    c.stop_criterion = 1
    with nsfsi.Solver(c) as s:
        with pytest.raises(nsfsi.NsfError):
            s.adj_configure(10, 4)
    c = nsfsi.config_load(nsfsi.case_path("adj32"))
    c.bc[1][0] = c.bc[1][1] = nsfsi.BC["symmetry"]
    with nsfsi.Solver(c) as s:
        with pytest.raises(nsfsi.NsfError):
            s.adj_configure(10, 4)


@pytest.mark.gpu
def test_adjoint_matches_dual_number_oracle_32():
    """32^3 channel with a sphere, 200 steps, J over the last 50: the GPU objective and adjoint gradient
    against the CPU oracle run with dual numbers (forward-mode derivatives, no truncation error) from the
    same level-0 field with the same frozen dt sequence, along two seeded joint directions (level-0 field and
    inflow profile)."""
    cfg_text = open(nsfsi.case_path("adj32")).read()
    with solver("adj32") as s:
        u0 = s.download(range(5))
        s.adj_configure(50, 20)
        J = s.adj_forward()
        gi, gu = s.adj_backward()
        dts = s.adj_dt()
        c = s.cfg
        ones = np.ones((int(c.NJ), int(c.NK)))
        rng = np.random.default_rng(32)
        scale = np.maximum(np.abs(u0).max(axis=1), 1e-3)[:, None]
        for d in range(2):
            du = rng.standard_normal(u0.shape) * scale
            di = rng.standard_normal(ones.shape)
            Jo, dJo = po.dual_objective(cfg_text, dts, 50, u0=u0, du0=du, inflow=ones, dinflow=di)
            ad = float((gu * du).sum() + (gi * di).sum())
            assert abs(Jo - J) <= 1e-10 * abs(J), (J, Jo)
            assert abs(ad - dJo) <= 1e-8 * abs(dJo), (ad, dJo)


@pytest.mark.gpu
def test_adjoint_all_periodic_box():
    """A sphere in a fully periodic box (no inlet or outlet: the recomputation of a step outside the
    averaging window stops before stage 4 entirely): gradient against central differences, h = 1e-5."""
    text = open(nsfsi.case_path("adj32")).read()
    text = text.replace('bc_x_min = "inlet";', 'bc_x_min = "periodic";').replace('bc_x_max = "outlet";',
                                                                          'bc_x_max = "periodic";')
    text = text.replace("stopTimeLevel = 200", "stopTimeLevel = 40")
    assert 'bc_x_min = "periodic"' in text and "stopTimeLevel = 40" in text
    with nsfsi.Solver(text) as s:
        u0 = s.download(range(5))
        s.adj_configure(10, 4)
        J = s.adj_forward()
        gi, gu = s.adj_backward()
        assert np.abs(gi).max() == 0.0  # no inlet: the profile factor does not enter
        h = 1e-5
        floor = 16 * np.finfo(float).eps * abs(J) / h
        for du, _ in seeded_directions(s, u0, 4, seed=9)[:3]:
            ad, fd, terms = fd_check(s, u0, gi, gu, du, None, h)
            assert abs(fd - ad) <= 1e-7 * max(abs(ad), terms) + floor, (ad, fd, terms)


@pytest.mark.gpu
def test_adjoint_body_near_the_inlet():
    """The sphere of adj32 moved next to the inlet: its filter and ghost nodes reach the planes the inlet's
    adjoint reads, so the adjoint boundary kernel runs its body and edge phases as one chain and the inlet
    planes come from the stage snapshots. 10 steps, J over the last 4: the gradient matches the central
    difference at h = 1e-5 to 1e-8."""
    h = 1e-5
    text = open(nsfsi.case_path("adj32")).read().replace("spheres = ( (0.4, 0.5, 0.5, 0.1) );",
                                                          "spheres = ( (0.21, 0.5, 0.5, 0.1) );")
    c = nsfsi.config_parse(text)
    c.stop_time_level = 10
    with nsfsi.Solver(c) as s:
        u0 = s.download(range(5))
        s.adj_configure(4, 3)
        J = s.adj_forward()
        gi, gu = s.adj_backward()
        floor = 16 * np.finfo(float).eps * abs(J) / h
        for du, di in seeded_directions(s, u0, 4, seed=11):
            ad, fd, terms = fd_check(s, u0, gi, gu, du, di, h)
            assert abs(fd - ad) <= 1e-8 * max(abs(ad), terms) + floor, (ad, fd, terms, floor)
