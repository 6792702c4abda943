"""Pins the CPU oracle to the reference solver on seeded random cases (tests/sweep_cases.py: the random_case,
wide_case and shipped_case families), beyond the fixed golden cases: the unmodified reference
(oracle/_ref/ref_runner, built from the reference sources by oracle/Makefile.ref) and the oracle run a few
RK4 steps of each case, and node classification, ghost and filter lists, the dt and norm histories and all
twelve fields must agree bit for bit; where the reference stops on one of its own exceptions the oracle
must stop too. Skipped where the reference build is absent.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import pyoracle as po
from sweep_cases import N_CASES, STEPS, ensemble_member_text, random_case, shipped_case, wide_case


def compare(text, level=STEPS):
    """Run the reference build and the oracle on one case file; level: the step to compare at ("final": where
    the run stops, for an end_time case)."""
    o = po.Oracle(text)
    finite = all(np.isfinite(g[:, 6:9]).all() for g, _, _ in o.bodies())
    o.close()
    if not finite:  # a ghost node on a body's axis or centre has no normal: its image point is NaN, and
        # the reference's box search then converts NaN to an index (undefined behaviour)
        pytest.skip("image point not finite")
    with tempfile.TemporaryDirectory(prefix="nsf_sweep_") as tmp:
        cfg = os.path.join(tmp, "case.cfg")
        with open(cfg, "w") as f:
            f.write(text)
        out = os.path.join(tmp, "ref")
        os.makedirs(out)
        try:
            po.run_reference(cfg, [STEPS if level == "final" else level], outdir=out, final=level == "final")
        except subprocess.CalledProcessError:
            # the reference stopped on one of its own exceptions (for instance a solid node around an image
            # point, Boundary.cpp:723-724): the oracle must stop there too
            o = po.Oracle(text)
            try:
                with pytest.raises(RuntimeError):
                    o.march(STEPS)
            finally:
                o.close()
            return
        ref = po.read_ref_setup(out)
        fin = po.read_ref_fields(out, level)
        hist = po.read_ref_history(out)
    o = po.Oracle(text)
    try:
        assert np.array_equal(o.geometry(), ref["geometry"])
        assert np.array_equal(o.node_types(), ref["types"])
        assert o.dt == ref["dt0"]
        bodies = o.bodies()
        assert len(bodies) == len(ref["bodies"])
        for (gh, fl, _), (rg, rf) in zip(bodies, ref["bodies"]):
            assert np.array_equal(gh, rg) and np.array_equal(fl, rf)
        o.march(fin["level"])
        assert o.t == fin["t"]
        f = o.fields()
        # a drawn flow can go non-finite in the reference's own algorithm (it prints and marches on, as the
        # oracle does): the NaN pattern must then agree as well
        assert np.array_equal(f, fin["fields"], equal_nan=True), [float(np.nanmax(np.abs(a - b)))
                                                                  for a, b in zip(f, fin["fields"])]
        h = o.history()
        assert np.array_equal(h[:, :2], hist[: len(h), :2], equal_nan=True)
        assert np.array_equal(h[:, 2:], hist[: len(h), 3:], equal_nan=True)
    finally:
        o.close()


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref/ref_runner absent")
@pytest.mark.parametrize("seed", range(N_CASES))
def test_oracle_matches_reference_random_case(seed):
    compare(random_case(seed))


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref/ref_runner absent")
@pytest.mark.parametrize("seed", range(N_CASES))
def test_oracle_matches_reference_wide_case(seed):
    """Cylinders along any periodic axis, stagnation starts, filter-interval changes, end_time stops."""
    o = po.Oracle(wide_case(seed))
    dt0 = o.dt
    o.close()
    compare(wide_case(seed, dt0), level="final")


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref/ref_runner absent")
@pytest.mark.parametrize("seed", range(N_CASES))
def test_oracle_matches_reference_shipped_case(seed):
    """The reference's default case (Solver::initialize unchanged) with seeded settings."""
    o = po.Oracle(shipped_case(seed))
    dt0 = o.dt
    o.close()
    compare(shipped_case(seed, dt0), level="final")


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref/ref_runner absent")
@pytest.mark.parametrize("member", range(0, 64, 8))
def test_oracle_matches_reference_ensemble_member(member):
    """Members of the batched-ensemble workload (the bench's 64 flows), three RK4 steps each."""
    import nsfsi
    c = nsfsi.ensemble_configs(n=64, steps=3)[member]
    compare(ensemble_member_text(c, 3), level=3)


@pytest.mark.slow
@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref/ref_runner absent")
def test_oracle_matches_reference_tgv256_one_step():
    """The benchmark workload at full size (Taylor-Green 256^3, 16.8 M nodes): one RK4 step."""
    import nsfsi
    text = open(nsfsi.case_path("tgv256")).read()
    compare(text, level=1)



def _smallest(name, n, periodic_y=True):
    text = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "3d-ns-fsi_b200", "cases",
                             name + ".cfg")).read()
    for ax in "IJK":
        text = text.replace("N%s = 48" % ax, "N%s = %d" % (ax, n)).replace("N%s = 128" % ax, "N%s = %d" % (ax, n))
    text = text.replace("  spheres = ( (0.4, 0.5, 0.5, 0.1) );\n", "")
    if not periodic_y:
        text = text.replace('bc_y_min = "periodic"', 'bc_y_min = "symmetry"').replace('bc_y_max = "periodic"',
                                                                                       'bc_y_max = "symmetry"')
    return text


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref/ref_runner absent")
@pytest.mark.parametrize("name,n,periodic_y", [("tgv128", 3, True), ("tgv128", 4, True), ("sphere48", 3, True),
                                               ("sphere48", 4, False), ("sphere48", 5, False)])
def test_oracle_matches_reference_on_the_smallest_grids(name, n, periodic_y):
    """The smallest grids each boundary type allows (3 nodes per periodic or inlet/outlet axis, 4 per
    symmetry axis): a 3^3 and 4^3 periodic Taylor-Green box and body-free channels with periodic or
    symmetry y faces match the reference bit for bit."""
    compare(_smallest(name, n, periodic_y))
