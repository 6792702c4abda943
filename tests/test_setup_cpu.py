"""Host-side setup of the product (no GPU): node classification, ghost lists with body-intercept and
image points, filter lists and the initial dt must be bit-exact with the reference (golden fixtures made
by the reference itself, tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import nsfsi
from nsfsi import Solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
CASES = {
    "sphere_small": "tests/golden/cases/sphere_small.cfg",
    "tgv_small": "tests/golden/cases/tgv_small.cfg",
    "two_spheres": "tests/golden/cases/two_spheres.cfg",
    "cylinder_sym": "tests/golden/cases/cylinder_sym.cfg",
    "shipped_small": "tests/golden/cases/shipped_small.cfg",
    "sphere48": "3d-ns-fsi_b200/cases/sphere48.cfg",
    "spheres16": "3d-ns-fsi_b200/cases/spheres16.cfg",
}


@pytest.mark.parametrize("name", list(CASES))
def test_classification_bit_exact(name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    s = Solver(os.path.join(ROOT, CASES[name]), device=-1)
    try:
        assert np.array_equal(s.node_types(), g["types"])
        bodies = s.bodies()
        assert len(bodies) == int(g["nbodies"])
        for b, (gh, fl, closure) in enumerate(bodies):
            assert closure == 0
            assert np.array_equal(gh, g["ghosts_%d" % b])  # same order, same doubles
            assert np.array_equal(fl, g["filter_%d" % b])
    finally:
        s.close()


def test_tgv256_has_no_bodies_and_all_interior():
    s = Solver(nsfsi.case_path("tgv256"), device=-1)
    t = s.node_types().reshape(256, 256, 256)
    assert (t[1:-1, 1:-1, 1:-1] == 0).all()
    assert (t[0] == 2).all() and (t[:, 0] == 2).all() and (t[:, :, 0] == 2).all()
    assert s.bodies() == []
    s.close()


def test_host_only_handle_refuses_to_march():
    s = Solver(nsfsi.case_path("sphere48"), device=-1)
    with pytest.raises(nsfsi.NsfError) as e:
        s.march(1)
    assert e.value.code == 7
    s.close()


def test_body_too_close_to_face_is_rejected():
    txt = open(nsfsi.case_path("sphere48")).read().replace("(0.4, 0.5, 0.5, 0.1)", "(0.4, 0.08, 0.5, 0.1)")
    with pytest.raises(nsfsi.NsfError) as e:
        Solver(txt, device=-1)
    assert e.value.code == 4


def test_ensemble_workload_members_are_valid_cases():
    """The 64 seeded ensemble members (5 grid shapes, Mach, Re, sphere size) all pass the host setup."""
    cfgs = nsfsi.ensemble_configs()
    shapes = set()
    for c in cfgs:
        s = Solver(c, device=-1)
        assert len(s.bodies()) == 1 and len(s.bodies()[0][0]) > 0
        shapes.add((c.NI, c.NJ, c.NK))
        s.close()
    assert len(cfgs) == 64 and shapes == set(nsfsi.ENSEMBLE_SHAPES)


def test_ensemble_needs_a_device():
    with pytest.raises(nsfsi.NsfError):
        nsfsi.Ensemble(nsfsi.ensemble_configs(n=2))


def test_interacting_bodies_run_and_are_flagged():
    """Two spheres whose filter layers overlap (48 nodes filtered by both) run, flagged as interacting;
    the well-separated pair does not interact."""
    with Solver(os.path.join(ROOT, "tests", "golden", "cases", "close_spheres.cfg"), device=-1) as s:
        assert s.bodies_interact()
        (g1, f1, _), (g2, f2, _) = s.bodies()
        assert len(set(f1.tolist()) & set(f2.tolist())) > 0
    with Solver(os.path.join(ROOT, "tests", "golden", "cases", "two_spheres.cfg"), device=-1) as s:
        assert not s.bodies_interact()


def test_filter_node_inside_a_later_body_is_refused():
    """A gap so small that a later sphere makes one of the first sphere's filter nodes solid."""
    text = open(os.path.join(ROOT, "tests", "golden", "cases", "close_spheres.cfg")).read()
    text = text.replace("(1.17, 0.55, 0.5, 0.2)", "(1.11, 0.55, 0.5, 0.2)")
    with pytest.raises(nsfsi.NsfError) as e:
        Solver(text, device=-1)
    assert e.value.code == 4 and "inside another" in str(e.value)


def _grid_case(name, n):
    text = open(nsfsi.case_path(name)).read()
    for ax in "IJK":
        text = text.replace("N%s = 48" % ax, "N%s = %d" % (ax, n)).replace("N%s = 128" % ax, "N%s = %d" % (ax, n))
    return nsfsi.config_parse(text)


@pytest.mark.parametrize("n", [0, 1, 2])
def test_grids_below_the_minimum_node_count_are_refused(n):
    """An axis with fewer nodes than its boundary type needs (3; 4 for symmetry faces, the reference
    ConfigFile's minimum counts) is a config error at setup, on a host-only handle, with no device work."""
    import ctypes
    L = nsfsi.lib()
    for name in ("tgv128", "sphere48"):
        c = _grid_case(name, n)
        h = ctypes.c_void_p()
        assert L.nsf_create(ctypes.byref(c), -1, ctypes.byref(h)) == 0
        try:
            assert L.nsf_initialize(h) == 1
            assert b"too few nodes" in L.nsf_last_error(h)
        finally:
            L.nsf_destroy(h)


def test_smallest_periodic_grid_sets_up():
    """Three nodes per periodic axis is the smallest grid the setup accepts: one interior fluid node, every
    face node a periodic boundary node (the reference's fluid ghost type)."""
    import ctypes
    L = nsfsi.lib()
    c = _grid_case("tgv128", 3)
    h = ctypes.c_void_p()
    assert L.nsf_create(ctypes.byref(c), -1, ctypes.byref(h)) == 0
    try:
        assert L.nsf_initialize(h) == 0
        types = np.empty(27, dtype=np.uint8)
        assert L.nsf_get_node_types(h, types.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))) == 0
        want = np.full(27, 2, dtype=np.uint8)
        want[13] = 0
        np.testing.assert_array_equal(types, want)
    finally:
        L.nsf_destroy(h)
