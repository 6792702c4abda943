"""Batched ensemble (nsf_ensemble_*): uneven grids with different Mach, Re and sphere size advanced by one
CUDA graph per step must give every member the fields its own plain solve gives, and those must match the
CPU oracle."""
import os

import numpy as np
import pytest

import nsfsi
from oracle import pyoracle as po
from test_parity_gpu import FIELD_TOL, field_errors

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def config_text(c):
    """ConfigFile text of an nsf_config (for the oracle)."""
    base = open(nsfsi.case_path("sphere48")).read().split("case = {")[0]
    lines = []
    for line in base.splitlines():
        key = line.split("=")[0].strip()
        val = {"NI": c.NI, "NJ": c.NJ, "NK": c.NK, "stopTimeLevel": c.stop_time_level, "Re": repr(c.re),
               "M_0": repr(c.m0), "L_x": repr(c.lx)}.get(key)
        lines.append("%s = %s" % (key, val) if val is not None else line)
    s = c.spheres[0]
    return "\n".join(lines) + """
case = {
  kind = "custom";
  bc_x_min = "inlet"; bc_x_max = "outlet";
  bc_y_min = "periodic"; bc_y_max = "periodic";
  bc_z_min = "periodic"; bc_z_max = "periodic";
  spheres = ( (%r, %r, %r, %r) );
  ic = "freestream_noise";
  noise_amp = 1e-4;
  seed = %dL;
};
""" % (s.cx, s.cy, s.cz, s.r, c.seed)


@pytest.mark.gpu
def test_ensemble_members_equal_their_plain_solves():
    cfgs = nsfsi.ensemble_configs(n=6, steps=20)
    with nsfsi.Ensemble(cfgs) as ens:
        tile, lps, items = ens.info()
        assert lps < 40  # one graph per step for all members
        ens.march(20)
        ens.sync()
        for m, c in enumerate(cfgs):
            em = ens.member(m)
            fe = em.download()
            te = em.time()
            with nsfsi.Solver(c) as s:
                s.march(20)
                s.sync()
                fs = s.download()
                assert s.time() == te
            e = field_errors(fe, fs)
            assert (e <= 1e-12).all(), (m, dict(zip(nsfsi.FIELDS, e)))


@pytest.mark.gpu
def test_single_member_ensemble_equals_plain_solve():
    c = nsfsi.ensemble_configs(n=1, steps=10)[0]
    with nsfsi.Ensemble([c]) as ens:
        ens.march(10)
        ens.sync()
        fe = ens.member(0).download()
    with nsfsi.Solver(c) as s:
        s.march(10)
        s.sync()
        e = field_errors(fe, s.download())
    assert (e <= 1e-12).all(), dict(zip(nsfsi.FIELDS, e))


@pytest.mark.gpu
def test_ensemble_member_matches_oracle():
    cfgs = nsfsi.ensemble_configs(n=3, steps=20)
    with nsfsi.Ensemble(cfgs) as ens:
        ens.march(20)
        ens.sync()
        for m in (0, 2):
            o = po.Oracle(config_text(cfgs[m]))
            o.march(20)
            em = ens.member(m)
            t, lv, dt = em.time()
            assert lv == 20 and abs(t - o.t) <= 1e-12 * o.t
            e = field_errors(em.download(), o.fields())
            assert (e <= FIELD_TOL).all(), (m, dict(zip(nsfsi.FIELDS, e)))
