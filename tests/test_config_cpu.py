"""ConfigFile reader (nsf_config_load / nsf_config_parse) against ConfigSettings semantics
(src/ConfigSettings.cpp:18-163): names, strict typing, the filter-list rule, derived precision buffer."""
import os

import numpy as np
import pytest

import nsfsi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_defaults_are_the_shipped_configfile():
    c = nsfsi.config_defaults()
    assert (c.NI, c.NJ, c.NK) == (161, 83, 3)
    assert c.stop_criterion == 1 and c.t_end == 200.0
    assert list(c.filter_intervals[:3]) == [50, 200, 1000]
    assert c.re == 400.0 and c.m0 == 0.25 and c.pr == 0.72
    assert c.shipped_case == 1
    assert c.machine_precision_buffer == np.finfo(float).eps * (2.0 + 1.0 + 0.05)


def test_workload_files_parse():
    c = nsfsi.config_load(nsfsi.case_path("tgv256"))
    assert (c.NI, c.NJ, c.NK) == (256, 256, 256) and c.ic == nsfsi.IC["tgv"] and c.n_spheres == 0
    c = nsfsi.config_load(nsfsi.case_path("sphere48"))
    assert c.n_spheres == 1 and c.spheres[0].r == 0.1 and c.seed == 20240101
    assert [list(c.bc[a]) for a in range(3)] == [[2, 3], [0, 0], [0, 0]]


@pytest.mark.parametrize("bad,msg", [
    ("NI = 4.0", "integer"),
    ("stopCriterion = \"forever\"", "stopCriterion"),
    ("filterIntervals = [50]", "filterIntervalChangeTimes"),
    ("saveConvergenceHistory = \"some\"", "saveConvergenceHistory"),
    ("Gamma = 1", "float"),
])
def test_config_errors(bad, msg):
    text = open(nsfsi.case_path("sphere48")).read()
    key = bad.split("=")[0].strip()
    lines = [l if not l.startswith(key + " ") else bad for l in text.splitlines()]
    with pytest.raises(nsfsi.NsfError) as e:
        nsfsi.config_parse("\n".join(lines))
    assert e.value.code == 1 and msg in str(e.value)


def test_missing_file_is_a_config_error():
    with pytest.raises(nsfsi.NsfError) as e:
        nsfsi.config_load("/nonexistent/ConfigFile")
    assert e.value.code == 1


def test_missing_setting_is_reported():
    text = "\n".join(l for l in open(nsfsi.case_path("sphere48")).read().splitlines() if not l.startswith("Pr "))
    with pytest.raises(nsfsi.NsfError) as e:
        nsfsi.config_parse(text)
    assert "not found: Pr" in str(e.value)
