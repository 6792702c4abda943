"""The stage kernel's reciprocal and square root (Newton-Raphson refinement of the hardware
approximations, recip_nr / sqrt_nr in nsf_physics.cuh) against CUDA's IEEE 1/x and sqrt(x) on the
device: within 2 ulps over the range the primitive values take (1 + rho, 1 + T, the viscosity
denominator) and over a wide range of positive normal numbers."""
import numpy as np
import pytest

import nsfsi


def ulps(a, b):
    return np.abs(a - b) / np.spacing(np.abs(b))


@pytest.mark.gpu
def test_newton_raphson_reciprocal_and_sqrt_match_ieee():
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(0.25, 4.0, 200000), np.exp(rng.uniform(-300 * np.log(10) / 10,
                                                                             300 * np.log(10) / 10, 100000)),
                        [1.0, 2.0, 0.5, 1.0 + 2 ** -52, 1.0 - 2 ** -53]])
    r_nr, r_ieee, s_nr, s_ieee = nsfsi.math_selftest(x)
    assert np.array_equal(r_ieee, 1.0 / x)
    assert np.array_equal(s_ieee, np.sqrt(x))
    assert ulps(r_nr, r_ieee).max() <= 2
    assert ulps(s_nr, s_ieee).max() <= 2
    print("max ulps: reciprocal %.1f, sqrt %.1f; exact share %.3f / %.3f" % (
        ulps(r_nr, r_ieee).max(), ulps(s_nr, s_ieee).max(), np.mean(r_nr == r_ieee), np.mean(s_nr == s_ieee)))
