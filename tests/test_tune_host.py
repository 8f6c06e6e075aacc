"""Field autotuner, host side: the grid-size rounding, the first-stage xi
candidates against the reference's geometry rules, and argument checks of
the tuning entry points.  No GPU needed."""
import math

import numpy as np
import pytest


def _factors_ok(n, primes):
    for p in primes:
        while n % p == 0:
            n //= p
    return n == 1


@pytest.mark.parametrize("n", [1, 7, 61, 80, 97, 238, 366, 1009])
def test_next_sizes(n):
    from cumpm_b200 import capi

    f = capi.tune_next_size(n)
    s = capi.tune_next_size(n, smooth23=True)
    assert f >= n and _factors_ok(f, (2, 3, 5, 7))
    assert s >= n and _factors_ok(s, (2, 3))
    assert all(not _factors_ok(k, (2, 3, 5, 7)) for k in range(n, f))
    assert all(not _factors_ok(k, (2, 3)) for k in range(n, s))


def test_next_size_examples():
    from cumpm_b200 import capi

    assert capi.tune_next_size(366) == 375          # 3 x 5^3 after 6 x 61
    assert capi.tune_next_size(366, True) == 384    # 2^7 x 3
    assert capi.tune_next_size(80) == 80
    assert capi.tune_next_size(0) == -1


def _rule_grid(box, tol, xi):
    rc = max(2.0, math.sqrt(-math.log(tol)) / xi)
    kcut = 2.0 * xi * xi * rc
    return [int(math.ceil(1.0 + L * kcut / math.pi)) for L in box], rc


def test_xi_candidates_follow_the_rules():
    """Each candidate's grid and cutoff are the reference's rules at that xi
    (monodisperse_ewald_electric_field.cu:546-616), the caller's xi comes
    first, and no candidate's cutoff passes half the box."""
    from cumpm_b200 import capi

    box = (308.4, 66.5, 200.0)   # the N=4000 monolayer in units of the radius
    c = capi.tune_xi_candidates(capi.FIELD_MONO, box, 1e-6, 0.5)
    assert c[0]["xi"] == 0.5
    assert len(c) >= 5
    for k in c:
        g, rc = _rule_grid(box, 1e-6, k["xi"])
        assert list(k["grid"]) == g
        assert k["rc"] == pytest.approx(rc)
        assert k["rc"] <= min(box) / 2
        assert k["support"] == int(math.ceil(-2.0 * math.log(1e-6) / math.pi))
    # the rule grid at the caller's xi is the field's own
    g = np.zeros(3, np.int32)
    from cumpm_b200.capi import _dp, _ip, lib
    import ctypes as C
    b = np.array(box)
    st = C.c_int()
    assert lib().mpm_ewald_geometry(b.ctypes.data_as(_dp), 1e-6, 0.5, g.ctypes.data_as(_ip), C.byref(st), None, None,
                                    None) == 0
    assert list(c[0]["grid"]) == list(g)


def test_xi_candidates_drop_cutoffs_beyond_half_the_box():
    from cumpm_b200 import capi

    box = (12.0, 12.0, 12.0)   # rc = 3.72 / xi must stay below 6
    c = capi.tune_xi_candidates(capi.FIELD_MONO, box, 1e-6, 0.7)
    xs = [k["xi"] for k in c]
    assert all(3.7169 / x <= 6.0 for x in xs)
    assert 0.7 * 0.7 not in xs   # 0.49: rc 7.6 > 6


def test_xi_candidates_polydisperse():
    from cumpm_b200 import capi

    rng = np.random.default_rng(3)
    radii = rng.uniform(1.0, 4.0, 50)
    box = (83.8, 83.8, 83.8)
    c = capi.tune_xi_candidates(capi.FIELD_POLY, box, 1e-6, 0.5, radius=radii)
    assert c and c[0]["xi"] == 0.5
    for k in c:
        assert k["rc"] >= 2.0 * radii.max() - 1e-12
        assert k["rc"] <= 83.8 / 2


def test_tuned_field_rejects_bad_overrides():
    """Argument checks run before any device work."""
    from cumpm_b200 import capi

    box = (20.0, 20.0, 20.0)
    with pytest.raises(ValueError):
        capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, tuning={"xi": 0.5, "tile": (12, 8)})
    with pytest.raises(ValueError):
        capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, tuning={"xi": 0.5, "tile": (16, 16)})
    with pytest.raises(ValueError):
        capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, tuning={"xi": -1.0})
    with pytest.raises(ValueError):
        capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, tuning={"xi": 0.5, "grid": (4, 32, 32)})


def test_solver_set_tuning_checks_arguments():
    import cumpm_b200 as cuMPM

    s = cuMPM.dipole_solver([100.0, 100.0, 100.0], [2.0 + 0.1j], radius=1.0, quiet=True)
    with pytest.raises(ValueError):
        s.set_tuning(0.5, tile=(8, 3))
    with pytest.raises(ValueError):
        s.set_tuning(0.0)
    s.set_tuning(0.6, grid=(0, 0, 0))   # accepted; used from the first frame on
