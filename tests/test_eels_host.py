"""Host side of cumpm_b200.eels (no GPU): the beam field and Bessel rules
against the EELS oracle, and the constructor's checks."""
import numpy as np
import pytest

from oracle import mpm_eels as E


def test_beam_field_matches_oracle():
    from cumpm_b200 import eels

    rng = np.random.default_rng(3)
    pos = rng.uniform(-20, 20, (40, 3))
    ls = 2.5
    for om, v in ((0.02, 0.3), (0.2, 0.7), (1.3, 0.45)):
        gamma = 1.0 / np.sqrt(1.0 - v * v)
        a = eels.beam_field(pos, np.array([1.5, -0.5]), om, v, gamma, ls)
        b = E.beam_field(pos, np.array([1.5, -0.5]), om, v, gamma, ls)
        np.testing.assert_allclose(a, b, rtol=1e-13, atol=1e-300)


@pytest.mark.parametrize("n", [0, 1])
def test_bessel_rules_match_oracle(n):
    from cumpm_b200 import eels

    z = np.array([0.3, 2.0, 7.5, 0.4j, -3.0j, 1.0 + 0.5j])
    np.testing.assert_allclose(eels._bessel_k(n, z), [E.eval_k(n, x) for x in z], rtol=1e-14)


def test_constructor_checks():
    from cumpm_b200 import eels

    with pytest.raises(ValueError, match="Both split_dist and N_split must be specified"):
        eels.EELS([50.0] * 3, [4.0], [0.1], 0.3, split_dist=2.0)
    with pytest.raises(ValueError, match="split_method"):
        eels.EELS([50.0] * 3, [4.0], [0.1], 0.3, split_method="hex")
    with pytest.raises(ValueError, match="field_type"):
        eels.EELS([50.0] * 3, [4.0], [0.1], 0.3, field_type="fast")
    with pytest.raises(ValueError, match="box must have length 3"):
        eels.EELS([50.0] * 2, [4.0], [0.1], 0.3)
    for kw in (dict(split_dist=4.0, N_split=27), dict(solve_quadrupoles=True), dict(asm_flag=True)):
        with pytest.raises(RuntimeError, match="not available in this build"):
            eels.EELS([50.0] * 3, [4.0], [0.1], 0.3, **kw)


def test_positions_and_beams_are_checked():
    from cumpm_b200 import eels

    s = eels.EELS([50.0] * 3, [4.0], [0.1], 0.3)
    with pytest.raises(ValueError, match="positions must be of shape"):
        s.compute([0.0, 0.0], np.zeros((3, 2)))
    with pytest.raises(ValueError, match="epos must be of shape"):
        s.compute([0.0, 0.0, 1.0], np.zeros((3, 3)))
