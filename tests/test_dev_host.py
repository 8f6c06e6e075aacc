"""cumpm_b200.dev argument handling that needs no GPU: the reference's
precision and mode parsing, and the gaps it names."""
import numpy as np
import pytest


def test_precision_and_mode_parsing():
    from cumpm_b200 import dev

    ef = dev.MonodisperseEwaldElectricField(20.0, 20.0, 20.0, 1e-6, 0.5, True, precision="mixed")
    assert ef.is_using_recip_fp32 and ef.recip_precision_mode == dev.PrecisionMode.MIXED
    assert ef.mode == dev.FieldCalcMode.SOLVER_AX
    ef = dev.MonodisperseEwaldElectricField(20.0, 20.0, 20.0, 1e-6, 0.5, False, precision="double")
    assert not ef.is_using_recip_fp32 and ef.mode == dev.FieldCalcMode.INTERACTION_FIELD
    d = dev.DirectElectricField(np.ones(3), mode=False, precision=dev.PrecisionMode.FP32)
    assert d.is_using_fp32 and d.precision_mode == dev.PrecisionMode.FP32
    with pytest.raises(ValueError):
        dev.DirectElectricField(np.ones(3), precision="quad")


def test_inputs_and_sizes():
    from cumpm_b200 import dev

    ef = dev.MonodisperseEwaldElectricField(20.0, 20.0, 20.0, 1e-6, 0.5, True, solve_quadrupoles=True,
                                            quad_idxs=[0, 2])
    ef.update_particle_coordinates([0, 4, 8, 12], [0, 0, 0, 0], [0, 0, 0, 0])
    ef.update_dipoles_complex(np.ones(4), np.zeros(4), np.zeros(4), np.ones(4), np.zeros(4), np.zeros(4))
    assert ef.num_particles == 4 and ef.num_quads == 2 and ef.num_field_points == 0
    xr, xi, yr, yi, zr, zi = ef.get_dipoles_complex_host()
    assert np.all(xr == 1) and np.all(yi == 1) and np.all(zr == 0)
    ef.set_self_coef(2.0)
    assert np.all(ef._self == 2.0)


def test_named_gaps():
    from cumpm_b200 import dev

    ef = dev.PolydisperseEwaldElectricField(20.0, 20.0, 20.0, 1e-6, 0.5, True, [1.0, 1.2], solve_quadrupoles=True)
    with pytest.raises(RuntimeError, match="Bloch"):
        ef.set_bloch_wavevector(0.1, 0.0)
    ef = dev.PolydisperseEwaldElectricField(20.0, 20.0, 20.0, 1e-6, 0.5, True, [1.0, 1.2])
    ef.set_bloch_wavevector(0.1, 0.0)   # dipoles: taken (applied at the next calculate)
    assert ef._bloch == (0.1, 0.0)
    with pytest.raises(ValueError, match="radius"):
        dev.MonodisperseEwaldElectricField(20.0, 20.0, 20.0, 1e-6, 0.5, True, radius=2.0)


def test_inputs_must_match_particle_count():
    """Mismatched inputs are rejected on the host, before any device call."""
    from cumpm_b200 import dev

    ef = dev.MonodisperseEwaldElectricField(20.0, 20.0, 20.0, 1e-6, 0.5, True)
    ef.set_self_coef(1.0)                       # no particles yet: zero entries
    ef.update_particle_coordinates([0, 4, 8], [0, 0, 0], [0, 0, 0])
    ef.update_dipoles(np.ones(3), np.zeros(3), np.zeros(3))
    with pytest.raises(ValueError, match="self coefficients"):
        ef._inputs()
    ef.set_self_coef(np.ones(3))
    ef.update_dipoles(np.ones(2), np.zeros(2), np.zeros(2))
    with pytest.raises(ValueError, match="dipoles"):
        ef._inputs()
