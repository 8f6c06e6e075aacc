"""Near_Field with unequal radii (the polydisperse field in INTERACTION
mode, near_field.cu:98-135) against the oracle's near field."""
import numpy as np
import pytest

from oracle import mpm_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("field_type", ["auto", "polydisperse"])
def test_polydisperse_near_field_matches_oracle(field_type):
    import cumpm_b200 as cuMPM

    rng = np.random.default_rng(17)
    box = [30.0, 28.0, 32.0]
    radius = [1.0, 1.3, 1.1]
    dip_pos = np.array([[3.0, 4.0, 5.0], [12.0, 14.0, 9.0], [20.0, 6.0, 25.0]])
    dip = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    fp = rng.uniform(0, 28, (6, 3))
    E0 = [1.0, 0.0, 0.0]
    nf = cuMPM.Near_Field(box, E0, radius=radius, dip=dip, dip_pos=dip_pos, field_points=fp, errortol=1e-6,
                          field_type=field_type)
    got = nf.calculate()
    ref = O.near_field_intensity(box, E0, radius, dip, dip_pos, fp, errortol=1e-6, field_type=field_type)
    # the near field runs the reference's default precision: fp32 reciprocal
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
