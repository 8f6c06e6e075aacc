"""Argument validation of the drop-in API (the reference's tests/test_inputs.py
cases and messages); every check fires before any device work."""
import numpy as np
import pytest

import cumpm_b200 as cuMPM


def test_invalid_box_size():
    with pytest.raises(ValueError, match="box must have length 3"):
        cuMPM.dipole_solver([10.0, 10.0], 4.0)


def test_invalid_field_type():
    with pytest.raises(ValueError, match="field_type must be 'auto'"):
        cuMPM.dipole_solver([10.0] * 3, 4.0, field_type="invalid_type")


def test_invalid_precision():
    with pytest.raises(ValueError, match="Unknown precision mode"):
        cuMPM.dipole_solver([10.0] * 3, 4.0, precision="half")


def test_invalid_quadrupoles_argument():
    with pytest.raises(TypeError):
        cuMPM.dipole_solver([10.0] * 3, 4.0, quadrupoles=3.5)


def test_E0_shapes():
    with pytest.raises(ValueError, match="divisible by 3"):
        cuMPM.dipole_solver([10.0] * 3, 4.0, E0=[1.0, 0.0])
    with pytest.raises(ValueError, match="last dimension of E0 must be 3"):
        cuMPM.dipole_solver([10.0] * 3, 4.0, E0=np.zeros((2, 2, 2)))


def test_coordinate_length_mismatch():
    mpm = cuMPM.dipole_solver([10.0] * 3, 4.0)
    with pytest.raises(Exception):
        mpm._solver.compute([0.0, 1.0], [0.0], [0.0, 0.0])


def test_positions_shape():
    mpm = cuMPM.dipole_solver([10.0] * 3, 4.0)
    with pytest.raises(ValueError, match="positions must be of shape"):
        mpm.compute(np.zeros((2, 2)))


def test_radii_count_mismatch():
    mpm = cuMPM.dipole_solver([10.0] * 3, 4.0, radius=[1.0, 1.0, 1.0])
    with pytest.raises(Exception, match="inconsistent with the number of radii"):
        mpm.compute([[0.0, 0.0, 0.0], [5.0, 5.0, 5.0]])


def test_monodisperse_with_mixed_radii():
    mpm = cuMPM.dipole_solver([10.0] * 3, 4.0, radius=[1.0, 2.0], field_type="monodisperse")
    with pytest.raises(Exception, match="field_type was set to 'monodisperse' but radii are not identical"):
        mpm.compute([[0.0, 0.0, 0.0], [5.0, 5.0, 5.0]])


def test_eps_particle_count_mismatch():
    mpm = cuMPM.dipole_solver([10.0] * 3, np.full((2, 3), 4.0 + 0j))
    with pytest.raises(Exception, match="inconsistent with eps_p"):
        mpm.compute([[0.0, 0.0, 0.0], [5.0, 5.0, 5.0]])


def test_E0_size_mismatch():
    mpm = cuMPM.dipole_solver([10.0] * 3, 4.0, E0=np.ones((1, 9)))
    with pytest.raises(Exception, match=r"Incident field E0\[0\] has size 9"):
        mpm.compute([[0.0, 0.0, 0.0], [5.0, 5.0, 5.0]])


def test_drude_dielectric():
    eps = cuMPM.drude_dielectric(np.array([1.0, 2.0]), 0.1, 1.8, 4.0)
    np.testing.assert_allclose(eps, 4.0 - 1.8 ** 2 / (np.array([1.0, 2.0]) ** 2 + 1j * np.array([1.0, 2.0]) * 0.1))
    with pytest.raises(ValueError, match="same number of values"):
        cuMPM.drude_dielectric(1.0, [0.1, 0.2], 1.8, 4.0)


def test_near_field_arguments():
    with pytest.raises(ValueError, match="E0 must have length 3"):
        cuMPM.Near_Field([10.0] * 3, [1.0, 0.0])
    nf = cuMPM.Near_Field([10.0] * 3, [1.0, 0.0, 0.0])
    with pytest.raises(ValueError, match="can't be set to None"):
        nf.set_dipoles(None)
    with pytest.raises(RuntimeError, match="must set dipoles"):
        nf.calculate()
