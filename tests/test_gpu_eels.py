"""EELS on the device batched solve (cumpm_b200.eels) against the reference's
golden vector and the EELS oracle."""
import numpy as np
import pytest

from oracle import mpm_eels as E

pytestmark = pytest.mark.gpu


def test_reference_golden_two_beams_five_frequencies(golden):
    """tests/test_eels_solver.py:114-173 of the reference, through the
    drop-in class: loss / (omega R) * (4 pi)^2 and the scaled dipoles to the
    reference test's 2e-2."""
    import cumpm_b200.eels as eels

    g = golden("ref_eels_vs_python_module.npz")
    R = float(g["radius"])
    s = eels.EELS(box=g["box"], eps_p=g["eps_p"], omega=g["omega_nm"], v=float(g["v"]), eps_m=float(g["eps_m"]),
                  radius=R, xi=0.5, tol=1e-3, field_type="direct", solver_type="bicgstab", quiet=True,
                  precision="double")
    s.compute(g["e_pos"], g["points"])
    loss = s.get_eels() / (g["omega_nm"] * R) * (4.0 * np.pi) ** 2
    np.testing.assert_allclose(loss, g["ref_eels"], rtol=2e-2, atol=1e-5)
    np.testing.assert_allclose(s.get_dipoles(physical=False), g["ref_dips_stacked"], rtol=2e-2, atol=1e-5)


@pytest.mark.parametrize("field_type,radius", [("direct", 3.0), ("monodisperse", 3.0),
                                               ("polydisperse", [3.0, 3.6, 2.5])])
def test_matches_oracle(field_type, radius):
    import cumpm_b200.eels as eels

    box = np.array([80.0, 80.0, 80.0])
    pts = np.array([[0.0, 0.0, 0.0], [9.0, 1.0, -2.0], [-3.0, 8.5, 4.0]])
    omega = np.array([0.04, 0.06, 0.09])
    eps = 4.0 - 1.5 ** 2 / (omega ** 2 * 100 + 0.05j)
    beams = np.array([[4.0, -5.0], [12.0, 3.0]])
    s = eels.EELS(box, eps, omega, 0.5, eps_m=1.3, radius=radius, tol=1e-9, field_type=field_type, quiet=True,
                  precision="double")
    s.compute(beams, pts)
    o = E.EELSOracle(box, eps, omega, 0.5, eps_m=1.3, radius=radius, tol=1e-9, field_type=field_type)
    for b in beams:
        o.compute(b, pts)
    ref = np.array(o.eels)
    np.testing.assert_allclose(s.get_eels(), ref, rtol=1e-6, atol=1e-9 * np.abs(ref).max())
    np.testing.assert_allclose(s.get_dipoles(physical=False), np.array(o.dipoles), rtol=1e-6,
                               atol=1e-8 * np.abs(np.array(o.dipoles)).max())


def test_split_systems_match_oracle():
    """Splitting near the beam (cubic, 27 -> 19 sub-dipoles): each beam
    position solves its own split system; the oracle solves the same split
    systems (built by the splitting that tests/test_eels_host.py pins
    against the reference's Python)."""
    import cumpm_b200.eels as eels

    box = np.array([80.0, 80.0, 80.0])
    pts = np.array([[0.0, 0.0, 0.0], [12.0, 0.0, 0.0], [0.0, 13.0, 2.0]])
    omega = np.array([0.05, 0.08])
    eps = 4.0 - 1.5 ** 2 / (omega ** 2 * 100 + 0.05j)
    beams = np.array([[2.0, 1.0], [11.0, -2.0]])
    s = eels.EELS(box, eps, omega, 0.5, radius=3.0, tol=1e-9, field_type="direct", quiet=True, split_dist=5.0,
                  N_split=27, precision="double")
    s.compute(beams, pts)
    off = eels.unit_offsets("cubic", 27)
    ref_eels, ref_dips = [], []
    for b in beams:
        sp, sr, se = eels.split_near_beam(pts, b, np.full(3, 3.0), np.repeat(eps[:, None], 3, axis=1), 5.0, off)
        o = E.EELSOracle(box, se, omega, 0.5, radius=sr, tol=1e-9, field_type="direct")
        l, d = o.compute(b, sp)
        ref_eels.append(l)
        ref_dips.append(d)
    np.testing.assert_allclose(s.get_eels(), np.array(ref_eels), rtol=1e-6)
    np.testing.assert_allclose(s.get_dipoles(physical=False), np.array(ref_dips), rtol=1e-6,
                               atol=1e-8 * np.abs(np.array(ref_dips)).max())
    assert len(s.get_positions()) == 2 and len(s.get_positions()[0]) == 2 + 19


@pytest.mark.parametrize("method,n", [("cubic", 27), ("fcc", 50)])
def test_reference_splitting_checks(method, n):
    """tests/test_eels_solver.py:176-230 of the reference: particle 0 near
    the beam is split; with fcc the sub-dipoles keep its centre."""
    import cumpm_b200 as cuMPM

    s = cuMPM.EELS(box=[100, 100, 100], eps_p=[4.0], omega=[0.15], v=0.3, radius=2.0, split_dist=4.0, N_split=n,
                   split_method=method, field_type="direct", precision="double", quiet=True)
    s.compute(np.array([1.0, 0.0]), np.array([[0.0, 0.0, 0.0], [10.0, 0.0, 0.0]]))
    split_pos = s.get_positions()
    assert len(split_pos) > 2
    if method == "fcc":
        assert np.linalg.norm(np.mean(split_pos[1:], axis=0)) < 1e-12
    assert np.all(np.isfinite(s.get_eels()))
