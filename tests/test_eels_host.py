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
    with pytest.raises(RuntimeError, match="not available in this build"):
        eels.EELS([50.0] * 3, [4.0], [0.1], 0.3, solve_quadrupoles=True)
    with pytest.raises(ValueError, match="asm_Nx and asm_Ny"):
        eels.EELS([50.0] * 3, [4.0], [0.1], 0.3, asm_flag=True, asm_Nx=0)
    s = eels.EELS([50.0] * 3, [4.0], [0.1], 0.3, asm_flag=True, asm_Nx=3, asm_Ny=2)
    assert s.asm_n == (3, 2)


def test_beam_field_images_match_the_oracle():
    """The zone sum's beam field (periodic images with the Bloch phase)
    agrees with the oracle's restatement term by term."""
    from cumpm_b200 import eels
    from oracle import mpm_eels as E

    rng = np.random.default_rng(2)
    pos = rng.uniform(0, 20, (7, 3))
    box = np.array([20.0, 18.0, 30.0])
    for k, asm in (((0.0, 0.0), False), ((0.07, -0.11), True)):
        a = eels.beam_field(pos, [3.0, 4.0], 0.05, 0.4, 1.0 / np.sqrt(1 - 0.16), 2.0, box, k, asm)
        b = E.beam_field(pos, [3.0, 4.0], 0.05, 0.4, 1.0 / np.sqrt(1 - 0.16), 2.0, box, k, asm)
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15 * np.abs(b).max())


def test_positions_and_beams_are_checked():
    from cumpm_b200 import eels

    s = eels.EELS([50.0] * 3, [4.0], [0.1], 0.3)
    with pytest.raises(ValueError, match="positions must be of shape"):
        s.compute([0.0, 0.0], np.zeros((3, 2)))
    with pytest.raises(ValueError, match="epos must be of shape"):
        s.compute([0.0, 0.0, 1.0], np.zeros((3, 3)))


@pytest.mark.parametrize("method", ["cubic", "fibonacci", "fcc"])
@pytest.mark.parametrize("n", [8, 27, 50, 100])
def test_unit_offsets_match_reference(golden, method, n):
    """Sub-dipole lattices against the reference's own Python
    (src/cuMPM/eels.py:177-258; fixture script
    tests/golden/make_eels_split_golden.py)."""
    from cumpm_b200 import eels

    ref = golden("ref_eels_split.npz")[f"offsets_{method}_{n}"]
    got = eels.unit_offsets(method, n)
    assert got.shape == ref.shape
    np.testing.assert_allclose(got, ref, rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("method,n", [("cubic", 27), ("fibonacci", 20), ("fcc", 50)])
def test_split_near_beam_matches_reference(golden, method, n):
    """Particles 0 and 2 lie within 4 of the beam at (1, 0) (particle 3 just
    outside, at 4.03): they become sub-dipoles after the untouched particles
    1 and 3 (eels.py:261-320)."""
    from cumpm_b200 import eels

    g = golden("ref_eels_split.npz")
    off = eels.unit_offsets(method, n)
    p, r, e = eels.split_near_beam(g["split_pos_in"], g["split_epos"], g["split_radii_in"], g["split_eps_in"],
                                   float(g["split_dist"]), off)
    np.testing.assert_allclose(p, g[f"split_{method}_{n}_pos"], rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(r, g[f"split_{method}_{n}_radii"], rtol=1e-14)
    np.testing.assert_array_equal(e, g[f"split_{method}_{n}_eps"])
    assert len(p) == 2 + 2 * len(off)
    # the sub-dipoles keep each particle's volume
    vol = np.sum(r ** 3)
    assert vol == pytest.approx(np.sum(g["split_radii_in"] ** 3), rel=1e-12)


def test_split_with_no_particle_near_the_beam_is_a_copy():
    from cumpm_b200 import eels

    pos = np.array([[10.0, 0, 0], [0, 12.0, 0]])
    p, r, e = eels.split_near_beam(pos, [0.0, 0.0], [1.0, 2.0], np.ones((3, 2)), 4.0, eels.unit_offsets("cubic", 8))
    np.testing.assert_array_equal(p, pos)
    assert r.tolist() == [1.0, 2.0] and e.shape == (3, 2)


@pytest.mark.parametrize("method,n", [("cubic", 27), ("cubic", 64), ("fcc", 50), ("fcc", 13)])
def test_symmetric_lattices_keep_the_centre(method, n):
    """The cubic and fcc sub-dipole lattices are symmetric about the centre,
    so a split particle's sub-dipoles keep its centre (the reference checks
    this for fcc, tests/test_eels_solver.py:229-230) and its volume."""
    from cumpm_b200 import eels

    off = eels.unit_offsets(method, n)
    assert np.linalg.norm(off.mean(axis=0)) < 1e-12
    assert np.all(np.linalg.norm(off, axis=1) <= 1.0)
