"""Polydisperse spectral Ewald on the host: the C++ restatement of the
reference's pair functions, table lookup, parameters and radius classes
against the oracle, and the oracle's polydisperse operator pinned by the
reference's own known answers (monodisperse equivalence at radius 1,
tests/test_electric_fields.py:30-82; direct sum in a large box,
tests/test_dipole_solvers.py:247-299).  No GPU needed."""
import numpy as np
import pytest

from oracle import mpm_oracle as O


@pytest.mark.parametrize("a,b", [(1.0, 1.0), (1.0, 1.2), (0.8, 1.1), (1.0, 4.0), (2.5, 3.7), (1.0, 1.00001)])
@pytest.mark.parametrize("xi", [0.3, 0.5, 0.8])
def test_pair_functions_match_oracle(a, b, xi):
    from cumpm_b200 import capi

    r = np.linspace(1.0, 9.0, 4001)
    f1, f2, sv = capi.poly_pair_functions(a, b, xi, r)
    g1, g2, sw = O.poly_pair_functions(r, a, b, xi)
    # the C++ form groups the reference's eight terms by symmetry; the sums
    # agree to rounding
    np.testing.assert_allclose(f1, g1, rtol=0, atol=1e-11 * np.abs(g1).max())
    np.testing.assert_allclose(f2, g2, rtol=0, atol=1e-11 * np.abs(g2).max())
    assert abs(sv - sw) <= 1e-12 * abs(sw)


def test_unequal_radii_keep_the_reference_fd2_term():
    """The fd2 exp(-(r+a-b)^2 xi^2) term differs from its symmetric partner
    for a != b; the C++ form must carry that difference."""
    from cumpm_b200 import capi

    r = np.linspace(1.0, 6.0, 501)
    a, b, xi = 1.0, 3.0, 0.5
    _, f2, _ = capi.poly_pair_functions(a, b, xi, r)
    _, g2, _ = O.poly_pair_functions(r, a, b, xi)
    np.testing.assert_allclose(f2, g2, rtol=0, atol=1e-11 * np.abs(g2).max())
    # and the term is not negligible here
    t = a - b
    k = 1.0 / (512 * np.pi ** 1.5 * a ** 3 * b ** 3 * r ** 3 * xi ** 5)
    extra = 8 * t * t * (a * a + 4 * a * b + b * b) * xi ** 4 * r * k * np.exp(-(r + t) ** 2 * xi ** 2)
    assert np.abs(extra).max() > 1e-6 * np.abs(g2).max()


@pytest.mark.parametrize("a,b,xi", [(1.0, 1.0, 0.5), (1.0, 1.2, 0.4), (1.0, 4.0, 0.5)])
def test_table_lookup_matches_oracle(a, b, xi):
    from cumpm_b200 import capi

    p = O.PolyParams([60.0, 60.0, 60.0], 1e-6, xi, [a, b])
    rng = np.random.default_rng(3)
    d = np.concatenate([rng.uniform(0, 1, 40), rng.uniform(1, p.rc + 1, 400), [0.0, 1.0, 1.0005, p.rc, p.rc + 2]])
    f1, f2, _ = capi.poly_pair_functions(a, b, xi, d, rc=p.rc, lookup=True)
    g1, g2 = O.poly_table_lookup(d, a, b, xi, p.r_table)
    np.testing.assert_allclose(f1, g1, rtol=0, atol=1e-11 * np.abs(g1).max())
    np.testing.assert_allclose(f2, g2, rtol=0, atol=1e-11 * np.abs(g2).max())


@pytest.mark.parametrize("box,radii", [
    ([84.0, 84.0, 84.0], [1.0, 1.5, 2.0, 1.5000001, 4.0]),
    ([20.0, 20.0, 20.0], [1.0] * 4),
    ([120.0, 120.0, 120.0], [1.0, 1.2, 0.8, 1.1]),
    ([30.0, 26.0, 40.0], list(np.random.default_rng(5).uniform(1, 2, 50))),
])
def test_parameters_and_classes_match_oracle(box, radii):
    from cumpm_b200 import capi

    g = capi.poly_geometry(box, 1e-6, 0.5, radii)
    p = O.PolyParams(box, 1e-6, 0.5, radii)
    assert g["grid"] == list(p.num_grid)
    assert g["P"] == p.P
    assert g["eta"] == pytest.approx(p.eta, rel=1e-15)
    assert g["rc"] == pytest.approx(p.rc, rel=1e-15)
    assert g["n_classes"] == len(p.unique)
    np.testing.assert_array_equal(g["cls"], p.ridx)


def test_cutoff_error_message():
    from cumpm_b200 import capi

    with pytest.raises(RuntimeError, match="larger than half the box length"):
        capi.poly_geometry([12.0, 12.0, 12.0], 1e-6, 0.5, [1.0, 1.0])
    with pytest.raises(RuntimeError, match="larger than half the box length"):
        O.PolyParams([12.0, 12.0, 12.0], 1e-6, 0.5, [1.0, 1.0])


def test_oracle_poly_matches_mono_at_unit_radius():
    """Reference KAT: polydisperse with radius 1 reproduces the monodisperse
    field to 1e-5 (tests/test_electric_fields.py:30-82)."""
    box = (20.0, 20.0, 20.0)
    pos = np.array([[0.0, 0, 0], [5, 0, 0], [10, 0, 0], [15, 0, 0]])
    p = np.zeros((4, 3), complex)
    p[:, 0] = 1.0
    sc = np.ones(4)
    m = O.MonoEwaldOperator(box, 1e-6, 0.5)
    m.set_positions(pos)
    q = O.PolyEwaldOperator(box, 1e-6, 0.5, [1.0] * 4)
    q.set_positions(pos)
    Em = m.apply(p.ravel(), sc)
    Eq, (Er, Es) = q.apply(p.ravel(), sc, split=True)
    np.testing.assert_allclose(Em, Eq, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(Eq, (Er + Es).ravel(), rtol=1e-12, atol=1e-12)


def test_oracle_poly_interaction_sign():
    """INTERACTION_FIELD: -(reciprocal + pairs), no self term (:2714-2730)."""
    rng = np.random.default_rng(7)
    box = (24.0, 24.0, 24.0)
    pos = rng.uniform(0, 24, (6, 3))
    fp = rng.uniform(0, 24, (5, 3))
    radii = [1.0, 1.3, 1.0, 1.6, 1.3, 1.0]
    p = rng.standard_normal((6, 3)) + 1j * rng.standard_normal((6, 3))
    q = O.PolyEwaldOperator(box, 1e-6, 0.5, radii, solver_ax=False)
    q.set_positions(pos, field_points=fp)
    E, (Er, Es) = q.apply(p.ravel(), split=True)
    np.testing.assert_allclose(E, -(Er + Es).ravel(), rtol=1e-14)


def drude(omega, gamma, omega_p, eps_inf):
    return eps_inf - omega_p ** 2 / (omega ** 2 + 1j * omega * gamma)


def test_oracle_poly_solver_matches_direct_in_large_box():
    """Reference KAT (dipoles): mixed radii in a 120^3 box, Ewald -> direct
    sum to 1e-3 (tests/test_dipole_solvers.py:247-299)."""
    d = 12.0
    eps = drude(np.linspace(2000, 6000, 3), 681, 12313, 4)
    pos = np.array([[0.0, 0.0, 0.0], [d, 0.0, 0.0], [-d, 0.0, 0.0], [0.0, d, 0.0]])
    radii = [1.0, 1.2, 0.8, 1.1]
    E = np.repeat(eps[:, None], 4, axis=1)
    a = O.DipoleSolverOracle([120.0] * 3, E, radius=radii, eps_m=1.8, tol=1e-6, field_type="direct")
    a.compute(pos)
    b = O.DipoleSolverOracle([120.0] * 3, E, radius=radii, eps_m=1.8, xi=0.4, tol=1e-6, field_type="polydisperse")
    b.compute(pos)
    np.testing.assert_allclose(a.get_eff_polarizability(), b.get_eff_polarizability(), rtol=1e-3, atol=1e-3)
    np.testing.assert_allclose(a.get_dipoles(), b.get_dipoles(), rtol=1e-3, atol=1e-3)


def test_near_field_polydisperse_branch():
    """Near field with field_type polydisperse (near_field.cu:98-135): at
    equal radii it is the monodisperse near field (the mono/poly
    equivalence at radius 1 holds for field points too), and "auto" with
    unequal radii takes it."""
    rng = np.random.default_rng(17)
    box = [30.0, 28.0, 32.0]
    dip_pos = np.array([[3.0, 4.0, 5.0], [12.0, 14.0, 9.0], [20.0, 6.0, 25.0]])
    dip = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    fp = rng.uniform(0, 28, (6, 3))
    E0 = [1.0, 0.0, 0.0]
    a = O.near_field_intensity(box, E0, 1.0, dip, dip_pos, fp, errortol=1e-6, field_type="monodisperse")
    b = O.near_field_intensity(box, E0, 1.0, dip, dip_pos, fp, errortol=1e-6, field_type="polydisperse")
    np.testing.assert_allclose(b, a, rtol=1e-5)
    c = O.near_field_intensity(box, E0, [1.0, 1.3, 1.1], dip, dip_pos, fp, errortol=1e-6, field_type="auto")
    d = O.near_field_intensity(box, E0, [1.0, 1.3, 1.1], dip, dip_pos, fp, errortol=1e-6, field_type="polydisperse")
    np.testing.assert_array_equal(c, d)
    assert np.abs(c - a).max() > 0
