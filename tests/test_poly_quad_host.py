"""Polydisperse quadrupoles in the oracle: the radius-1 quadrupole tables the
polydisperse field builds for itself, its point-Gaussian quadrupole grid and
joint scale, pinned by the reference CPU operator's tables where the two
fields share an expression and by the reference's own solver-level checks
(tests/test_dipole_solvers.py:190-290 of the reference).  No GPU needed."""
import numpy as np
import pytest

from oracle import mpm_oracle as O

SHARED = {"fq1": "field_quad_1", "fq2": "field_quad_2", "fq3": "field_quad_3", "gq1": "grad_quad_1",
          "gq4": "grad_quad_4"}


def drude(omega, gamma, omega_p, eps_inf):
    return eps_inf - omega_p ** 2 / (omega ** 2 + 1j * omega * gamma)


@pytest.mark.parametrize("xi", [0.4, 0.5])
def test_shared_quadrupole_tables_match_reference_cpu(golden, xi):
    """fq1-fq3, gq1 and gq4 of the polydisperse field are the monodisperse
    expressions: they reproduce the reference CPU operator's tables."""
    g = golden("refcpu_tables.npz")
    r = g[f"r@{xi}"][1:]
    _, T, _, _ = O.mono_real_tables(xi, r, variant="poly")
    for k, n in SHARED.items():
        ref = g[f"{n}@{xi}"][1:]
        np.testing.assert_allclose(T[k][1:], ref, rtol=1e-11, atol=1e-13 * np.abs(ref).max())


@pytest.mark.parametrize("xi", [0.4, 0.5])
def test_gq3_differs_only_in_two_signs(xi):
    """The polydisperse gq3 flips the r^5 and r^4 terms of its
    exp(-(r+2)^2 xi^2) coefficient (polydisperse_ewald_electric_field.cu:1927-1933
    against monodisperse_ewald_electric_field.cu:375-383)."""
    r = 1.0 + np.arange(1, 4000) * 0.002
    _, M, _, _ = O.mono_real_tables(xi, r)
    _, P, _, _ = O.mono_real_tables(xi, r, variant="poly")
    x = xi
    c = -15.0 / (65536 * np.pi ** 1.5 * x ** 9 * r ** 5)
    term = (216 * x ** 4 + 144 * x ** 6 + 128 * x ** 8) * r ** 5 - (480 * x ** 6 + 256 * x ** 8) * r ** 4
    want = -2.0 * c * term * np.exp(-(r + 2.0) ** 2 * x * x)
    np.testing.assert_allclose(P["gq3"][1:] - M["gq3"][1:], want, rtol=1e-9, atol=1e-12 * np.abs(M["gq3"]).max())
    for k in SHARED:
        np.testing.assert_array_equal(P[k], M[k])


def test_self_gradient_at_radius_one_is_monodisperse():
    for xi in (0.3, 0.4, 0.5, 0.7):
        _, _, _, sg = O.mono_real_tables(xi, np.array([1.0, 1.5]))
        assert abs(O.poly_self_grad(1.0, xi) - sg) <= 1e-14 * abs(sg)
        # a^-5 scaling with xi a
        assert abs(O.poly_self_grad(2.0, xi) - O.poly_self_grad(1.0, 2.0 * xi) / 32.0) <= 1e-14 * abs(sg)


def test_point_weights_are_a_normalised_gaussian():
    """Summed over a support large enough, the point weights integrate the
    unit Gaussian (2 xi^2/pi)^1.5 exp(-2 xi^2 r^2): their sum is 1."""
    prm = O.PolyParams((30.0, 28.0, 32.0), 1e-8, 0.5, [1.0])
    idx, w = O.poly_point_weights(prm, np.array([[3.3, 7.1, 30.9], [15.0, 14.0, 16.0]]))
    np.testing.assert_allclose(w.sum(axis=1), 1.0, rtol=1e-6)
    assert idx.min() >= 0 and idx.max() < np.prod(prm.num_grid)


def _setup(rng, radii, qi, box=(26.0, 24.0, 28.0)):
    pos = np.array([[2, 2, 2], [8, 3, 4], [14, 9, 5], [3, 15, 12], [18, 18, 18], [10, 20, 7.0]])[:len(radii)]
    op = O.PolyEwaldOperator(box, 1e-6, 0.5, radii, True, qi)
    op.set_positions(pos)
    N, Nq = len(radii), len(qi)
    X = np.concatenate([(rng.standard_normal((N, 3)) + 1j * rng.standard_normal((N, 3))).ravel(),
                        (rng.standard_normal((Nq, 5)) + 1j * rng.standard_normal((Nq, 5))).ravel()])
    sc = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    return op, X, sc


def test_dipole_block_is_the_dipole_operator():
    """With the quadrupoles zero, E is the dipole-only field exactly."""
    rng = np.random.default_rng(21)
    radii = [1.0, 1.3, 1.0, 1.6, 1.3, 1.0]
    op, X, sc = _setup(rng, radii, [0, 3, 4])
    N = len(radii)
    X[3 * N:] = 0.0
    d = O.PolyEwaldOperator(op.p.box, 1e-6, 0.5, radii, True)
    d.set_positions(op.pos)
    np.testing.assert_allclose(op.apply(X, sc)[:3 * N], d.apply(X[:3 * N], sc), rtol=1e-13,
                               atol=1e-14 * np.abs(d.apply(X[:3 * N], sc)).max())


def test_operator_is_linear():
    rng = np.random.default_rng(22)
    op, X, sc = _setup(rng, [1.0, 1.3, 1.0, 1.6], [0, 1, 2, 3])
    _, Y, _ = _setup(rng, [1.0, 1.3, 1.0, 1.6], [0, 1, 2, 3])
    a, b = 0.7 - 0.2j, -1.3 + 0.4j
    np.testing.assert_allclose(op.apply(a * X + b * Y, sc), a * op.apply(X, sc) + b * op.apply(Y, sc),
                               rtol=1e-11, atol=1e-12 * np.abs(op.apply(X, sc)).max())


def test_subset_spreads_quadrupole_q_on_particle_q():
    """The quadrupole grid takes quadrupole q on particle q's stencil
    (polydisperse_ewald_electric_field.cu:994-1005): the reciprocal E of a
    quadrupole carried by particle 2 equals that of the same quadrupole on
    particle 0."""
    rng = np.random.default_rng(23)
    radii = [1.0, 1.3, 1.0, 1.6]
    a, X, _ = _setup(rng, radii, [2])
    b, _, _ = _setup(rng, radii, [0])
    N = len(radii)
    X[:3 * N] = 0.0
    Ea, _ = a.reciprocal(X[:3 * N].reshape(N, 3), X[3 * N:].reshape(1, 5))
    Eb, _ = b.reciprocal(X[:3 * N].reshape(N, 3), X[3 * N:].reshape(1, 5))
    np.testing.assert_array_equal(Ea, Eb)
    assert np.abs(Ea).max() > 0


def test_field_points_with_quadrupoles_are_refused():
    op = O.PolyEwaldOperator((24.0, 24.0, 24.0), 1e-6, 0.5, [1.0, 1.2], False, [0])
    with pytest.raises(NotImplementedError):
        op.set_positions(np.array([[2.0, 2, 2], [9, 9, 9]]), field_points=np.array([[5.0, 5, 5]]))


def test_reference_check_equal_radii_subset_matches_monodisperse():
    """Reference KAT: four particles in a line, quadrupoles on particles 0
    and 2; the polydisperse solve matches the monodisperse quadrupole solve
    to 1e-3 (tests/test_dipole_solvers.py:190-241)."""
    d = 10.0
    eps = drude(np.linspace(1000, 7000, 3), 681, 12313, 4)
    pos = np.array([[0.0, 0, 0], [d, 0, 0], [2 * d, 0, 0], [3 * d, 0, 0]])
    E = np.repeat(eps[:, None], 4, axis=1)
    kw = dict(radius=[1.0], eps_m=2.13, tol=1e-6, solve_quadrupoles=True, quad_idxs=[0, 2])
    a = O.DipoleSolverOracle([5 * d] * 3, E, field_type="monodisperse", **kw)
    a.compute(pos)
    b = O.DipoleSolverOracle([5 * d] * 3, E, field_type="polydisperse", **kw)
    b.compute(pos)
    assert b.get_quadrupoles().shape == (1, 3, 2, 3, 5)
    for f in ("get_eff_polarizability", "get_dipoles", "get_quadrupoles"):
        np.testing.assert_allclose(getattr(a, f)(), getattr(b, f)(), rtol=1e-3, atol=1e-3)


def test_reference_check_mixed_radii_large_box_matches_direct():
    """Reference KAT: mixed radii with quadrupoles on particles 0 and 2 in a
    120^3 box, Ewald -> direct sum to 1e-3 (tests/test_dipole_solvers.py:244-290);
    the middle one of the reference's three frequencies keeps the CPU time
    short."""
    d = 12.0
    eps = drude(np.linspace(2000, 6000, 3), 681, 12313, 4)[1:2]
    pos = np.array([[0.0, 0.0, 0.0], [d, 0.0, 0.0], [-d, 0.0, 0.0], [0.0, d, 0.0]])
    radii = [1.0, 1.2, 0.8, 1.1]
    E = np.repeat(eps[:, None], 4, axis=1)
    kw = dict(radius=radii, eps_m=1.8, tol=1e-6, solve_quadrupoles=True, quad_idxs=[0, 2])
    a = O.DipoleSolverOracle([120.0] * 3, E, field_type="direct", **kw)
    a.compute(pos)
    b = O.DipoleSolverOracle([120.0] * 3, E, xi=0.4, field_type="polydisperse", **kw)
    b.compute(pos)
    for f in ("get_eff_polarizability", "get_dipoles", "get_quadrupoles"):
        np.testing.assert_allclose(getattr(a, f)(), getattr(b, f)(), rtol=1e-3, atol=1e-3)


@pytest.mark.parametrize("xi,rc", [(0.4, 9.3), (0.5, 7.43), (0.3, 12.4), (0.8, 1.0005)])
def test_library_tables_match_oracle(xi, rc):
    """The C++ tables behind the C-ABI (mpm_poly_quad_tables) against the
    oracle on the same nodes."""
    from cumpm_b200 import capi

    r, T = capi.poly_quad_tables(xi, rc)
    n = int(np.ceil((max(rc, 1.001) - 1.0) / 0.001)) + 1
    assert len(r) == n and r[0] == 0.0
    np.testing.assert_allclose(r[1:], 1.0 + np.arange(n - 1) * 0.001, rtol=0, atol=1e-12)
    _, W, _, sg = O.mono_real_tables(xi, r[1:], variant="poly")
    # the closed forms cancel terms of size xi^-10; the C++ groups them by
    # parity, the oracle term by term, so the two agree to that rounding
    for k in ("fq1", "fq2", "fq3", "gq1", "gq2", "gq3", "gq4"):
        np.testing.assert_allclose(T[k], W[k], rtol=1e-10, atol=1e-11 * np.abs(W[k]).max(), err_msg=k)
    assert T["gq1"][0] == T["gq4"][0] and abs(T["gq2"][0] - sg) <= 1e-15 * abs(sg)


def test_library_self_values_match_oracle():
    from cumpm_b200 import capi

    radii = np.array([0.8, 1.0, 1.2, 2.5, 4.0])
    for xi in (0.3, 0.5):
        np.testing.assert_allclose(capi.poly_quad_self(xi, radii), [O.poly_self_grad(a, xi) for a in radii],
                                   rtol=1e-14)


def test_library_table_arguments_are_checked():
    from cumpm_b200 import capi

    with pytest.raises(ValueError):
        capi.poly_quad_tables(-0.5, 7.0)
    with pytest.raises(ValueError):
        capi.poly_quad_self(0.5, [1.0, -1.0])


def _line_of_four():
    """The reference's field-level subset case: four unit spheres in a line
    10 apart, box 50, xi 0.4, quadrupoles on particles 0 and 2, self
    coefficient 1.5 + 0.1i, moments from the legacy seed 42."""
    d = 10.0
    pos = np.array([[0.0, 0, 0], [d, 0, 0], [2 * d, 0, 0], [3 * d, 0, 0]])
    rs = np.random.RandomState(42)
    P = rs.rand(4, 3) + 1j * rs.rand(4, 3)
    Q = rs.rand(2, 5) + 1j * rs.rand(2, 5)
    return pos, [5 * d] * 3, [0, 2], np.concatenate([P.ravel(), Q.ravel()]), np.full(4, 1.5 + 0.1j)


def test_reference_check_subset_field_matches_monodisperse():
    """Reference KAT at the field level: the polydisperse field with a
    quadrupole subset matches the monodisperse one to 1e-3
    (tests/test_electric_fields.py:158-223)."""
    pos, box, qi, X, sc = _line_of_four()
    m = O.MonoEwaldOperator(box, 1e-6, 0.4, True, qi)
    m.set_positions(pos)
    p = O.PolyEwaldOperator(box, 1e-6, 0.4, [1.0] * 4, True, qi)
    p.set_positions(pos)
    a, b = m.apply(X, sc), p.apply(X, sc)
    np.testing.assert_allclose(b[:12], a[:12], rtol=1e-3, atol=1e-3)
    np.testing.assert_allclose(b[12:], a[12:], rtol=1e-3, atol=1e-3)


def test_reference_check_bloch_wavevector_matches_monodisperse():
    """Reference KAT: with the Bloch wavevector (0.15, -0.22) the
    polydisperse field with quadrupoles on particles 0 and 2 matches the
    monodisperse one to 1e-3 (tests/test_electric_fields.py:226-284)."""
    pos = np.array([[0.0, 0, 0], [4.5, 0, 0], [9.0, 0, 0], [13.5, 0, 0]])
    box, qi, k = [18.0] * 3, [0, 2], (0.15, -0.22)
    rs = np.random.RandomState(123)
    P = rs.rand(4, 3) + 1j * rs.rand(4, 3)
    Q = rs.rand(2, 5) + 1j * rs.rand(2, 5)
    X, sc = np.concatenate([P.ravel(), Q.ravel()]), np.ones(4, complex)
    m = O.MonoEwaldOperator(box, 1e-6, 0.5, True, qi, bloch=k)
    m.set_positions(pos)
    p = O.PolyEwaldOperator(box, 1e-6, 0.5, [1.0] * 4, True, qi, bloch=k)
    p.set_positions(pos)
    a, b = m.apply(X, sc), p.apply(X, sc)
    np.testing.assert_allclose(b[:12], a[:12], rtol=1e-3, atol=1e-3)
    np.testing.assert_allclose(b[12:], a[12:], rtol=1e-3, atol=1e-3)
    # the wavevector is felt: without it the field moves by about 1.7e-3
    m0 = O.MonoEwaldOperator(box, 1e-6, 0.5, True, qi)
    m0.set_positions(pos)
    assert np.abs(m0.apply(X, sc) - a).max() > 5e-4
