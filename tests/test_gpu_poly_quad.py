"""Polydisperse quadrupoles on the GPU against the oracle, through the C ABI,
and the reference's two polydisperse quadrupole solver checks through the
drop-in ``dipole_solver`` (tests/test_dipole_solvers.py:190-290 of the
reference)."""
import numpy as np
import pytest

from oracle import mpm_oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.first_gpu_run]

BOX = (26.0, 24.0, 28.0)
POS = np.array([[2, 2, 2], [8, 3, 4], [14, 9, 5], [3, 15, 12], [18, 18, 18], [10, 20, 7.0]])
RADII = [1.0, 1.3, 1.0, 1.6, 1.3, 1.0]


def _field(qi, radii=RADII):
    from cumpm_b200 import capi

    return capi.Field(capi.FIELD_POLY, BOX, 1e-6, 0.5, radius=radii, quad_idxs=qi, solve_quads=True)


def _inputs(seed, N, Nq, M):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((3 * N + 5 * Nq, M)) + 1j * rng.standard_normal((3 * N + 5 * Nq, M))
    sc = rng.standard_normal((N, M)) + 1j * rng.standard_normal((N, M))
    return X, sc


@pytest.mark.parametrize("qi", [[0, 1, 2, 3, 4, 5], [0, 3, 4], [2]])
@pytest.mark.parametrize("recip_fp32", [False, True])
def test_operator_matches_oracle(qi, recip_fp32):
    import torch

    F = _field(qi)
    F.set_positions(POS)
    X, sc = _inputs(31, len(RADII), len(qi), 2)
    Y = F.apply(torch.tensor(X, device="cuda"), self_coef=torch.tensor(sc, device="cuda"),
                recip_fp32=recip_fp32).cpu().numpy()
    op = O.PolyEwaldOperator(BOX, 1e-6, 0.5, RADII, True, qi)
    op.set_positions(POS)
    tol = 1e-5 if recip_fp32 else 1e-9
    for m in range(X.shape[1]):
        ref = op.apply(X[:, m], sc[:, m])
        np.testing.assert_allclose(Y[:, m], ref, rtol=tol, atol=tol * np.abs(ref).max())


def test_real_and_reciprocal_parts_match_oracle():
    import torch

    qi = [0, 3, 4]
    F = _field(qi)
    F.set_positions(POS)
    X, sc = _inputs(32, len(RADII), len(qi), 1)
    Xt = torch.tensor(X, device="cuda")
    Yr = F.apply_part(Xt, 0).cpu().numpy()[:, 0]
    Ys = F.apply_part(Xt, 1, self_coef=torch.tensor(sc, device="cuda")).cpu().numpy()[:, 0]
    op = O.PolyEwaldOperator(BOX, 1e-6, 0.5, RADII, True, qi)
    op.set_positions(POS)
    _, (Er, Es, Gr, Gs) = op.apply(X[:, 0], sc[:, 0], split=True)
    rr = np.concatenate([Er.ravel(), Gr.ravel()])
    rs = np.concatenate([Es.ravel(), Gs.ravel()])
    np.testing.assert_allclose(Yr, rr, rtol=1e-9, atol=1e-10 * np.abs(rr).max())
    np.testing.assert_allclose(Ys, rs, rtol=1e-9, atol=1e-10 * np.abs(rs).max())


def test_subset_field_matches_monodisperse_field():
    """The reference's field-level subset check on the device: four unit
    spheres in a line, quadrupoles on particles 0 and 2, polydisperse
    against monodisperse to 1e-3 (tests/test_electric_fields.py:158-223)."""
    import torch
    from cumpm_b200 import capi

    d = 10.0
    pos = np.array([[0.0, 0, 0], [d, 0, 0], [2 * d, 0, 0], [3 * d, 0, 0]])
    box = (5 * d,) * 3
    rs = np.random.RandomState(42)
    P = rs.rand(4, 3) + 1j * rs.rand(4, 3)
    Q = rs.rand(2, 5) + 1j * rs.rand(2, 5)
    X = torch.tensor(np.concatenate([P.ravel(), Q.ravel()]).reshape(-1, 1), device="cuda")
    sc = torch.tensor(np.full((4, 1), 1.5 + 0.1j), device="cuda")
    Fp = capi.Field(capi.FIELD_POLY, box, 1e-6, 0.4, radius=[1.0] * 4, quad_idxs=[0, 2], solve_quads=True)
    Fm = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.4, quad_idxs=[0, 2], solve_quads=True)
    Fp.set_positions(pos)
    Fm.set_positions(pos)
    a = Fm.apply(X, self_coef=sc).cpu().numpy()[:, 0]
    b = Fp.apply(X, self_coef=sc).cpu().numpy()[:, 0]
    np.testing.assert_allclose(b, a, rtol=1e-3, atol=1e-3)


def _drude(omega, gamma, omega_p, eps_inf):
    return eps_inf - omega_p ** 2 / (omega ** 2 + 1j * omega * gamma)


def test_solver_subset_matches_monodisperse_solver():
    """Equal radii, quadrupoles on particles 0 and 2: the polydisperse
    quadrupole solve against the monodisperse one to 1e-3
    (tests/test_dipole_solvers.py:190-241 of the reference)."""
    import cumpm_b200 as cuMPM

    d = 10.0
    omega = np.linspace(1000, 7000, 3)
    eps = _drude(omega, 681, 12313, 4)
    pos = np.array([[0.0, 0, 0], [d, 0, 0], [2 * d, 0, 0], [3 * d, 0, 0]])
    box = np.array([5 * d] * 3)
    epsm = np.repeat(eps[:, None], 4, axis=1)
    out = {}
    for ft in ("monodisperse", "polydisperse"):
        s = cuMPM.dipole_solver(box, epsm, radius=1.0, eps_m=2.13, tol=1e-6, field_type=ft, quadrupoles=[0, 2],
                                precision="double", quiet=True)
        s.compute(pos)
        out[ft] = (s.get_eff_polarizability(), s.get_dipoles(), s.get_quadrupoles())
    assert out["polydisperse"][2].shape == (3, 2, 3, 5)
    for a, b in zip(out["monodisperse"], out["polydisperse"]):
        np.testing.assert_allclose(b, a, rtol=1e-3, atol=1e-3)


def test_solver_mixed_radii_matches_direct_in_large_box():
    """Mixed radii with quadrupoles on particles 0 and 2 in a 120^3 box:
    polydisperse Ewald against the direct sum to 1e-3
    (tests/test_dipole_solvers.py:244-290 of the reference)."""
    import cumpm_b200 as cuMPM

    d = 12.0
    omega = np.linspace(2000, 6000, 3)
    eps = _drude(omega, 681, 12313, 4)
    pos = np.array([[0.0, 0, 0], [d, 0, 0], [-d, 0, 0], [0, d, 0]])
    box = np.array([120.0] * 3)
    radii = [1.0, 1.2, 0.8, 1.1]
    epsm = np.repeat(eps[:, None], 4, axis=1)
    out = {}
    for ft, xi in (("direct", 0.5), ("polydisperse", 0.4)):
        s = cuMPM.dipole_solver(box, epsm, radius=radii, eps_m=1.8, xi=xi, tol=1e-6, field_type=ft,
                                quadrupoles=[0, 2], precision="double", quiet=True)
        s.compute(pos)
        out[ft] = (s.get_eff_polarizability(), s.get_dipoles(), s.get_quadrupoles())
    for a, b in zip(out["direct"], out["polydisperse"]):
        np.testing.assert_allclose(b, a, rtol=1e-3, atol=1e-3)


@pytest.mark.parametrize("solver_type", ["gmres", "bicgstab"])
def test_solver_matches_oracle_solver(solver_type):
    """The polydisperse quadrupole solve through dipole_solver against the
    oracle's driver on the same discretisation (tol 1e-9)."""
    import cumpm_b200 as cuMPM

    omega = np.array([0.5, 0.7])
    eps = 4.0 - 1.8 ** 2 / (omega ** 2 + 1j * omega * 0.1)
    rad_nm = np.array(RADII) * 2.0
    kw = dict(radius=rad_nm, eps_m=1.77, tol=1e-9, field_type="polydisperse", solver_type=solver_type)
    box_nm = np.array(BOX) * 2.0
    s = cuMPM.dipole_solver(box_nm, eps, quiet=True, precision="double", quadrupoles=[0, 3, 4], **kw)
    s.compute(POS * 2.0)
    o = O.DipoleSolverOracle(box_nm, eps, solve_quadrupoles=True, quad_idxs=[0, 3, 4], **kw)
    o.compute(POS * 2.0)
    for got, ref in ((s.get_dipoles(), o.get_dipoles()[0]), (s.get_quadrupoles(), o.get_quadrupoles()[0])):
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-7 * np.abs(ref).max())
