"""Polydisperse spectral-Ewald field on the GPU (FIELD_POLY) against the
oracle's restatement of polydisperse_ewald_electric_field.cu, through the
C ABI."""
import numpy as np
import pytest

from oracle import mpm_oracle as O

pytestmark = pytest.mark.gpu


def packing(rng, n, box, rmin, rmax):
    """Random sequential addition of non-overlapping spheres (periodic)."""
    box = np.asarray(box, dtype=float)
    pos, rad = [], []
    while len(pos) < n:
        p = rng.uniform(0, 1, 3) * box
        a = rng.uniform(rmin, rmax)
        ok = True
        for q, b in zip(pos, rad):
            d = p - q
            d -= box * np.round(d / box)
            if np.sqrt(d @ d) < a + b:
                ok = False
                break
        if ok:
            pos.append(p)
            rad.append(a)
    return np.array(pos), np.array(rad)


def rand_c(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def gpu_apply(kind, box, tol, xi, pos, radii, X, sc=None, recip_fp32=False, real_fp32=False, mode=None,
              field_points=None):
    from cumpm_b200 import capi
    import torch
    F = capi.Field(kind, box, tol, xi, radius=radii, mode=capi.MODE_SOLVER_AX if mode is None else mode)
    if field_points is not None:
        F.set_field_points(field_points)
    F.set_positions(pos)
    Xt = torch.tensor(X, device="cuda")
    St = None if sc is None else torch.tensor(sc, device="cuda")
    return F.apply(Xt, self_coef=St, recip_fp32=recip_fp32, real_fp32=real_fp32).cpu().numpy(), F


@pytest.mark.parametrize("seed,n,box,rmin,rmax", [
    (1, 30, (30.0, 30.0, 30.0), 1.0, 2.5),
    (2, 60, (32.0, 28.0, 36.0), 1.0, 4.0),
    (3, 12, (20.0, 20.0, 20.0), 1.0, 1.0),
])
def test_operator_matches_oracle_fp64(seed, n, box, rmin, rmax):
    from cumpm_b200 import capi
    rng = np.random.default_rng(seed)
    pos, rad = packing(rng, n, box, rmin, rmax)
    M = 3
    X = rand_c(rng, 3 * n, M)
    sc = rand_c(rng, n, M)
    Y, F = gpu_apply(capi.FIELD_POLY, box, 1e-6, 0.5, pos, rad, X, sc)
    info = F.info()
    op = O.PolyEwaldOperator(box, 1e-6, 0.5, rad)
    op.set_positions(pos)
    assert info["grid"] == list(op.p.num_grid)
    assert info["stencil"] == op.p.P
    for m in range(M):
        ref = op.apply(X[:, m], sc[:, m])
        np.testing.assert_allclose(Y[:, m], ref, rtol=1e-10, atol=1e-11 * np.abs(ref).max())


def test_parts_match_oracle():
    from cumpm_b200 import capi
    import torch
    rng = np.random.default_rng(4)
    box = (30.0, 30.0, 30.0)
    pos, rad = packing(rng, 25, box, 1.0, 3.0)
    X = rand_c(rng, 75, 2)
    sc = rand_c(rng, 25, 2)
    F = capi.Field(capi.FIELD_POLY, box, 1e-6, 0.5, radius=rad)
    F.set_positions(pos)
    Xt = torch.tensor(X, device="cuda")
    St = torch.tensor(sc, device="cuda")
    Yr = F.apply_part(Xt, 0).cpu().numpy()
    Ys = F.apply_part(Xt, 1, self_coef=St).cpu().numpy()
    op = O.PolyEwaldOperator(box, 1e-6, 0.5, rad)
    op.set_positions(pos)
    for m in range(2):
        _, (Er, Es) = op.apply(X[:, m], sc[:, m], split=True)
        np.testing.assert_allclose(Yr[:, m], Er.ravel(), rtol=1e-10, atol=1e-11 * np.abs(Er).max())
        np.testing.assert_allclose(Ys[:, m], Es.ravel(), rtol=1e-10, atol=1e-11 * np.abs(Es).max())


def test_fp32_reciprocal_close_to_fp64():
    from cumpm_b200 import capi
    rng = np.random.default_rng(5)
    box = (30.0, 30.0, 30.0)
    pos, rad = packing(rng, 40, box, 1.0, 2.0)
    X = rand_c(rng, 120, 4)
    sc = rand_c(rng, 40, 4)
    Y64, _ = gpu_apply(capi.FIELD_POLY, box, 1e-6, 0.5, pos, rad, X, sc)
    Y32, _ = gpu_apply(capi.FIELD_POLY, box, 1e-6, 0.5, pos, rad, X, sc, recip_fp32=True, real_fp32=True)
    assert np.abs(Y32 - Y64).max() <= 1e-5 * np.abs(Y64).max()


def test_interaction_field_points_match_oracle():
    from cumpm_b200 import capi
    rng = np.random.default_rng(6)
    box = (24.0, 24.0, 24.0)
    pos, rad = packing(rng, 8, box, 1.0, 1.8)
    fp = rng.uniform(0, 24, (11, 3))
    X = rand_c(rng, 24, 1)
    Y, _ = gpu_apply(capi.FIELD_POLY, box, 1e-6, 0.5, pos, rad, X, mode=capi.MODE_INTERACTION, field_points=fp)
    op = O.PolyEwaldOperator(box, 1e-6, 0.5, rad, solver_ax=False)
    op.set_positions(pos, field_points=fp)
    ref = op.apply(X[:, 0])
    np.testing.assert_allclose(Y[:, 0], ref, rtol=1e-10, atol=1e-11 * np.abs(ref).max())


def test_unit_radius_matches_monodisperse():
    """Reference KAT on the GPU: polydisperse at radius 1 == monodisperse to 1e-5."""
    from cumpm_b200 import capi
    box = (20.0, 20.0, 20.0)
    pos = np.array([[0.0, 0, 0], [5, 0, 0], [10, 0, 0], [15, 0, 0]])
    X = np.zeros((12, 1), complex)
    X[0::3, 0] = 1.0
    sc = np.ones((4, 1), complex)
    Yp, _ = gpu_apply(capi.FIELD_POLY, box, 1e-6, 0.5, pos, [1.0] * 4, X, sc)
    Ym, _ = gpu_apply(capi.FIELD_MONO, box, 1e-6, 0.5, pos, None, X, sc)
    np.testing.assert_allclose(Yp, Ym, rtol=1e-5, atol=1e-5)


def drude(omega, gamma, omega_p, eps_inf):
    return eps_inf - omega_p ** 2 / (omega ** 2 + 1j * omega * gamma)


@pytest.mark.parametrize("solver_type", ["gmres", "bicgstab"])
def test_dipole_solver_polydisperse_matches_oracle(solver_type):
    import cumpm_b200 as cuMPM
    rng = np.random.default_rng(8)
    box = np.array([60.0, 60.0, 60.0])
    pos, rad = packing(rng, 24, box, 2.0, 5.0)
    eps = drude(np.linspace(0.4, 0.8, 3), 0.1, 1.8, 4.0)
    kw = dict(radius=list(rad), eps_m=1.77, tol=1e-9, solver_type=solver_type, field_type="polydisperse")
    s = cuMPM.dipole_solver(box, eps, quiet=True, precision="double", **kw)
    s.compute(pos)
    o = O.DipoleSolverOracle(box, eps, **kw)
    o.compute(pos)
    d_o = o.get_dipoles()[0]
    np.testing.assert_allclose(s.get_dipoles(), d_o, rtol=1e-6, atol=1e-7 * np.abs(d_o).max())
    a_o = o.get_eff_polarizability()
    np.testing.assert_allclose(s.get_eff_polarizability(), a_o, rtol=1e-6, atol=1e-9 * np.abs(a_o).max())


def test_auto_field_type_picks_polydisperse():
    import cumpm_b200 as cuMPM
    rng = np.random.default_rng(9)
    box = np.array([60.0, 60.0, 60.0])
    pos, rad = packing(rng, 16, box, 2.0, 4.0)
    eps = drude(np.array([0.5]), 0.1, 1.8, 4.0)
    kw = dict(radius=list(rad), eps_m=1.77, tol=1e-8, quiet=True, precision="double")
    a = cuMPM.dipole_solver(box, eps, field_type="auto", **kw)
    a.compute(pos)
    b = cuMPM.dipole_solver(box, eps, field_type="polydisperse", **kw)
    b.compute(pos)
    np.testing.assert_array_equal(a.get_dipoles(), b.get_dipoles())


def test_batched_mixed_precision_solve():
    """All frequencies x polarisations in one batch, fp32 operator inside
    fp64 refinement: every column reaches the fp64 true residual and the
    dipoles agree with the plain fp64 solve."""
    from cumpm_b200 import capi
    import torch
    rng = np.random.default_rng(10)
    box = (40.0, 40.0, 40.0)
    pos, rad = packing(rng, 80, box, 1.0, 4.0)
    N = len(pos)
    F = capi.Field(capi.FIELD_POLY, box, 1e-6, 0.5, radius=rad)
    F.set_positions(pos)
    eps = drude(np.linspace(0.2, 1.2, 8), 0.1, 1.8, 4.0) / 1.77
    K = 3
    M = len(eps) * K
    sc = np.stack([np.repeat(3.0 / (4 * np.pi * (eps - 1)), K) / a ** 3 for a in rad])
    B = np.zeros((3 * N, M), complex)
    for m in range(M):
        B[m % 3::3, m] = 1.0
    Bt = torch.tensor(B, device="cuda")
    St = torch.tensor(sc, device="cuda")
    X = torch.zeros_like(Bt)
    rep = F.batch_solve(Bt, X, St, tol=1e-6, refine=True)
    assert rep["num_converged"] == M
    R = Bt - F.apply(X, self_coef=St)
    rr = (torch.linalg.vector_norm(R, dim=0) / torch.linalg.vector_norm(Bt, dim=0)).max().item()
    assert rr <= 1e-6
    X64 = torch.zeros_like(Bt)
    F.batch_solve(Bt, X64, St, tol=1e-9, recip_fp32=False)
    d = (X - X64).abs().max().item() / X64.abs().max().item()
    assert d < 1e-5
