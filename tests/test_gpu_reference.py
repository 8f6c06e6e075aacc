"""Parity against the reference implementation itself: the reference's
CUDA extension compiled from its own sources into oracle/_ref (make -C
oracle ref).  Skipped when that build is not present."""
import glob
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


@pytest.fixture(scope="module")
def ref():
    if not glob.glob(os.path.join(REF_DIR, "_cuMPM*.so")):
        pytest.skip("reference build oracle/_ref not present")
    sys.path.insert(0, REF_DIR)
    try:
        import _cuMPM as R
    finally:
        sys.path.remove(REF_DIR)
    return R


def rand_c(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def ref_field(R, box, tol, xi, pos, P, sc, mode, quad_idxs=(), Q=None, field_points=None):
    ef = R.Monodisperse_Ewald_Electric_Field(box[0], box[1], box[2], tol, xi, mode, 1.0, Q is not None,
                                             list(quad_idxs), R.PrecisionMode.DOUBLE)
    if field_points is not None:
        ef.updateFieldCoordinates(*[list(field_points[:, d]) for d in range(3)])
    ef.updateParticleCoordinates(*[list(pos[:, d]) for d in range(3)])
    ef.updateDipolesComplex(*[list(f(P[:, d])) for d in range(3) for f in (np.real, np.imag)])
    if Q is not None:
        ef.updateQuadrupolesComplex(*[list(f(Q[:, c])) for c in range(5) for f in (np.real, np.imag)])
    ef.setSelfCoef(list(sc.real), list(sc.imag))
    ef.calculate()
    return np.asarray(ef.getEPointHost())


def test_operator_vs_reference_dipoles(ref):
    from cumpm_b200 import capi
    import torch
    rng = np.random.default_rng(1)
    for box, pos in [((20.0, 20.0, 20.0), rng.uniform(0, 20, (16, 3))),
                     ((30.0, 26.0, 60.0), np.c_[rng.uniform(0, 30, 40), rng.uniform(0, 26, 40), np.full(40, 0.3)])]:
        N = len(pos)
        P, sc = rand_c(rng, N, 3), rand_c(rng, N)
        E_ref = ref_field(ref, box, 1e-6, 0.5, pos, P, sc, ref.FieldCalcMode.SOLVER_AX)
        F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
        F.set_positions(pos)
        Y = F.apply(torch.tensor(P.reshape(-1, 1), device="cuda"),
                    self_coef=torch.tensor(sc.reshape(-1, 1), device="cuda")).cpu().numpy()[:, 0]
        np.testing.assert_allclose(Y, E_ref, rtol=1e-11, atol=1e-12 * np.abs(E_ref).max())


def test_operator_vs_reference_quadrupole_pairs(ref):
    """Quadrupoles with real-space pairs inside rc (the cross-coupling sign)."""
    from cumpm_b200 import capi
    import torch
    rng = np.random.default_rng(2)
    box = (20.0, 20.0, 20.0)
    pos = np.array([[0.0, 0, 0], [4.0, 0, 0], [8.0, 0, 0], [12.0, 0, 0], [3, 5, 1]])
    qi = [0, 2, 4]
    P, Q, sc = rand_c(rng, 5, 3), rand_c(rng, 3, 5), rand_c(rng, 5)
    E_ref = ref_field(ref, box, 1e-6, 0.5, pos, P, sc, ref.FieldCalcMode.SOLVER_AX, qi, Q)
    if isinstance(E_ref, tuple) or E_ref.dtype == object:
        E_ref = np.concatenate([np.ravel(np.asarray(e)) for e in E_ref])
    F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, quad_idxs=qi, solve_quads=True)
    F.set_positions(pos)
    X = np.concatenate([P.ravel(), Q.ravel()]).reshape(-1, 1)
    Y = F.apply(torch.tensor(X, device="cuda"), self_coef=torch.tensor(sc.reshape(-1, 1), device="cuda"))
    np.testing.assert_allclose(Y.cpu().numpy()[:, 0], np.ravel(E_ref), rtol=1e-10,
                               atol=1e-11 * np.abs(E_ref).max())


def test_interaction_field_vs_reference(ref):
    from cumpm_b200 import capi
    import torch
    rng = np.random.default_rng(3)
    box = (30.0, 30.0, 30.0)
    pos, fp = rng.uniform(0, 30, (12, 3)), rng.uniform(0, 30, (20, 3))
    P = rand_c(rng, 12, 3)
    E_ref = ref_field(ref, box, 1e-5, 0.5, pos, P, np.zeros(12, complex), ref.FieldCalcMode.INTERACTION_FIELD,
                      field_points=fp)
    F = capi.Field(capi.FIELD_MONO, box, 1e-5, 0.5, mode=capi.MODE_INTERACTION)
    F.set_field_points(fp)
    F.set_positions(pos)
    Y = F.apply(torch.tensor(P.reshape(-1, 1), device="cuda")).cpu().numpy()[:, 0]
    np.testing.assert_allclose(Y, np.ravel(E_ref), rtol=1e-11, atol=1e-12 * np.abs(E_ref).max())


@pytest.mark.parametrize("solver_type", ["gmres", "bicgstab"])
def test_dipole_solver_vs_reference(ref, solver_type):
    import cumpm_b200 as cuMPM
    sp = 12.0
    pts = [[(i + 0.5 * (j % 2)) * sp, j * np.sqrt(3) / 2 * sp, 0.0] for j in range(8) for i in range(10)]
    pos = np.array(pts)
    box = [pos[:, 0].max() + sp, max(pos[:, 1].max() + sp * 0.87, 100.0), 1000.0]
    omega = np.linspace(0.3, 0.9, 4)
    eps = 4.0 - 1.8 ** 2 / (omega ** 2 + 1j * omega * 0.1)
    args = dict(radius=[5.0], eps_m=1.77, xi=0.5, tol=1e-9, quiet=True, guess_type="derivative",
                solver_type=solver_type, field_type="monodisperse", E0=[], solve_quadrupoles=False, quad_idxs=[])
    R = ref.Dipole_Solver(list(box), [complex(e) for e in eps], precision=ref.PrecisionMode.DOUBLE, **args)
    R.compute(list(pos[:, 0]), list(pos[:, 1]), list(pos[:, 2]))
    dr = np.asarray(R.get_dipoles(True))
    s = cuMPM.dipole_solver(box, eps, radius=5.0, eps_m=1.77, tol=1e-9, quiet=True, solver_type=solver_type,
                            field_type="monodisperse", precision="double")
    s.compute(pos)
    d = s._solver.get_dipoles(True)
    np.testing.assert_allclose(d, dr, rtol=1e-6, atol=1e-7 * np.abs(dr).max())


def ref_poly_field(R, box, tol, xi, pos, radii, P, sc, mode, field_points=None):
    ef = R.Polydisperse_Ewald_Electric_Field(box[0], box[1], box[2], tol, xi, mode, list(map(float, radii)), False,
                                             [], R.PrecisionMode.DOUBLE)
    if field_points is not None:
        ef.updateFieldCoordinates(*[list(field_points[:, d]) for d in range(3)])
    ef.updateParticleCoordinates(*[list(pos[:, d]) for d in range(3)])
    ef.updateDipolesComplex(*[list(f(P[:, d])) for d in range(3) for f in (np.real, np.imag)])
    ef.setSelfCoef(list(sc.real), list(sc.imag))
    ef.calculate()
    return np.ravel(np.asarray(ef.getEPointHost()))


def nonoverlapping(rng, n, box, rmin, rmax):
    box = np.asarray(box, dtype=float)
    pos, rad = [], []
    while len(pos) < n:
        p = rng.uniform(0, 1, 3) * box
        a = rng.uniform(rmin, rmax)
        if all(np.linalg.norm((p - q) - box * np.round((p - q) / box)) >= a + b for q, b in zip(pos, rad)):
            pos.append(p)
            rad.append(a)
    return np.array(pos), np.array(rad)


@pytest.mark.parametrize("seed,rmax", [(11, 1.0), (12, 2.5), (13, 4.0)])
def test_polydisperse_operator_vs_reference(ref, seed, rmax):
    """Mixed radii (one class per particle) against the reference's own
    polydisperse field, fp64 reciprocal space."""
    from cumpm_b200 import capi
    import torch
    rng = np.random.default_rng(seed)
    box = (32.0, 30.0, 34.0)
    pos, rad = nonoverlapping(rng, 30, box, 1.0, rmax)
    P, sc = rand_c(rng, 30, 3), rand_c(rng, 30)
    E_ref = ref_poly_field(ref, box, 1e-6, 0.5, pos, rad, P, sc, ref.FieldCalcMode.SOLVER_AX)
    F = capi.Field(capi.FIELD_POLY, box, 1e-6, 0.5, radius=rad)
    F.set_positions(pos)
    Y = F.apply(torch.tensor(P.reshape(-1, 1), device="cuda"),
                self_coef=torch.tensor(sc.reshape(-1, 1), device="cuda")).cpu().numpy()[:, 0]
    np.testing.assert_allclose(Y, E_ref, rtol=1e-9, atol=1e-10 * np.abs(E_ref).max())


def test_polydisperse_interaction_vs_reference(ref):
    from cumpm_b200 import capi
    import torch
    rng = np.random.default_rng(14)
    box = (30.0, 30.0, 30.0)
    pos, rad = nonoverlapping(rng, 10, box, 1.0, 2.0)
    fp = rng.uniform(0, 30, (14, 3))
    P = rand_c(rng, 10, 3)
    E_ref = ref_poly_field(ref, box, 1e-6, 0.5, pos, rad, P, np.zeros(10, complex),
                           ref.FieldCalcMode.INTERACTION_FIELD, field_points=fp)
    F = capi.Field(capi.FIELD_POLY, box, 1e-6, 0.5, radius=rad, mode=capi.MODE_INTERACTION)
    F.set_field_points(fp)
    F.set_positions(pos)
    Y = F.apply(torch.tensor(P.reshape(-1, 1), device="cuda")).cpu().numpy()[:, 0]
    np.testing.assert_allclose(Y, E_ref, rtol=1e-9, atol=1e-10 * np.abs(E_ref).max())


def test_polydisperse_dipole_solver_vs_reference(ref):
    import cumpm_b200 as cuMPM
    rng = np.random.default_rng(15)
    box = [60.0, 60.0, 60.0]
    pos, rad = nonoverlapping(rng, 20, box, 2.0, 5.0)
    omega = np.linspace(0.3, 0.9, 3)
    eps = 4.0 - 1.8 ** 2 / (omega ** 2 + 1j * omega * 0.1)
    args = dict(radius=list(map(float, rad)), eps_m=1.77, xi=0.5, tol=1e-9, quiet=True, guess_type="derivative",
                solver_type="gmres", field_type="polydisperse", E0=[], solve_quadrupoles=False, quad_idxs=[])
    R = ref.Dipole_Solver(list(box), [complex(e) for e in eps], precision=ref.PrecisionMode.DOUBLE, **args)
    R.compute(list(pos[:, 0]), list(pos[:, 1]), list(pos[:, 2]))
    dr = np.asarray(R.get_dipoles(True))
    s = cuMPM.dipole_solver(box, eps, radius=list(rad), eps_m=1.77, tol=1e-9, quiet=True, field_type="polydisperse",
                            precision="double")
    s.compute(pos)
    d = s._solver.get_dipoles(True)
    np.testing.assert_allclose(d, dr, rtol=1e-6, atol=1e-7 * np.abs(dr).max())
