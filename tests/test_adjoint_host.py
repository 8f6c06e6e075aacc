"""The adjoint oracle (oracle/mpm_adjoint.py) against central finite
differences of its own loss: positions, radii and Drude parameters, for the
polydisperse Ewald operator and the open-boundary direct sum.  No GPU."""
import numpy as np
import pytest

from oracle import mpm_adjoint as A
from oracle import mpm_oracle as O


def system(seed, box, radius, margin=0.3):
    """Non-overlapping positions away from the grid's rounding boundaries
    (so that finite differences do not cross a support shift)."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=float)
    prm = O.PolyParams(box, 1e-6, 0.5, radius)
    pos = []
    while len(pos) < len(radius):
        p = rng.uniform(0, 1, 3) * box
        f = (p / prm.h) % 1.0
        if np.any(np.abs(f - 0.5) < 0.05):
            continue
        k = len(pos)
        if all(np.linalg.norm((p - q) - box * np.round((p - q) / box)) >= radius[k] + radius[j] + margin
               for j, q in enumerate(pos)):
            pos.append(p)
    return np.array(pos), prm


def drude_rel(om, wp, gam, einf, em):
    return (einf - wp ** 2 / (om ** 2 + 1j * om * gam)) / em


def problem(N, seed):
    rng = np.random.default_rng(seed + 100)
    om = np.array([0.5, 0.7])
    wp, gam, einf, em = 1.8, 0.1, 4.0, 1.77
    e = drude_rel(om, wp, gam, einf, em)
    eps_rel = np.repeat(e[:, None], N, axis=1)
    de_dwp = (-2 * wp / (om ** 2 + 1j * om * gam)) / em
    de_dg = (wp ** 2 * 1j * om / (om ** 2 + 1j * om * gam) ** 2) / em
    deps = np.stack([np.repeat(de_dwp[:, None], N, axis=1), np.repeat(de_dg[:, None], N, axis=1)])
    E0 = np.array([[1, 0, 0], [0, 1, 0]], complex)
    c = rng.standard_normal((2, 2, 3 * N)) + 1j * rng.standard_normal((2, 2, 3 * N))
    return om, (wp, gam, einf, em), eps_rel, deps, E0, c


@pytest.mark.parametrize("kind", ["poly", "direct"])
def test_adjoint_oracle_matches_finite_differences(kind):
    radius = np.array([1.0, 1.3, 1.1, 1.6, 1.2, 1.0])
    box = (20.0, 20.0, 20.0)
    pos, prm = system(3, box, radius)
    N = len(pos)
    om, (wp, gam, einf, em), eps_rel, deps, E0, c = problem(N, 3)
    L, gx, ga, gt = A.loss_and_grad(kind, box, pos, radius, eps_rel, deps, c, E0, params=prm)

    def f(P, R, ER):
        return A.loss_and_grad(kind, box, P, R, ER, deps, c, E0, params=prm, grad=False)[0]

    h = 1e-4
    for i, d in [(0, 0), (1, 2), (3, 1), (5, 0)]:
        Pp, Pm = pos.copy(), pos.copy()
        Pp[i, d] += h
        Pm[i, d] -= h
        fd = (f(Pp, radius, eps_rel) - f(Pm, radius, eps_rel)) / (2 * h)
        assert abs(fd - gx[i, d]) <= 1e-5 * np.abs(gx).max(), (i, d, fd, gx[i, d])
    for i in range(N):
        hr = 1e-4 * radius[i]
        Rp, Rm = radius.copy(), radius.copy()
        Rp[i] += hr
        Rm[i] -= hr
        fd = (f(pos, Rp, eps_rel) - f(pos, Rm, eps_rel)) / (2 * hr)
        assert abs(fd - ga[i]) <= 1e-5 * np.abs(ga).max(), (i, fd, ga[i])
    for t, (dwp, dg) in enumerate([(1e-4 * wp, 0.0), (0.0, 1e-4 * gam)]):
        Ep = np.repeat(drude_rel(om, wp + dwp, gam + dg, einf, em)[:, None], N, axis=1)
        Em = np.repeat(drude_rel(om, wp - dwp, gam - dg, einf, em)[:, None], N, axis=1)
        fd = (f(pos, radius, Ep) - f(pos, radius, Em)) / (2 * (dwp + dg))
        assert abs(fd - gt[t]) <= 1e-5 * abs(gt[t]), (t, fd, gt[t])


def test_adjoint_oracle_ewald_gradient_matches_direct_in_large_box():
    """The periodic (polydisperse Ewald) gradient tends to the open-boundary
    direct-sum gradient in a large box (cf. tests/test_dipole_solvers.py:247)."""
    d = 12.0
    pos = np.array([[0.0, 0.0, 0.0], [d, 0.0, 0.0], [-d, 0.0, 0.0], [0.0, d, 0.0]]) + 60.0
    radius = np.array([1.0, 1.2, 0.8, 1.1]) / 0.8
    box = (150.0, 150.0, 150.0)
    N = len(pos)
    om, _, eps_rel, deps, E0, c = problem(N, 5)
    prm = O.PolyParams(box, 1e-6, 0.4, radius)
    Le, gxe, gae, gte = A.loss_and_grad("poly", box, pos, radius, eps_rel, deps, c, E0, xi=0.4, params=prm)
    Ld, gxd, gad, gtd = A.loss_and_grad("direct", box, pos, radius, eps_rel, deps, c, E0)
    assert abs(Le - Ld) <= 1e-3 * abs(Ld)
    np.testing.assert_allclose(gxe, gxd, rtol=0, atol=5e-3 * np.abs(gxd).max())
    np.testing.assert_allclose(gae, gad, rtol=0, atol=5e-3 * np.abs(gad).max())
    np.testing.assert_allclose(gte, gtd, rtol=5e-3)
