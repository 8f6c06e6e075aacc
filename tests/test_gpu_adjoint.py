"""Adjoint gradients on the GPU: the operator-derivative kernels against the
oracle (oracle/mpm_adjoint.py), the differentiable extinction loss against
the oracle and against central finite differences (step 1e-4 relative, the
criterion 1e-5), and the periodic gradient against the open-boundary
direct-sum gradient in a large box."""
import numpy as np
import pytest

from oracle import mpm_adjoint as A
from oracle import mpm_oracle as O

pytestmark = pytest.mark.gpu


def system(seed, box, radius, xi=0.5, margin=0.3):
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=float)
    prm = O.PolyParams(box, 1e-6, xi, radius)
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


def rand_c(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def smooth_coords(pos, box, rc, h_grid, step):
    """Coordinates (i, d) along which a central difference of +-step stays
    inside one linear segment of every pair-table lookup of particle i (the
    reference's tables interpolate linearly between nodes 0.001 apart, so the
    discrete operator has kinks there) and inside one grid rounding cell."""
    box = np.asarray(box, dtype=float)
    out = []
    for i in range(len(pos)):
        r = pos - pos[i]
        r -= box * np.round(r / box)
        d = np.sqrt(np.sum(r * r, axis=1))
        near = (d > 0) & (d < rc + 2 * step)
        seg = ((d[near] - 1.0) / 1e-3) % 1.0
        if np.any(np.minimum(seg, 1.0 - seg) * 1e-3 < 2 * step):
            continue
        for dd in range(3):
            f = (pos[i, dd] / h_grid[dd]) % 1.0
            if abs(f - 0.5) > 0.05:
                out.append((i, dd))
    return out


@pytest.mark.parametrize("kind", ["poly", "direct"])
def test_operator_gradient_matches_oracle(kind):
    from cumpm_b200 import capi
    import torch
    radius = np.array([1.0, 1.3, 1.1, 1.6, 1.2, 1.0, 2.0, 1.5])
    box = (22.0, 21.0, 23.0)
    pos, prm = system(11, box, radius)
    N, M = len(pos), 3
    rng = np.random.default_rng(12)
    lam, p = rand_c(rng, 3 * N, M), rand_c(rng, 3 * N, M)
    F = capi.Field(capi.FIELD_POLY if kind == "poly" else capi.FIELD_DIRECT, box, 1e-6, 0.5, radius=radius)
    F.set_positions(pos)
    gx, ga = F.grad(torch.tensor(lam, device="cuda"), torch.tensor(p, device="cuda"))
    gx, ga = gx.cpu().numpy(), ga.cpu().numpy()
    rx = np.zeros((N, 3), complex)
    ra = np.zeros(N, complex)
    op = A.make_operator(kind, box, pos, radius, 0.5, 1e-6)
    for m in range(M):
        if kind == "poly":
            bx, ba = A.poly_bilinear_grad(op, lam[:, m], p[:, m])
        else:
            bx, ba = A.direct_bilinear_grad(pos, radius, lam[:, m], p[:, m])
        rx += bx
        ra += ba
    np.testing.assert_allclose(gx, rx, rtol=0, atol=1e-9 * np.abs(rx).max())
    # radius derivatives of the pair tables are central differences (step
    # 1e-5 relative) on both sides
    np.testing.assert_allclose(ga, ra, rtol=0, atol=1e-7 * np.abs(ra).max())


def extinction_setup(kind, seed=21):
    radius = np.array([1.0, 1.3, 1.1, 1.6, 1.2, 1.0])
    box = (20.0, 20.0, 20.0)
    pos, prm = system(seed, box, radius)
    cfg = dict(box=box, omega=np.array([0.5, 0.7]), species=np.zeros(len(pos), int), eps_inf=[4.0], eps_m=1.77,
               E0=((1.0, 0.0, 0.0), (0.0, 1.0, 0.0)), wavenumber=np.array([1.0, 1.3]),
               field_type="ewald" if kind == "poly" else "direct", length_scale=1.0)
    return pos, radius, prm, cfg


@pytest.mark.parametrize("kind", ["poly", "direct"])
def test_extinction_gradient_matches_oracle(kind):
    import torch
    from cumpm_b200.adjoint import extinction_loss
    pos, radius, prm, cfg = extinction_setup(kind)
    N = len(pos)
    P = torch.tensor(pos, requires_grad=True)
    R = torch.tensor(radius, requires_grad=True)
    wp = torch.tensor([1.8], dtype=torch.float64, requires_grad=True)
    gm = torch.tensor([0.1], dtype=torch.float64, requires_grad=True)
    L = extinction_loss(P, R, wp, gm, **cfg)
    L.backward()
    # oracle with the same loss weights c = 4 pi k_w eps_m E0_k
    om, em = cfg["omega"], cfg["eps_m"]
    e = (4.0 - 1.8 ** 2 / (om ** 2 + 1j * om * 0.1)) / em
    eps_rel = np.repeat(e[:, None], N, axis=1)
    dwp = (-2 * 1.8 / (om ** 2 + 1j * om * 0.1)) / em
    dg = (1.8 ** 2 * 1j * om / (om ** 2 + 1j * om * 0.1) ** 2) / em
    deps = np.stack([np.repeat(dwp[:, None], N, axis=1), np.repeat(dg[:, None], N, axis=1)])
    E0 = np.array(cfg["E0"], complex)
    c = np.stack([np.stack([4 * np.pi * k * em * np.tile(E0[q], N) for q in range(2)]) for k in cfg["wavenumber"]])
    Lo, gx, ga, gt = A.loss_and_grad(kind, cfg["box"], pos, radius, eps_rel, deps, c, E0, params=prm)
    assert abs(L.item() - Lo) <= 1e-9 * abs(Lo)
    np.testing.assert_allclose(P.grad.numpy(), gx, rtol=0, atol=1e-7 * np.abs(gx).max())
    np.testing.assert_allclose(R.grad.numpy(), ga, rtol=0, atol=1e-7 * np.abs(ga).max())
    np.testing.assert_allclose([wp.grad.item(), gm.grad.item()], gt, rtol=1e-7)


@pytest.mark.parametrize("kind", ["poly", "direct"])
def test_extinction_gradient_matches_finite_differences(kind):
    """Central differences agree to 1e-5: steps of 1e-4 relative for radii and
    Drude parameters; for positions 1e-5 of the length unit, along
    coordinates whose step stays within one table segment of every pair."""
    import torch
    from cumpm_b200.adjoint import extinction_loss
    pos, radius, _, cfg = extinction_setup(kind, seed=22)
    cfg["solve_tol"] = 1e-13
    P = torch.tensor(pos, requires_grad=True)
    R = torch.tensor(radius, requires_grad=True)
    wp = torch.tensor([1.8], dtype=torch.float64, requires_grad=True)
    gm = torch.tensor([0.1], dtype=torch.float64, requires_grad=True)
    extinction_loss(P, R, wp, gm, **cfg).backward()

    def f(p_, r_, w_, g_):
        with torch.no_grad():
            return extinction_loss(torch.tensor(p_), torch.tensor(r_), torch.tensor([w_], dtype=torch.float64),
                                   torch.tensor([g_], dtype=torch.float64), **cfg).item()

    gx, ga = P.grad.numpy(), R.grad.numpy()
    h = 1e-5  # of the length unit (the smallest radius)
    prm = O.PolyParams(cfg["box"], 1e-6, 0.5, radius)
    coords = smooth_coords(pos, cfg["box"], prm.rc, prm.h, h)
    assert len(coords) >= 3
    for i, d in coords[:: max(1, len(coords) // 4)][:4]:
        pp, pm = pos.copy(), pos.copy()
        pp[i, d] += h
        pm[i, d] -= h
        fd = (f(pp, radius, 1.8, 0.1) - f(pm, radius, 1.8, 0.1)) / (2 * h)
        assert abs(fd - gx[i, d]) <= 1e-5 * np.abs(gx).max(), (i, d, fd, gx[i, d])
    for i in (1, 3):
        h = 1e-4 * radius[i]
        rp, rm = radius.copy(), radius.copy()
        rp[i] += h
        rm[i] -= h
        fd = (f(pos, rp, 1.8, 0.1) - f(pos, rm, 1.8, 0.1)) / (2 * h)
        assert abs(fd - ga[i]) <= 1e-5 * np.abs(ga).max(), (i, fd, ga[i])
    h = 1e-4 * 1.8
    fd = (f(pos, radius, 1.8 + h, 0.1) - f(pos, radius, 1.8 - h, 0.1)) / (2 * h)
    assert abs(fd - wp.grad.item()) <= 1e-5 * abs(wp.grad.item())
    h = 1e-4 * 0.1
    fd = (f(pos, radius, 1.8, 0.1 + h) - f(pos, radius, 1.8, 0.1 - h)) / (2 * h)
    assert abs(fd - gm.grad.item()) <= 1e-5 * abs(gm.grad.item())


def test_periodic_gradient_matches_direct_sum_in_large_box():
    """FP64 direct-sum gradient as the reference for the periodic one."""
    import torch
    from cumpm_b200.adjoint import extinction_loss
    d = 12.0
    pos = np.array([[0.0, 0.0, 0.0], [d, 0.0, 0.0], [-d, 0.0, 0.0], [0.0, d, 0.0]]) + 60.0
    radius = np.array([1.0, 1.2, 0.8, 1.1]) / 0.8
    out = {}
    for ft in ("ewald", "direct"):
        P = torch.tensor(pos, requires_grad=True)
        R = torch.tensor(radius, requires_grad=True)
        wp = torch.tensor([1.8], dtype=torch.float64, requires_grad=True)
        gm = torch.tensor([0.1], dtype=torch.float64, requires_grad=True)
        L = extinction_loss(P, R, wp, gm, box=(150.0, 150.0, 150.0), omega=np.array([0.5, 0.7]),
                            species=np.zeros(4, int), eps_inf=[4.0], eps_m=1.77, xi=0.4, field_type=ft)
        L.backward()
        out[ft] = (L.item(), P.grad.numpy(), R.grad.numpy(), wp.grad.item(), gm.grad.item())
    (Le, gxe, gae, we, ge), (Ld, gxd, gad, wd, gd) = out["ewald"], out["direct"]
    assert abs(Le - Ld) <= 1e-3 * abs(Ld)
    np.testing.assert_allclose(gxe, gxd, rtol=0, atol=5e-3 * np.abs(gxd).max())
    np.testing.assert_allclose(gae, gad, rtol=0, atol=5e-3 * np.abs(gad).max())
    # periodic images shift the small damping derivative most; compare the
    # Drude gradient as a vector
    np.testing.assert_allclose([we, ge], [wd, gd], rtol=0, atol=5e-3 * max(abs(wd), abs(gd)))


def test_two_species_lattice_gradient():
    """Rock-salt lattice of Drude spheres (a = 3) and constant-permittivity
    spheres (a = 2, eps 2.5): gradients of a few coordinates and of the
    Drude parameters against central differences."""
    import torch
    from cumpm_b200.adjoint import extinction_loss, wavenumber_from_ev
    n = 3
    a_nn = 7.0
    sites, species, rad = [], [], []
    for i in range(2 * n):
        for j in range(2 * n):
            for k in range(2 * n):
                sites.append([i * a_nn, j * a_nn, k * a_nn])
                s = (i + j + k) % 2
                species.append(0 if s == 0 else -1)
                rad.append(3.0 if s == 0 else 2.0)
    # a jittered lattice (a perfect one has vanishing forces, below the
    # resolution of a finite difference of the loss)
    rng = np.random.default_rng(31)
    pos = np.array(sites) + 0.37 + rng.uniform(-0.5, 0.5, (len(sites), 3))
    rad = np.array(rad)
    species = np.array(species)
    box = (2 * n * a_nn,) * 3
    omega = np.linspace(0.3, 1.0, 4)
    cfg = dict(box=box, omega=omega, species=species, eps_inf=[4.0], eps_m=1.77,
               eps_const=np.where(species < 0, 2.5, 0.0), wavenumber=wavenumber_from_ev(omega, 1.77),
               length_scale=2.0, xi=0.5, tol=1e-6, solve_tol=1e-13)
    P = torch.tensor(pos, requires_grad=True)
    R = torch.tensor(rad, requires_grad=True)
    wp = torch.tensor([1.8], dtype=torch.float64, requires_grad=True)
    gm = torch.tensor([0.1], dtype=torch.float64, requires_grad=True)
    extinction_loss(P, R, wp, gm, **cfg).backward()

    def f(p_, r_, w_, g_):
        with torch.no_grad():
            return extinction_loss(torch.tensor(p_), torch.tensor(r_), torch.tensor([w_], dtype=torch.float64),
                                   torch.tensor([g_], dtype=torch.float64), **cfg).item()

    gx = P.grad.numpy()
    prm = O.PolyParams(np.asarray(box) / 2.0, 1e-6, 0.5, rad / 2.0)
    step = 1e-5                      # of the length unit (the smallest radius, 2)
    safe = smooth_coords(pos / 2.0, np.asarray(box) / 2.0, prm.rc, prm.h, step)
    big = sorted(safe, key=lambda t: -abs(gx[t]))
    for i, d in big[:2] + big[len(big) // 2:len(big) // 2 + 1]:
        h = step * 2.0
        pp, pm = pos.copy(), pos.copy()
        pp[i, d] += h
        pm[i, d] -= h
        fd = (f(pp, rad, 1.8, 0.1) - f(pm, rad, 1.8, 0.1)) / (2 * h)
        assert abs(fd - gx[i, d]) <= 1e-5 * np.abs(gx).max(), (i, d, fd, gx[i, d])
    h = 1e-4 * 1.8
    fd = (f(pos, rad, 1.8 + h, 0.1) - f(pos, rad, 1.8 - h, 0.1)) / (2 * h)
    assert abs(fd - wp.grad.item()) <= 1e-5 * abs(wp.grad.item())
    h = 1e-4 * 0.1
    fd = (f(pos, rad, 1.8, 0.1 + h) - f(pos, rad, 1.8, 0.1 - h)) / (2 * h)
    assert abs(fd - gm.grad.item()) <= 1e-5 * abs(gm.grad.item())
