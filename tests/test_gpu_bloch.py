"""Bloch wavevector on the device field (the EELS Brillouin-zone sum)
against the oracle's restatement (shifted k in the k-space Green tensor, a
phase on every real-space pair), and the device EELS zone sum against the
oracle's EELS."""
import numpy as np
import pytest

from oracle import mpm_oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.first_gpu_run]


def rand_c(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


CASES = {
    # full layout; pruned multi-plane slab; single layer (pruned, column kernel with a Bloch shift)
    "bulk": ((20.0, 20.0, 20.0), lambda r: r.uniform(0, 20, (14, 3))),
    "slab_wrap": ((28.0, 30.0, 70.0), lambda r: np.c_[r.uniform(0, 28, 30), r.uniform(0, 30, 30),
                                                       r.uniform(-0.8, 0.8, 30)]),
    "layer": ((30.0, 26.0, 60.0), lambda r: np.c_[r.uniform(0, 30, 40), r.uniform(0, 26, 40), np.full(40, 0.3)]),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_mono_bloch_operator_matches_oracle(case):
    import torch
    from cumpm_b200 import capi
    box, gen = CASES[case]
    rng = np.random.default_rng(len(case))
    pos = gen(rng)
    N = len(pos)
    k = (np.pi / box[0] * 0.37, -np.pi / box[1] * 0.81)
    op = O.MonoEwaldOperator(box, 1e-6, 0.5, True, bloch=k)
    op.set_positions(pos)
    M = 3
    X, sc = rand_c(rng, 3 * N, M), rand_c(rng, N, M)
    ref = np.stack([op.apply(X[:, m], sc[:, m]) for m in range(M)], axis=1)
    F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    F.set_positions(pos)
    F.set_bloch(*k)
    Xt, St = torch.tensor(X, device="cuda"), torch.tensor(sc, device="cuda")
    Y = F.apply(Xt, self_coef=St).cpu().numpy()
    assert rel(Y, ref) < 1e-12, rel(Y, ref)
    Y32 = F.apply(Xt, self_coef=St, recip_fp32=True, real_fp32=True).cpu().numpy()
    assert rel(Y32, ref) < 2e-6
    # back to the plain operator
    F.set_bloch(0.0, 0.0)
    F0 = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    F0.set_positions(pos)
    assert np.array_equal(F.apply(Xt, self_coef=St).cpu().numpy(), F0.apply(Xt, self_coef=St).cpu().numpy())


def test_poly_bloch_operator_matches_oracle():
    import torch
    from cumpm_b200 import capi
    rng = np.random.default_rng(7)
    box = (30.0, 30.0, 30.0)
    pos, rad = [], []
    while len(pos) < 24:
        p, a = rng.uniform(0, 30, 3), rng.uniform(1.0, 2.5)
        if all(np.linalg.norm((p - q) - 30.0 * np.round((p - q) / 30.0)) >= a + b for q, b in zip(pos, rad)):
            pos.append(p)
            rad.append(a)
    pos, rad = np.array(pos), np.array(rad)
    k = (0.05, 0.02)
    op = O.PolyEwaldOperator(box, 1e-6, 0.5, rad, bloch=k)
    op.set_positions(pos)
    X, sc = rand_c(rng, 72, 2), rand_c(rng, 24, 2)
    ref = np.stack([op.apply(X[:, m], sc[:, m]) for m in range(2)], axis=1)
    F = capi.Field(capi.FIELD_POLY, box, 1e-6, 0.5, radius=rad)
    F.set_positions(pos)
    F.set_bloch(*k)
    Y = F.apply(torch.tensor(X, device="cuda"), self_coef=torch.tensor(sc, device="cuda")).cpu().numpy()
    assert rel(Y, ref) < 1e-10, rel(Y, ref)


def test_bloch_refused_with_quadrupoles_and_direct_fields():
    from cumpm_b200 import capi
    F = capi.Field(capi.FIELD_MONO, (20.0, 20.0, 20.0), 1e-6, 0.5, solve_quads=True)
    with pytest.raises(ValueError):
        F.set_bloch(0.1, 0.0)
    D = capi.Field(capi.FIELD_DIRECT, radius=np.ones(3))
    with pytest.raises(ValueError):
        D.set_bloch(0.1, 0.0)


def test_eels_zone_sum_matches_oracle():
    """Two zone points per axis, three frequencies, a small monodisperse
    array: loss and zone-averaged dipoles against the oracle's EELS
    (eels_solver.cu:495-881 restated)."""
    from cumpm_b200 import eels
    from oracle import mpm_eels as E
    rng = np.random.default_rng(3)
    box = np.array([60.0, 54.0, 60.0])   # every edge above twice the cutoff (8 radii at tol 1e-7)
    pos = np.c_[rng.uniform(0, 60, 6), rng.uniform(0, 54, 6), np.zeros(6)]
    pos = pos[np.argsort(pos[:, 0])]
    omega = [0.03, 0.05, 0.08]
    eps = 4.0 - 1.8 ** 2 / (np.array([0.6, 0.9, 1.2]) ** 2 + 0.1j * np.array([0.6, 0.9, 1.2]))
    kw = dict(eps_m=1.0, radius=3.0, xi=0.5, tol=1e-7)
    ref = E.EELSOracle(box, eps, omega, 0.5, field_type="monodisperse", asm=True, asm_n=(2, 2), **kw)
    z_ref, d_ref = ref.compute([11.0, 7.0], pos)
    s = eels.EELS(box, eps, omega, 0.5, field_type="monodisperse", asm_flag=True, asm_Nx=2, asm_Ny=2, quiet=True,
                  **kw)
    s.compute([11.0, 7.0], pos)
    z = s.get_eels()
    d = np.asarray(s.get_dipoles(physical=False))
    assert rel(z, z_ref) < 1e-5, (z, z_ref)
    assert rel(d, d_ref) < 1e-5
