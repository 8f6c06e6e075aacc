"""Field operator on the GPU (through the C ABI) against the FP64 oracle."""
import numpy as np
import pytest

from oracle import mpm_oracle as O

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rand_c(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def oracle_apply(op, X, sc):
    return np.stack([op.apply(X[:, m], None if sc is None else sc[:, m]) for m in range(X.shape[1])], axis=1)


def gpu_apply(F, X, sc, **kw):
    torch = _torch()
    Xt = torch.tensor(X, device="cuda")
    St = None if sc is None else torch.tensor(sc, device="cuda")
    return F.apply(Xt, self_coef=St, **kw).cpu().numpy()


CASES = {
    # name: (box, positions generator, tol, xi)
    "bulk": ((20.0, 20.0, 20.0), lambda r: r.uniform(0, 20, (14, 3)), 1e-6, 0.5),
    "bulk_tol3": ((24.0, 22.0, 26.0), lambda r: r.uniform(-3, 27, (20, 3)), 1e-3, 0.5),
    "slab": ((30.0, 26.0, 60.0), lambda r: np.c_[r.uniform(0, 30, 40), r.uniform(0, 26, 40), np.full(40, 0.3)],
             1e-6, 0.5),
    "slab_wrap": ((28.0, 30.0, 70.0),
                  lambda r: np.c_[r.uniform(0, 28, 30), r.uniform(0, 30, 30), r.uniform(-0.8, 0.8, 30)], 1e-6, 0.45),
    "bilayer": ((30.0, 30.0, 80.0), lambda r: np.c_[r.uniform(0, 30, 50), r.uniform(0, 30, 50),
                                                    np.where(r.uniform(size=50) < 0.5, 1.0, 4.5)], 1e-5, 0.5),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("M", [1, 3, 7])
def test_mono_solver_ax_fp64(case, M):
    from cumpm_b200 import capi
    box, gen, tol, xi = CASES[case]
    rng = np.random.default_rng(hash(case) % 1000 + M)
    pos = gen(rng)
    N = len(pos)
    op = O.MonoEwaldOperator(box, tol, xi, True)
    op.set_positions(pos)
    X = rand_c(rng, 3 * N, M)
    sc = rand_c(rng, N, M)
    ref = oracle_apply(op, X, sc)
    F = capi.Field(capi.FIELD_MONO, box, tol, xi)
    F.set_positions(pos)
    info = F.info()
    if case.startswith("slab") or case == "bilayer":
        assert info["pruned"] == 1
        # slab and slab_wrap (y lines of 32 and 33 points) take the fused
        # y-transform / Green-tensor pass; the bilayer's 37-point y lines
        # (prime) take the separate transforms and Toeplitz column kernel
        assert info["slab_fused"] == (0 if case == "bilayer" else 1)
        # the slab case is one plane (z = 0.3 for every particle): a single
        # layer, one stored z slot; slab_wrap spreads z over several planes
        assert info["single_layer"] == (1 if case == "slab" else 0)
        assert (info["z_slots"] == 1) == (case == "slab")
    Y = gpu_apply(F, X, sc)
    assert rel(Y, ref) < 1e-12, rel(Y, ref)
    # fp32 reciprocal / fp32 real space: single-precision agreement
    Y32 = gpu_apply(F, X, sc, recip_fp32=True, real_fp32=True)
    assert rel(Y32, ref) < 2e-6


def test_pruned_equals_full_layout():
    """The occupied-plane transform is the same discrete operator as the full
    3-D FFT: a slab evaluated both ways agrees to rounding."""
    from cumpm_b200 import capi
    rng = np.random.default_rng(11)
    box = (30.0, 26.0, 60.0)
    slab = np.c_[rng.uniform(0, 30, 25), rng.uniform(0, 26, 25), np.full(25, 0.4)]
    # one far particle spanning the box forces the full layout
    full = np.vstack([slab, [[15.0, 13.0, 30.0]]])
    X = rand_c(rng, 3 * 26, 2)
    X[-3:] = 0.0
    sc = rand_c(rng, 26, 2)
    Fs = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    Fs.set_positions(slab)
    Ff = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    Ff.set_positions(full)
    assert Fs.info()["pruned"] == 1 and Ff.info()["pruned"] == 0
    Ys = gpu_apply(Fs, X[:75], sc[:25])
    Yf = gpu_apply(Ff, X, sc)[:75]
    # the far particle has zero moment; its pairs with the slab are outside rc
    assert rel(Ys, Yf) < 1e-12


def test_jacobi_epilogue():
    from cumpm_b200 import capi
    rng = np.random.default_rng(2)
    box, gen, tol, xi = CASES["bulk"]
    pos = gen(rng)
    N = len(pos)
    op = O.MonoEwaldOperator(box, tol, xi, True)
    op.set_positions(pos)
    X, sc = rand_c(rng, 3 * N, 2), rand_c(rng, N, 2)
    ref = oracle_apply(op, X, sc)
    dinv = np.stack([O.jacobi_inverse(sc[:, m], N) for m in range(2)], axis=1)
    F = capi.Field(capi.FIELD_MONO, box, tol, xi)
    F.set_positions(pos)
    Y = gpu_apply(F, X, sc, jacobi=True)
    assert rel(Y, dinv * ref) < 1e-12


def test_split_real_plus_reciprocal():
    from cumpm_b200 import capi
    torch = _torch()
    rng = np.random.default_rng(4)
    box, gen, tol, xi = CASES["bulk"]
    pos = gen(rng)
    N = len(pos)
    F = capi.Field(capi.FIELD_MONO, box, tol, xi)
    F.set_positions(pos)
    X = torch.tensor(rand_c(rng, 3 * N, 3), device="cuda")
    sc = torch.tensor(rand_c(rng, N, 3), device="cuda")
    tot = F.apply(X, self_coef=sc)
    rec = F.apply_part(X, 0, self_coef=sc)
    real = F.apply_part(X, 1, self_coef=sc)
    np.testing.assert_allclose((rec + real).cpu().numpy(), tot.cpu().numpy(), rtol=1e-12, atol=1e-12)


def test_batch_columns_independent():
    from cumpm_b200 import capi
    rng = np.random.default_rng(6)
    box, gen, tol, xi = CASES["slab"]
    pos = gen(rng)
    N = len(pos)
    F = capi.Field(capi.FIELD_MONO, box, tol, xi)
    F.set_positions(pos)
    X, sc = rand_c(rng, 3 * N, 5), rand_c(rng, N, 5)
    Y = gpu_apply(F, X, sc)
    for m in (0, 3):
        Ym = gpu_apply(F, np.ascontiguousarray(X[:, m:m + 1]), np.ascontiguousarray(sc[:, m:m + 1]))
        assert rel(Ym[:, 0], Y[:, m]) < 1e-13


@pytest.mark.parametrize("quad_idxs", [None, [0, 2, 5]])
def test_mono_quadrupoles_fp64(quad_idxs):
    from cumpm_b200 import capi
    rng = np.random.default_rng(8)
    box = (20.0, 20.0, 20.0)
    pos = np.array([[1.0, 1, 1], [5.2, 1.3, 0.7], [3, 6, 2], [9, 9, 9], [12, 3, 15], [15, 14, 3], [4, 4, 5]])
    N = len(pos)
    qi = list(range(N)) if quad_idxs is None else quad_idxs
    op = O.MonoEwaldOperator(box, 1e-6, 0.5, True, quad_idxs=qi)
    op.set_positions(pos)
    rows = 3 * N + 5 * len(qi)
    X, sc = rand_c(rng, rows, 2), rand_c(rng, N, 2)
    ref = oracle_apply(op, X, sc)
    F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, quad_idxs=qi, solve_quads=True)
    F.set_positions(pos)
    assert F.info()["num_quads"] == len(qi)
    Y = gpu_apply(F, X, sc)
    assert rel(Y, ref) < 1e-11, rel(Y, ref)


@pytest.mark.parametrize("quads", [False, True])
def test_direct_fp64_fp32(quads):
    from cumpm_b200 import capi
    rng = np.random.default_rng(9)
    N = 37
    pos = rng.uniform(0, 15, (N, 3))
    pos[5] = pos[4] + [0.3, 0.0, 0.0]  # overlapping pair exercises the softening
    rad = rng.uniform(0.8, 1.4, N)
    qi = list(range(0, N, 3)) if quads else None
    op = O.DirectOperator(rad, True, qi)
    op.set_positions(pos)
    rows = 3 * N + (5 * len(qi) if quads else 0)
    X, sc = rand_c(rng, rows, 3), rand_c(rng, N, 3)
    ref = oracle_apply(op, X, sc)
    F = capi.Field(capi.FIELD_DIRECT, None, radius=rad, quad_idxs=qi, solve_quads=quads)
    F.set_positions(pos)
    assert rel(gpu_apply(F, X, sc), ref) < 1e-12
    assert rel(gpu_apply(F, X, sc, recip_fp32=True), ref) < 1e-5


def test_interaction_field_mono_and_direct():
    from cumpm_b200 import capi
    rng = np.random.default_rng(10)
    box = (30.0, 30.0, 30.0)
    pos = rng.uniform(0, 30, (15, 3))
    fp = rng.uniform(0, 30, (23, 3))
    X = rand_c(rng, 45, 2)
    op = O.MonoEwaldOperator(box, 1e-5, 0.5, solver_ax=False)
    op.set_positions(pos, fp)
    ref = oracle_apply(op, X, None)
    F = capi.Field(capi.FIELD_MONO, box, 1e-5, 0.5, mode=capi.MODE_INTERACTION)
    F.set_field_points(fp)
    F.set_positions(pos)
    assert rel(gpu_apply(F, X, None), ref) < 1e-12
    opd = O.DirectOperator(np.ones(15), solver_ax=False)
    opd.set_positions(pos, fp)
    refd = oracle_apply(opd, X, None)
    Fd = capi.Field(capi.FIELD_DIRECT, None, radius=np.ones(15), mode=capi.MODE_INTERACTION)
    Fd.set_field_points(fp)
    Fd.set_positions(pos)
    assert rel(gpu_apply(Fd, X, None), refd) < 1e-12


def test_hex_monolayer_operator_fp64():
    """The headline geometry (hexagonal monolayer with a vacuum gap) at a
    reduced size: pruned layout, cell-list pairs, FP64 agreement."""
    from cumpm_b200 import capi
    rng = np.random.default_rng(12)
    sp = 2.4
    pts = [[(i + 0.5 * (j % 2)) * sp, j * np.sqrt(3) / 2 * sp, 0.0] for j in range(12) for i in range(14)]
    pos = np.array(pts)
    box = (max(pos[:, 0].max() + sp, 16.0), max(pos[:, 1].max() + sp * np.sqrt(3) / 2, 16.0), 200.0)
    op = O.MonoEwaldOperator(box, 1e-6, 0.5, True)
    op.set_positions(pos)
    N = len(pos)
    X, sc = rand_c(rng, 3 * N, 2), rand_c(rng, N, 2)
    ref = oracle_apply(op, X, sc)
    F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    F.set_positions(pos)
    info = F.info()
    # every particle at z = 0: a single layer (one stored z slot); the 31-point
    # y lines (prime) take the column kernel, with the layer's z weights
    assert info["pruned"] == 1 and info["z_slots"] == 1 and info["single_layer"] == 1
    assert info["slab_fused"] == 0
    assert info["num_pairs"] == len(op.pi_)
    assert rel(gpu_apply(F, X, sc), ref) < 1e-12
