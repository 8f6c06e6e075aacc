"""Field autotuner on the GPU: the pick's operator against the FP64 oracle
within the tuner's own error bound, overrides that leave the operator
unchanged, and the tuned dipole solver against the rule's."""
import numpy as np
import pytest

from oracle import mpm_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rand_c(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def apply(F, X, sc):
    import torch
    return F.apply(torch.tensor(X, device="cuda"), self_coef=torch.tensor(sc, device="cuda")).cpu().numpy()


def hex_layer(nx=14, ny=12, sp=2.4):
    pos = np.array([[(i + 0.5 * (j % 2)) * sp, j * np.sqrt(3) / 2 * sp, 0.0] for j in range(ny) for i in range(nx)])
    box = (max(pos[:, 0].max() + sp, 16.0), max(pos[:, 1].max() + sp * np.sqrt(3) / 2, 16.0), 60.0)
    return pos, box


def test_rule_tuning_is_the_rule_bit_for_bit():
    from cumpm_b200 import capi
    rng = np.random.default_rng(1)
    pos, box = hex_layer()
    N = len(pos)
    X, sc = rand_c(rng, 3 * N, 3), rand_c(rng, N, 3)
    F0 = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    F1 = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, tuning={"xi": 0.5})
    F0.set_positions(pos)
    F1.set_positions(pos)
    assert np.array_equal(apply(F0, X, sc), apply(F1, X, sc))


@pytest.mark.parametrize("tile", [(16, 8), (8, 16), (4, 8)])
def test_spread_tile_leaves_the_operator(tile):
    from cumpm_b200 import capi
    rng = np.random.default_rng(2)
    pos, box = hex_layer()
    pos[:, 2] = rng.uniform(-0.5, 0.5, len(pos))   # several z planes: the general spread kernel too
    N = len(pos)
    for M in (1, 3, 12):
        X, sc = rand_c(rng, 3 * N, M), rand_c(rng, N, M)
        F0 = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
        F1 = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, tuning={"xi": 0.5, "tile": tile})
        F0.set_positions(pos)
        F1.set_positions(pos)
        assert rel(apply(F1, X, sc), apply(F0, X, sc)) < 1e-13


@pytest.mark.parametrize("case", ["layer", "bulk"])
def test_autotune_pick_meets_its_bound(case):
    """The pick's operator differs from the oracle (the rule's operator) by
    at most its own error plus the rule's, both within the bound."""
    from cumpm_b200 import capi
    rng = np.random.default_rng(3)
    if case == "layer":
        pos, box = hex_layer()
    else:
        box = (22.0, 20.0, 24.0)
        pos = rng.uniform(0, 20, (40, 3))
    N = len(pos)
    M = 6
    pick = capi.autotune(capi.FIELD_MONO, box, 1e-6, 0.5, pos, M)
    assert pick["candidates"] >= 5 and pick["accepted"] >= 1
    assert pick["error"] <= pick["error_bound"]
    assert pick["error_bound"] == pytest.approx(max(1e-6, pick["error_rule"]))
    assert pick["apply_ms"] <= pick["apply_ms_rule"] * 1.0000001
    op = O.MonoEwaldOperator(box, 1e-6, 0.5, True)
    op.set_positions(pos)
    X, sc = rand_c(rng, 3 * N, 2), rand_c(rng, N, 2)
    ref = np.stack([op.apply(X[:, m], sc[:, m]) for m in range(2)], axis=1)
    F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, tuning=pick)
    F.set_positions(pos)
    # the error measure is normwise per column; the self terms (identical in
    # both) only make the comparison easier
    got = apply(F, X, sc)
    err = max(np.linalg.norm(got[:, m] - ref[:, m]) / np.linalg.norm(ref[:, m]) for m in range(2))
    assert err <= 3.0 * pick["error_bound"], (err, pick)


def test_grid_and_support_overrides_stay_accurate():
    """A grid rounded up to 2^a 3^b sizes and the support trimmed by one
    point: the operator stays within 10 tol of the oracle."""
    from cumpm_b200 import capi
    rng = np.random.default_rng(4)
    box = (22.0, 20.0, 24.0)
    pos = rng.uniform(0, 20, (30, 3))
    N = len(pos)
    op = O.MonoEwaldOperator(box, 1e-6, 0.5, True)
    op.set_positions(pos)
    X, sc = rand_c(rng, 3 * N, 2), rand_c(rng, N, 2)
    ref = np.stack([op.apply(X[:, m], sc[:, m]) for m in range(2)], axis=1)
    grid = [capi.tune_next_size(n, smooth23=True) for n in capi.tune_xi_candidates(capi.FIELD_MONO, box, 1e-6,
                                                                                      0.5)[0]["grid"]]
    for t in ({"xi": 0.5, "grid": grid}, {"xi": 0.5, "support": 8}):
        F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5, tuning=t)
        F.set_positions(pos)
        got = apply(F, X, sc)
        err = max(np.linalg.norm(got[:, m] - ref[:, m]) / np.linalg.norm(ref[:, m]) for m in range(2))
        assert err <= 2e-5, (t, err)


def test_autotune_polydisperse():
    from cumpm_b200 import capi
    rng = np.random.default_rng(5)
    radii = rng.uniform(1.0, 2.0, 30)
    box = (26.0, 26.0, 26.0)
    pos = rng.uniform(0, 26, (30, 3))
    pick = capi.autotune(capi.FIELD_POLY, box, 1e-5, 0.5, pos, 4, radius=radii)
    assert pick["error"] <= pick["error_bound"]
    F0 = capi.Field(capi.FIELD_POLY, box, 1e-5, 0.5, radius=radii)
    F1 = capi.Field(capi.FIELD_POLY, box, 1e-5, 0.5, radius=radii, tuning=pick)
    F0.set_positions(pos)
    F1.set_positions(pos)
    X, sc = rand_c(rng, 90, 2), rand_c(rng, 30, 2)
    a, b = apply(F1, X, sc), apply(F0, X, sc)
    err = max(np.linalg.norm(a[:, m] - b[:, m]) / np.linalg.norm(b[:, m]) for m in range(2))
    assert err <= 3.0 * pick["error_bound"], (err, pick)


def test_dipole_solver_autotune():
    """dipole_solver.autotune picks a field for the batch; the tuned solve
    agrees with the rule's to the accuracy both carry."""
    import cumpm_b200 as cuMPM
    pos, box = hex_layer(12, 10, 2.4)
    pos_nm = pos * 5.0
    box_nm = [b * 5.0 for b in box]
    w = np.linspace(0.3, 0.9, 4)
    eps = 4.0 - 1.8 ** 2 / (w ** 2 + 1j * w * 0.1)
    out = {}
    for tuned in (False, True):
        s = cuMPM.dipole_solver(box_nm, eps, radius=5.0, eps_m=1.77, tol=1e-6, quiet=True)
        s.set_solver_options(batch_all=True, refine=True)
        if tuned:
            pick = s.autotune(pos_nm)
            assert pick["error"] <= pick["error_bound"]
        s.compute(pos_nm)
        out[tuned] = np.asarray(s.get_dipoles())
    d = np.linalg.norm(out[True] - out[False]) / np.linalg.norm(out[False])
    assert d < 1e-4, d
