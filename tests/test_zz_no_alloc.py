"""The allocation-free field apply (mpm_field_apply_noalloc) through the C ABI.

It exists for callers that cannot allocate device memory while they solve
(their GPU memory belongs to another allocator, or their loop must not call
into the driver's allocator): its reciprocal-space grid is a static device
array of the library.  It must give the same fields as mpm_field_apply.
This file is collected after the operator and solver tests so that a
failure here leaves them already run; it passes alone in a fresh process and
after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call_noalloc(F, X, Y, sc, recip_fp32):
    import torch
    from cumpm_b200 import capi
    capi.check(capi.lib().mpm_field_apply_noalloc(
        F._h, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), X.shape[1], C.c_void_p(sc.data_ptr()), 0,
        int(recip_fp32), 0, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return Y


@pytest.mark.parametrize("recip_fp32", [False, True])
def test_noalloc_apply_matches_apply_twice(recip_fp32):
    import torch
    from cumpm_b200 import capi
    rng = np.random.default_rng(7)
    box = (20.0, 20.0, 20.0)
    pos = rng.uniform(0, 20, (14, 3))
    N, M = len(pos), 2
    F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    F.set_positions(pos)
    assert capi.lib().mpm_noalloc_scratch_bytes() == 16 << 20
    for call in range(2):  # the static grid keeps the previous call's contents
        X = torch.tensor(rng.standard_normal((3 * N, M)) + 1j * rng.standard_normal((3 * N, M)), device="cuda")
        S = torch.tensor(rng.standard_normal((N, M)) + 1j * rng.standard_normal((N, M)), device="cuda")
        ref = F.apply(X, self_coef=S, recip_fp32=recip_fp32).cpu().numpy()
        Y = torch.full_like(X, float("nan"))
        got = _call_noalloc(F, X, Y, S, recip_fp32).cpu().numpy()
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err < 1e-12, f"call {call}: rel err {err:.3e}"


def _fresh(kind):
    """A field of each kind, its positions set (per-frame data allocated)
    but never applied, so nothing has sized its own reciprocal grid yet."""
    from cumpm_b200 import capi
    rng = np.random.default_rng({"mono": 21, "poly": 22, "direct": 23}[kind])
    if kind == "mono":
        box = (20.0, 20.0, 20.0)
        pos = rng.uniform(0, 20, (14, 3))
        F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    elif kind == "poly":
        box = (26.0, 24.0, 28.0)
        pos = np.array([[2, 2, 2], [8, 3, 4], [14, 9, 5], [3, 15, 12], [18, 18, 18], [10, 20, 7.0]])
        F = capi.Field(capi.FIELD_POLY, box, 1e-6, 0.5, radius=[1.0, 1.3, 1.0, 1.6, 1.3, 1.0])
    else:
        pos = rng.uniform(0, 30, (12, 3))
        F = capi.Field(capi.FIELD_DIRECT, None, 1e-6, 0.5, radius=np.ones(12))
    F.set_positions(pos)
    return F, len(pos)


@pytest.mark.parametrize("kind", ["mono", "poly", "direct"])
def test_noalloc_first_call_on_a_fresh_field_allocates_nothing(kind):
    """Called before any mpm_field_apply on a new field, the entry point
    leaves the device's free memory where it was, and then agrees with
    mpm_field_apply.  A warm-up call on another field of the same kind loads
    the kernels first (module loading may take device memory)."""
    import torch
    rng = np.random.default_rng(9)
    W, Nw = _fresh(kind)
    F, N = _fresh(kind)
    M = 2
    mk = lambda n, r: torch.tensor(rng.standard_normal((r, M)) + 1j * rng.standard_normal((r, M)), device="cuda")
    Xw, Sw, Yw = mk(Nw, 3 * Nw), mk(Nw, Nw), torch.empty((3 * Nw, M), dtype=torch.complex128, device="cuda")
    X, S = mk(N, 3 * N), mk(N, N)
    got = {fp32: torch.full((3 * N, M), float("nan"), dtype=torch.complex128, device="cuda") for fp32 in (False, True)}
    for fp32 in (False, True):
        _call_noalloc(W, Xw, Yw, Sw, fp32)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for fp32 in (False, True):   # nothing is allocated inside this window, by torch or by the library
        _call_noalloc(F, X, got[fp32], S, fp32)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    for fp32 in (False, True):
        ref = F.apply(X, self_coef=S, recip_fp32=fp32).cpu().numpy()
        err = np.max(np.abs(got[fp32].cpu().numpy() - ref)) / np.max(np.abs(ref))
        assert err < 1e-12, f"fp32={fp32}: rel err {err:.3e}"


def test_noalloc_rejects_grid_beyond_static_scratch():
    import torch
    from cumpm_b200 import capi
    rng = np.random.default_rng(8)
    box = (60.0, 60.0, 60.0)
    pos = rng.uniform(0, 60, (20, 3))
    F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    F.set_positions(pos)
    M = 40  # 72^3 voxels x 3 x 40 columns of complex64 = 342 MiB > 16 MiB
    X = torch.zeros((60, M), dtype=torch.complex128, device="cuda")
    Y = torch.zeros_like(X)
    S = torch.ones((20, M), dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError, match="exceeds the 16777216-byte static scratch"):
        _call_noalloc(F, X, Y, S, True)
