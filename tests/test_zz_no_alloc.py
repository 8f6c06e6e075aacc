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
