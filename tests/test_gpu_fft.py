"""The in-house batched line DFT (the grid transform of the spectral-Ewald
fields, replacing the reference's cuFFT plans) against numpy's FFT, through
the C-ABI entry mpm_line_fft: both kernels (two-pass in-register and general
multi-pass), both precisions, forward, inverse and the fused
forward-scale-inverse pass, for the line layouts the fields use (lines
contiguous: z axis; lines strided across the outer index: x axis)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

# two-pass splits in registers: 2 = 2x1, 16 = 4x4, 49 = 7x7, 80 = 10x8,
# 108 = 12x9, 112 = 14x8, 143 = 13x11, 256 = 16x16; with a Rader prime pass
# (p - 1 = A x B in registers): 34 = 2x17 (16 = 4x4, radix <= 8 class),
# 97 = 1x97 (96 = 12x8), 238 = 14x17 (16 = 4x4), 366 = 6x61 (60 = 10x6); with
# a streamed prime pass: 206 = 2x103 (102 has no such split); general only:
# 289 = 17*17
LENGTHS = [2, 16, 34, 49, 80, 97, 108, 112, 143, 206, 238, 256, 289, 366]
SPLITS = {2: (2, 1), 16: (4, 4), 34: (2, 17), 49: (7, 7), 80: (10, 8), 108: (12, 9), 112: (14, 8),
          143: (13, 11), 256: (16, 16), 97: (1, 97), 206: (2, 103), 238: (14, 17), 366: (6, 61)}


def run_case(n, layout, ncols, nouter, fp64, mode, general, seed=0, sb=4):
    from cumpm_b200 import capi

    rng = np.random.default_rng(seed + n)
    if layout == "z":
        shape, axis = (nouter, n, ncols), 1        # element stride ncols, line stride n*ncols
        es, os = ncols, n * ncols
    else:
        shape, axis = (n, nouter, ncols), 0        # element stride nouter*ncols, line stride ncols
        es, os = nouter * ncols, ncols
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    sz = (ncols + sb - 1) // sb
    sc = rng.uniform(0.5, 1.5, (n, nouter, sz))
    cdt, rdt = (torch.complex128, torch.float64) if fp64 else (torch.complex64, torch.float32)
    d = torch.tensor(a, dtype=cdt, device="cuda").contiguous()
    s = torch.tensor(sc, dtype=rdt, device="cuda").contiguous()
    split = capi.line_fft(d, n, es, ncols, os, nouter, mode=mode, scale=s if mode == 2 else None, sz=sz, sb=sb,
                          general=general)
    if mode == 0:
        ref = np.fft.fft(a, axis=axis)
    elif mode == 1:
        ref = np.fft.ifft(a, axis=axis) * n
    else:
        f = np.fft.fft(a, axis=axis)
        fac = sc[:, :, np.arange(ncols) // sb]                                    # (n, nouter, ncols)
        f = f * (fac.transpose(1, 0, 2) if layout == "z" else fac)
        ref = np.fft.ifft(f, axis=axis) * n
    got = d.cpu().numpy()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    return err, split


@pytest.mark.parametrize("fp64", [False, True])
@pytest.mark.parametrize("n", LENGTHS)
def test_line_fft_matches_numpy(n, fp64):
    tol = 1e-12 if fp64 else 2e-6
    for layout in ("z", "x"):
        for general in (False, True):
            for mode in (0, 1, 2):
                err, split = run_case(n, layout, 40, 3, fp64, mode, general)
                assert err < tol, (layout, general, mode, err)
                want = (0, 0) if general else SPLITS.get(n, (0, 0))
                if mode == 2 and want[1] > 16:
                    want = (0, 0)   # the fused pass has no streamed-prime variant
                assert split == want, (split, want)


# grid lengths the field autotuner proposes for the benchmark geometries
# (rule sizes rounded up to prime factors 2, 3, 5, 7 or to 2^a 3^b)
TUNER_LENGTHS = [81, 84, 90, 96, 120, 375, 378, 384]


@pytest.mark.parametrize("n", TUNER_LENGTHS)
def test_line_fft_tuner_lengths(n):
    for fp64 in (False, True):
        tol = 1e-12 if fp64 else 2e-6
        for layout in ("z", "x"):
            for mode in (0, 1, 2):
                err, _ = run_case(n, layout, 40, 3, fp64, mode, False)
                assert err < tol, (fp64, layout, mode, err)


@pytest.mark.parametrize("ncols", [1, 5, 17, 33, 70])
def test_line_fft_ragged_column_groups(ncols):
    """Column counts that leave the last CTA's column group partly empty, and
    fewer columns than one group (general kernel below 16 columns)."""
    for n in (108, 206, 366):
        for mode in (0, 1, 2):
            err, _ = run_case(n, "x", ncols, 5, True, mode, False, seed=ncols)
            assert err < 1e-12, (n, mode, err)


def test_line_fft_rejects_bad_arguments():
    from cumpm_b200 import capi

    d = torch.zeros(64, dtype=torch.complex64, device="cuda")
    with pytest.raises(ValueError):
        capi.line_fft(d, 8, 1, 8, 8, 1, mode=2)            # scale missing
    with pytest.raises(ValueError):
        capi.line_fft(d.to(torch.complex128), 8, 1, 8, 8, 1, mode=2,
                      scale=torch.ones(8, dtype=torch.float32, device="cuda"))
    with pytest.raises(ValueError):
        capi.line_fft(d, 0, 1, 8, 8, 1)
