"""numpy restatements of the index algebra the in-house line transforms use
(mpm_fft.cu), checked against numpy's FFT on the CPU: the two-pass Stockham
split n = r1 * r2, the fused forward-scale-inverse pass (the forward pass-2
outputs of butterfly j are the inputs of the first inverse butterfly j), and
the Rader prime pass with its tables (primitive root g, a_q = x[g^-q],
y[g^m] = x[0] + (a (*) b)_m, Bh = DFT_N(b) / N, DFT_N split as A * B)."""
import numpy as np
import pytest


def W(n, t, inv=False):
    return np.exp((2j if inv else -2j) * np.pi * np.asarray(t) / n)


def two_pass(x, r1, r2, inv=False):
    """Pass 1 (Ns = 1): butterfly j < r2 reads x[j + q r2], writes S[j r1 + p];
    pass 2 (Ns = r1): butterfly j < r1 reads S[j + q r1] W_n^(q j), writes
    y[p r1 + j]."""
    n = r1 * r2
    S = np.empty(n, complex)
    for j in range(r2):
        v = x[j + r2 * np.arange(r1)]
        S[j * r1 + np.arange(r1)] = np.fft.ifft(v) * r1 if inv else np.fft.fft(v)
    y = np.empty(n, complex)
    for j in range(r1):
        q = np.arange(r2)
        v = S[j + q * r1] * W(n, q * j, inv)
        y[q * r1 + j] = np.fft.ifft(v) * r2 if inv else np.fft.fft(v)
    return y


@pytest.mark.parametrize("r1,r2", [(10, 8), (12, 9), (16, 16), (7, 7), (2, 1)])
def test_two_pass_split(r1, r2):
    rng = np.random.default_rng(r1 * 31 + r2)
    x = rng.standard_normal(r1 * r2) + 1j * rng.standard_normal(r1 * r2)
    np.testing.assert_allclose(two_pass(x, r1, r2), np.fft.fft(x), atol=1e-12)
    np.testing.assert_allclose(two_pass(x, r1, r2, True), np.fft.ifft(x) * r1 * r2, atol=1e-12)


@pytest.mark.parametrize("r1,r2", [(12, 9), (10, 8)])
def test_fused_forward_scale_inverse(r1, r2):
    """Forward pass 2 leaves y[p r1 + j] (p < r2) with thread j; an inverse
    transform whose first radix is r2 has butterfly j reading exactly
    y[j + p r1]: scale and run it in place, then the inverse radix-r1 pass
    (Ns = r2) reads S[j + q r2] W_n^(-q j) and writes x[p r2 + j]."""
    n = r1 * r2
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    sc = rng.uniform(0.5, 1.5, n)
    y = two_pass(x, r1, r2)
    S = np.empty(n, complex)
    for j in range(r1):
        p = np.arange(r2)
        v = y[p * r1 + j] * sc[p * r1 + j]
        S[j * r2 + p] = np.fft.ifft(v) * r2
    out = np.empty(n, complex)
    for j in range(r2):
        q = np.arange(r1)
        v = S[j + q * r2] * W(n, q * j, True)
        out[q * r2 + j] = np.fft.ifft(v) * r1
    np.testing.assert_allclose(out, np.fft.ifft(np.fft.fft(x) * sc) * n, atol=1e-11)


def primitive_root(p):
    fac = [d for d in range(2, p) if (p - 1) % d == 0 and all(d % e for e in range(2, d))]
    return next(g for g in range(2, p) if all(pow(g, (p - 1) // f, p) != 1 for f in fac))


def rader(x, A, B, inv=False):
    p = len(x)
    N = p - 1
    assert A * B == N
    g = primitive_root(p)
    gp = [pow(g, s, p) for s in range(N)]
    pin = [gp[(N - q) % N] for q in range(N)]            # a_q = x[g^-q]
    pout = gp                                             # y[g^m]
    b = W(p, np.array(gp), inv)                           # b_s = W_p^(g^s)
    Bh = np.fft.fft(b) / N
    a = x[pin]
    # DFT_N(a): q = B q1 + q2, k = k1 + A k2
    T = np.empty((B, A), complex)
    for q2 in range(B):
        T[q2] = np.fft.fft(a[B * np.arange(A) + q2]) * W(N, q2 * np.arange(A))
    Ah = np.empty(N, complex)
    for k1 in range(A):
        Ah[k1 + A * np.arange(B)] = np.fft.fft(T[:, k1])
    C = Ah * Bh
    # inverse DFT_N: k = k1 + A k2, m = m1 + B m2
    D = np.empty((B, A), complex)
    for k1 in range(A):
        D[:, k1] = np.fft.ifft(C[k1 + A * np.arange(B)]) * B * W(N, np.arange(B) * k1, True)
    c = np.empty(N, complex)
    for m1 in range(B):
        c[m1 + B * np.arange(A)] = np.fft.ifft(D[m1]) * A
    y = np.empty(p, complex)
    y[0] = x[0] + Ah[0]
    y[np.array(pout)] = x[0] + c
    return y


@pytest.mark.parametrize("p,A,B", [(17, 4, 4), (61, 10, 6), (97, 12, 8), (101, 10, 10)])
def test_rader_prime_pass(p, A, B):
    rng = np.random.default_rng(p)
    x = rng.standard_normal(p) + 1j * rng.standard_normal(p)
    np.testing.assert_allclose(rader(x, A, B), np.fft.fft(x), atol=1e-11)
    np.testing.assert_allclose(rader(x, A, B, True), np.fft.ifft(x) * p, atol=1e-11)
