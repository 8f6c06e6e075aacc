"""CPU oracle for the adjoint (gradient) of a spectral loss of the dipole solve.

TEST INFRASTRUCTURE ONLY: the checker for ``cumpm_b200.adjoint``; only
``tests/`` may import it.

The reference has no gradients (its parity is unpinned there); this module
restates, in float64 numpy, the derivative of the reference's own discrete
operators so that the GPU gradients can be checked against it, and it is
itself checked against central finite differences of the loss
(``tests/test_adjoint_host.py``).

Loss, per frequency w and incident field k (the extinction cross-section
C_ext = 4 pi k_w sum_i Im(E0_k^* . p_i), examples/mpm_hex_monolayer_sweep.py:
117-119, with p = eps_m L0^3 p~ the physical dipoles):

    L = sum_{w,k} Im( c_{w,k}^H p_{w,k} ),   A_w p_{w,k} = E0_k

A_w = G(x, a) + diag(s_w) with s_i = 3 / (4 pi (eps_i/eps_m - 1) a_i^3) and
G the field operator in SOLVER_AX mode (its self value included).  G is
complex-symmetric (real symmetric kernels, no Bloch phase), so the adjoint
solve reuses A_w:

    A_w lam_{w,k} = conj(c_{w,k}),   dL/dtheta = -sum Im( lam^T (dA/dtheta) p )

with dA/dtheta for positions and radii from the derivative of the operator's
pieces (reciprocal-space weights, real-space pair tables, self values) and
for the permittivity parameters from ds_i/deps_i.

All lengths are in units of a fixed L0 (the smallest radius of the forward
point); the discretisation (grid, support, eta, cutoff, table nodes) is the
one of the forward point and is held fixed.
"""
from __future__ import annotations

import math

import numpy as np

from . import mpm_oracle as O

PI = math.pi

# ---------------------------------------------------------------------------
# Polydisperse spreading weights and their derivatives
# (spread_precalcs_kernel_polydisperse, polydisperse_ewald_electric_field.cu:189-263)
# ---------------------------------------------------------------------------


def poly_weight_derivs(params: O.PolyParams, pos, radius):
    """idx (n,P^3), w (n,P^3,3), dw/dx (n,P^3,3c,3e), dw/da (n,P^3,3).

    w_c = F(d, a) g_c with g = (grid node) - (particle), d = |g|, so
    dw_c/dx_e = -(F delta_ce + F_d g_c g_e / d) and dw_c/da = F_a g_c.
    """
    pos = np.asarray(pos, dtype=np.float64)
    radius = np.asarray(radius, dtype=np.float64)
    h, xi, eta = params.h, params.xi, params.eta
    N = params.num_grid
    g0 = O.c_round(pos / h)
    d0 = g0 * h - pos
    o = params.offsets
    ox, oy, oz = np.meshgrid(o, o, o, indexing="ij")
    off = np.stack([ox.ravel(), oy.ravel(), oz.ravel()], axis=1)
    g = d0[:, None, :] + off[None, :, :] * h[None, None, :]
    d = np.sqrt(np.sum(g * g, axis=-1))
    a = radius[:, None]
    x2 = xi * xi
    C = 3.0 / (8.0 * math.sqrt(2.0) * PI ** 1.5 * math.sqrt(eta) * xi)
    far = d >= 1e-6
    ds = np.where(far, d, 1.0)
    ep = np.exp(-2.0 * (ds + a) ** 2 * x2 / eta)
    em = np.exp(-2.0 * (ds - a) ** 2 * x2 / eta)
    tp = (eta + 4.0 * a * x2 * ds) * ep
    tm = (eta - 4.0 * a * x2 * ds) * em
    tp_d = 4.0 * a * x2 * ep + (eta + 4.0 * a * x2 * ds) * (-4.0 * (ds + a) * x2 / eta) * ep
    tm_d = -4.0 * a * x2 * em + (eta - 4.0 * a * x2 * ds) * (-4.0 * (ds - a) * x2 / eta) * em
    tp_a = 4.0 * x2 * ds * ep + (eta + 4.0 * a * x2 * ds) * (-4.0 * (ds + a) * x2 / eta) * ep
    tm_a = -4.0 * x2 * ds * em + (eta - 4.0 * a * x2 * ds) * (4.0 * (ds - a) * x2 / eta) * em
    F = C / (a ** 3 * ds ** 3) * (tp - tm)
    F_d = C / a ** 3 * ((tp_d - tm_d) / ds ** 3 - 3.0 * (tp - tm) / ds ** 4)
    F_a = C / ds ** 3 * (-3.0 / a ** 4 * (tp - tm) + (tp_a - tm_a) / a ** 3)
    kn = 8.0 * math.sqrt(2.0) * xi ** 5 * np.exp(-2.0 * a * x2 / eta) / (PI ** 1.5 * eta ** 2.5)
    kn_a = kn * (-2.0 * x2 / eta)
    F = np.where(far, F, kn)
    F_d = np.where(far, F_d, 0.0)
    F_a = np.where(far, F_a, kn_a)
    w = F[..., None] * g
    eye = np.eye(3)
    dw_dx = -(F[..., None, None] * eye + (F_d / ds)[..., None, None] * g[..., :, None] * g[..., None, :])
    dw_da = F_a[..., None] * g
    gi = np.mod(g0[:, None, :] + off[None, :, :], N[None, None, :])
    idx = (gi[..., 0] * N[1] + gi[..., 1]) * N[2] + gi[..., 2]
    return idx, w, dw_dx, dw_da


# ---------------------------------------------------------------------------
# Pair-table lookup with derivatives
# (interpolate_table_gpu_polydisperse, :170-187; helper_compute_pair_tables, :1434-1627)
# ---------------------------------------------------------------------------


def _node_values(rnodes, a, b, xi):
    """fd1, fd2 at table nodes; node 0 (r = 0) is the self value."""
    rn = np.asarray(rnodes, dtype=np.float64)
    f1 = np.empty_like(rn)
    f2 = np.empty_like(rn)
    z = rn == 0.0
    if np.any(~z):
        g1, g2, _ = O.poly_pair_functions(rn[~z], a, b, xi)
        f1[~z], f2[~z] = g1, g2
    if np.any(z):
        sv = O.poly_pair_functions(np.array([1.0]), a, b, xi)[2]
        f1[z] = f2[z] = sv
    return f1, f2


def poly_lookup_derivs(d, a, b, xi, r_table, step=1e-5):
    """perp, para and their derivatives in d, a and b at distances d (a <= b).

    The lookup is the reference's linear interpolation between table nodes;
    d-derivatives are the slopes of the interpolating segments, radius
    derivatives interpolate central differences of the node values.
    """
    d = np.asarray(d, dtype=np.float64)
    n = len(r_table)
    last = r_table[-1]
    k = np.where(d < 1.0, 0, 1 + ((d - 1.0) / O.TABLE_DR).astype(np.int64))
    clamp = (d >= last) | (k >= n - 1)
    k = np.clip(k, 0, n - 2)
    r0, r1 = r_table[k], r_table[k + 1]
    t = np.where(d < 1.0, d, (d - r0) / (r1 - r0))
    t = np.where(clamp, 1.0, t)
    r0 = np.where(clamp, last, r0)
    r1 = np.where(clamp, last, r1)

    def vals(aa, bb):
        y0 = _node_values(r0, aa, bb, xi)
        y1 = _node_values(r1, aa, bb, xi)
        return [y0[q] * (1.0 - t) + y1[q] * t for q in (0, 1)], [(y1[q] - y0[q]) for q in (0, 1)]

    (perp, para), (s1, s2) = vals(a, b)
    width = np.where(d < 1.0, 1.0, r1 - r0)
    dperp_dd = np.where(clamp, 0.0, s1 / np.where(width > 0, width, 1.0))
    dpara_dd = np.where(clamp, 0.0, s2 / np.where(width > 0, width, 1.0))
    ha, hb = step * a, step * b
    (pa_p, qa_p), _ = vals(a + ha, b) if a + ha <= b else vals(b, a + ha)
    (pa_m, qa_m), _ = vals(a - ha, b)
    (pb_p, qb_p), _ = vals(a, b + hb)
    (pb_m, qb_m), _ = vals(a, b - hb) if a <= b - hb else vals(b - hb, a)
    return dict(perp=perp, para=para, perp_d=dperp_dd, para_d=dpara_dd,
                perp_a=(pa_p - pa_m) / (2 * ha), para_a=(qa_p - qa_m) / (2 * ha),
                perp_b=(pb_p - pb_m) / (2 * hb), para_b=(qb_p - qb_m) / (2 * hb))


def self_value_deriv(a, xi, step=1e-5):
    """d/da of self(a, a) by central differences."""
    h = step * a
    f = lambda x: O.poly_pair_functions(np.array([1.0]), x, x, xi)[2]
    return (f(a + h) - f(a - h)) / (2 * h)


# ---------------------------------------------------------------------------
# Bilinear-form gradients: d/dx and d/da of lam^T G(x, a) p
# ---------------------------------------------------------------------------


def poly_bilinear_grad(op: O.PolyEwaldOperator, lam, p):
    """(dB/dx (N,3), dB/da (N,)) complex, B = lam^T G p for the polydisperse
    operator in SOLVER_AX mode (reciprocal + pairs + self value)."""
    prm = op.p
    N = len(op.pos)
    lam = np.asarray(lam, dtype=np.complex128).reshape(N, 3)
    p = np.asarray(p, dtype=np.complex128).reshape(N, 3)
    Nx, Ny, Nz = prm.num_grid
    V = Nx * Ny * Nz
    idx, w, dw_dx, dw_da = poly_weight_derivs(prm, op.pos, op.radii)

    def potential(q):
        rho = np.zeros(V, dtype=np.complex128)
        np.add.at(rho, idx.ravel(), np.einsum("noc,nc->no", w, q).ravel())
        F = np.fft.fftn(rho.reshape(Nx, Ny, Nz)) * op.scale
        return (np.fft.ifftn(F) * float(V)).ravel()

    phi_p, phi_l = potential(p), potential(lam)
    h3 = float(np.prod(prm.h))
    Pp, Pl = phi_p[idx], phi_l[idx]                       # (n, P^3)
    gx = h3 * (np.einsum("noce,nc,no->ne", dw_dx, lam, Pp) + np.einsum("noce,nc,no->ne", dw_dx, p, Pl))
    ga = h3 * (np.einsum("noc,nc,no->n", dw_da, lam, Pp) + np.einsum("noc,nc,no->n", dw_da, p, Pl))
    # self value sigma(a_j) lam_j . p_j
    u, ridx = prm.unique, prm.ridx
    for j in range(N):
        ga[j] += self_value_deriv(u[ridx[j]], prm.xi) * np.dot(lam[j], p[j])
    # pairs: f = lam_j^T T(r; a_i, a_j) p_i, r = x_i - x_j (source i, target j)
    if len(op.pi_):
        i, j = op.pi_, op.pj
        r = op.pr
        de = op.deff
        dl = r / de[:, None]
        ai, aj = u[ridx[i]], u[ridx[j]]
        perp = np.zeros(len(de)); para = np.zeros(len(de))
        pd_ = np.zeros(len(de)); qd_ = np.zeros(len(de))
        pai = np.zeros(len(de)); qai = np.zeros(len(de)); paj = np.zeros(len(de)); qaj = np.zeros(len(de))
        lo, hi = np.minimum(ai, aj), np.maximum(ai, aj)
        for A_ in np.unique(lo):
            for B_ in np.unique(hi[lo == A_]):
                m = (lo == A_) & (hi == B_)
                D = poly_lookup_derivs(de[m], A_, B_, prm.xi, prm.r_table)
                perp[m], para[m], pd_[m], qd_[m] = D["perp"], D["para"], D["perp_d"], D["para_d"]
                # radius of the source: the 'a' slot when it is the smaller one
                src_lo = ai[m] <= aj[m]
                pai[m] = np.where(src_lo, D["perp_a"], D["perp_b"])
                qai[m] = np.where(src_lo, D["para_a"], D["para_b"])
                tgt_lo = aj[m] < ai[m]
                paj[m] = np.where(tgt_lo, D["perp_a"], D["perp_b"])
                qaj[m] = np.where(tgt_lo, D["para_a"], D["para_b"])
                eq = ai[m] == aj[m]
                # equal radii: either slot (the functions are symmetric there)
                paj[m] = np.where(eq, D["perp_a"], paj[m])
                qaj[m] = np.where(eq, D["para_a"], qaj[m])
        L_, P_ = lam[j], p[i]
        lp = np.sum(L_ * P_, axis=1)
        ld = np.sum(L_ * dl, axis=1)
        pdl = np.sum(P_ * dl, axis=1)
        # gradient of f in r
        grad = (pd_ * lp)[:, None] * dl + ((qd_ - pd_) * ld * pdl)[:, None] * dl \
            + ((para - perp) / de)[:, None] * ((L_ - ld[:, None] * dl) * pdl[:, None]
                                               + ld[:, None] * (P_ - pdl[:, None] * dl))
        np.add.at(gx, i, grad)
        np.add.at(gx, j, -grad)
        fa_i = pai * (lp - ld * pdl) + qai * ld * pdl
        fa_j = paj * (lp - ld * pdl) + qaj * ld * pdl
        np.add.at(ga, i, fa_i)
        np.add.at(ga, j, fa_j)
    return gx, ga


def direct_bilinear_grad(pos, radius, lam, p):
    """(dB/dx, dB/da) for the open-boundary SOLVER_AX operator
    (direct_electric_field.cu:42-324): E_j = -(1/4 pi) sum_i [3 u (u.p_i) - p_i]
    / r^3 with r = |x_i - x_j| (>= a_i), plus the self value 1/(4 pi a_j^3)."""
    pos = np.asarray(pos, dtype=np.float64)
    radius = np.asarray(radius, dtype=np.float64)
    N = len(pos)
    lam = np.asarray(lam, dtype=np.complex128).reshape(N, 3)
    p = np.asarray(p, dtype=np.complex128).reshape(N, 3)
    gx = np.zeros((N, 3), dtype=np.complex128)
    ga = np.zeros(N, dtype=np.complex128)
    k = -1.0 / (4.0 * PI)
    for j in range(N):
        for i in range(N):
            if i == j:
                continue
            r = pos[i] - pos[j]
            d = math.sqrt(r @ r)
            if d < radius[i]:
                raise ValueError("direct gradient assumes non-overlapping spheres")
            u = r / d
            lp, lu, pu = lam[j] @ p[i], lam[j] @ u, p[i] @ u
            # f = k (3 lu pu - lp) / d^3
            df_dd = k * (-3.0) * (3 * lu * pu - lp) / d ** 4
            dlu = (lam[j] - lu * u) / d
            dpu = (p[i] - pu * u) / d
            grad = df_dd * u + k * 3.0 * (dlu * pu + lu * dpu) / d ** 3
            gx[i] += grad
            gx[j] -= grad
        ga[j] += -3.0 / (4.0 * PI * radius[j] ** 4) * (lam[j] @ p[j])
    return gx, ga


# ---------------------------------------------------------------------------
# Loss and gradient with dense solves (small systems)
# ---------------------------------------------------------------------------


def make_operator(kind, box, pos, radius, xi, tol, params=None):
    if kind == "direct":
        op = O.DirectOperator(radius, True)
    else:
        op = O.PolyEwaldOperator(box, tol, xi, radius, True)
        if params is not None:
            # hold the forward point's discretisation (grid, support, eta,
            # cutoff, table nodes); radius classes follow the radii
            for name in ("num_grid", "h", "P", "eta", "offsets", "rc", "r_table"):
                setattr(op.p, name, getattr(params, name))
            op.scale = O.poly_scale(op.p)
    op.set_positions(pos)
    return op


def dense(op, N, sc):
    n = 3 * N
    A = np.zeros((n, n), dtype=np.complex128)
    e = np.zeros(n, dtype=np.complex128)
    for q in range(n):
        e[:] = 0.0
        e[q] = 1.0
        A[:, q] = op.apply(e, sc)
    return A


def loss_and_grad(kind, box, pos, radius, eps_rel, deps, c, E0, xi=0.5, tol=1e-6, params=None, grad=True):
    """L and (dL/dx, dL/da, dL/dtheta) for the loss of the module docstring.

    eps_rel (W, N): eps_i / eps_m per frequency; deps (T, W, N): d eps_rel /
    d theta_t; c (W, K, 3N): loss weights; E0 (K, 3) incident fields.
    """
    pos = np.asarray(pos, dtype=np.float64)
    radius = np.asarray(radius, dtype=np.float64)
    N = len(pos)
    W, K = c.shape[0], c.shape[1]
    op = make_operator(kind, box, pos, radius, xi, tol, params)
    L = 0.0
    gx = np.zeros((N, 3))
    ga = np.zeros(N)
    gt = np.zeros(deps.shape[0])
    for w in range(W):
        e = eps_rel[w]
        s = 3.0 / (4.0 * PI * (e - 1.0) * radius ** 3)
        A = dense(op, N, s)
        B = np.stack([np.tile(np.asarray(E0[k], dtype=np.complex128), N) for k in range(K)], axis=1)
        P = np.linalg.solve(A, B)
        L += float(np.sum(np.imag(np.sum(np.conj(c[w].T) * P, axis=0))))
        if not grad:
            continue
        Lam = np.linalg.solve(A, np.conj(c[w].T))          # A^T = A
        ds_de = -3.0 / (4.0 * PI * radius ** 3 * (e - 1.0) ** 2)
        ds_da = -3.0 * s / radius
        for k in range(K):
            lam = Lam[:, k].reshape(N, 3)
            p = P[:, k].reshape(N, 3)
            lp = np.sum(lam * p, axis=1)
            if kind == "direct":
                bx, ba = direct_bilinear_grad(pos, radius, lam, p)
            else:
                bx, ba = poly_bilinear_grad(op, lam, p)
            gx -= np.imag(bx)
            ga -= np.imag(ba + ds_da * lp)
            for t in range(deps.shape[0]):
                gt[t] -= float(np.imag(np.sum(ds_de * deps[t, w] * lp)))
    return L, gx, ga, gt
