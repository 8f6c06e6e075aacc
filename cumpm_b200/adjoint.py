"""Differentiable extinction spectrum of the self-consistent dipole solve.

``extinction_loss`` returns the extinction cross-section summed over
frequencies and incident fields,

    L = sum_{w,k} C_ext(w, k),   C_ext = 4 pi k_w sum_i Im(E0_k^* . p_i)

(the formula of the reference's examples/mpm_hex_monolayer_sweep.py:117-119)
as a torch scalar whose gradient with respect to particle positions, radii
and the Drude plasma frequency / damping of each species comes from a
hand-written adjoint rather than from autograd through the solver:

* forward: one batched fp64 solve of A(w) p = E0_k for all W x K columns
  (A = G(x, a) + diag(s), s_i = 3 / (4 pi (eps_i/eps_m - 1) a_i^3)); only
  the converged dipoles are kept;
* backward: one batched adjoint solve with the same operator (A is
  complex-symmetric, A^T = A), A lam = conj(c), then the derivative of the
  operator contracted with lam and p on the GPU (``Field.grad``), plus the
  self-coefficient terms:  dL/dtheta = -Im(sum lam^T dA/dtheta p).

The periodic field is the polydisperse spectral-Ewald operator (equal radii
included: it reproduces the monodisperse field to the Ewald tolerance);
``field_type="direct"`` uses the open-boundary sum.  Lengths are made
dimensionless with ``length_scale`` (default: the smallest radius, held
fixed), and the Ewald discretisation of the forward point is the one
differentiated.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import capi

__all__ = ["extinction_loss", "wavenumber_from_ev"]

HC_EV_NM = 1239.8419843320026  # h c in eV nm


def wavenumber_from_ev(omega_ev, eps_m):
    """k = 2 pi sqrt(eps_m) / lambda in 1/nm for photon energies in eV."""
    return 2.0 * math.pi * math.sqrt(eps_m) * np.asarray(omega_ev, dtype=np.float64) / HC_EV_NM


def _permittivity(omega, species, omega_p, gamma, eps_inf, eps_const):
    """eps (W, N) complex and d eps / d omega_p, d eps / d gamma (W, N)."""
    W, N = len(omega), len(species)
    w = omega[:, None]
    eps = np.empty((W, N), dtype=np.complex128)
    d_wp = np.zeros((W, N), dtype=np.complex128)
    d_g = np.zeros((W, N), dtype=np.complex128)
    drude = species >= 0
    s = np.where(drude, species, 0)
    wp, g, ei = omega_p[s][None, :], gamma[s][None, :], eps_inf[s][None, :]
    den = w * w + 1j * w * g
    e_d = ei - wp * wp / den
    eps[:] = np.where(drude[None, :], e_d, eps_const[None, :])
    d_wp[:] = np.where(drude[None, :], -2.0 * wp / den, 0.0)
    d_g[:] = np.where(drude[None, :], wp * wp * 1j * w / den ** 2, 0.0)
    return eps, d_wp, d_g


class _Extinction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, radii, omega_p, gamma, cfg):
        dev = torch.device("cuda")
        pos = positions.detach().cpu().numpy().astype(np.float64)
        rad = radii.detach().cpu().numpy().astype(np.float64)
        wp = omega_p.detach().cpu().numpy().astype(np.float64)
        gm = gamma.detach().cpu().numpy().astype(np.float64)
        N = len(pos)
        L0 = float(cfg["length_scale"] or rad.min())
        omega = cfg["omega"]
        W = len(omega)
        E0 = cfg["E0"]
        K = len(E0)
        M = W * K
        species = cfg["species"]
        eps, d_wp, d_g = _permittivity(omega, species, wp, gm, cfg["eps_inf"], cfg["eps_const"])
        e = eps / cfg["eps_m"]
        a = rad / L0
        kind = capi.FIELD_DIRECT if cfg["field_type"] == "direct" else capi.FIELD_POLY
        box = np.asarray(cfg["box"], dtype=np.float64) / L0
        F = capi.Field(kind, box, cfg["tol"], cfg["xi"], radius=a)
        F.set_positions(pos / L0)
        s = 3.0 / (4.0 * math.pi * (e - 1.0) * a[None, :] ** 3)              # (W, N)
        col_w = np.repeat(np.arange(W), K)
        col_k = np.tile(np.arange(K), W)
        SC = np.ascontiguousarray(s[col_w].T)                              # (N, M)
        B = np.zeros((3 * N, M), dtype=np.complex128)
        for m in range(M):
            for c in range(3):
                B[c::3, m] = E0[col_k[m]][c]
        kw = cfg["wavenumber"]
        cw = 4.0 * math.pi * kw[col_w] * cfg["eps_m"] * L0 ** 3           # (M,) loss weight per column
        Bt = torch.tensor(B, device=dev)
        St = torch.tensor(SC, device=dev)
        X = torch.zeros_like(Bt)
        rep = F.batch_solve(Bt, X, St, tol=cfg["solve_tol"], recip_fp32=False, refine=False,
                            maxiter=cfg["maxiter"])
        if rep["num_converged"] < M:
            raise RuntimeError(f"forward solve: {M - rep['num_converged']} of {M} columns did not converge")
        # L = sum_m cw_m Im(E0^H p)  (E0 real or complex, broadcast over particles)
        E0c = torch.tensor(np.conj(B), device=dev)
        loss = float(torch.sum(torch.imag(torch.sum(E0c * X, dim=0)) * torch.tensor(cw, device=dev)).item())
        ctx.F, ctx.X, ctx.St, ctx.E0c, ctx.cw = F, X, St, E0c, cw
        ctx.meta = dict(N=N, L0=L0, a=a, e=e, s=s, col_w=col_w, d_wp=d_wp, d_g=d_g, species=species,
                        eps_m=cfg["eps_m"], n_species=len(wp), cfg=cfg)
        ctx.dtypes = (positions.dtype, radii.dtype, omega_p.dtype, gamma.dtype)
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        F, X, St, E0c, cw, md = ctx.F, ctx.X, ctx.St, ctx.E0c, ctx.cw, ctx.meta
        dev = X.device
        N, L0 = md["N"], md["L0"]
        cfg = md["cfg"]
        # adjoint right-hand side conj(c_m) = cw_m conj(E0) on the dipole rows
        C = E0c * torch.tensor(cw, device=dev)[None, :]
        Lam = torch.zeros_like(X)
        rep = F.batch_solve(C, Lam, St, tol=cfg["solve_tol"], recip_fp32=False, refine=False, maxiter=cfg["maxiter"])
        if rep["num_converged"] < X.shape[1]:
            raise RuntimeError("adjoint solve did not converge")
        gx_c, ga_c = F.grad(Lam, X)
        # lam_i . p_i per particle and column
        lp = torch.sum((Lam * X).reshape(N, 3, -1), dim=1).cpu().numpy()    # (N, M)
        gx = -np.imag(gx_c.cpu().numpy())
        a, s, e = md["a"], md["s"], md["e"]
        col_w = md["col_w"]
        s_col = s[col_w].T                                                   # (N, M)
        ds_da = -3.0 * s_col / a[:, None]
        ga = -np.imag(ga_c.cpu().numpy() + np.sum(ds_da * lp, axis=1))
        ds_de = (-3.0 / (4.0 * math.pi * a[None, :] ** 3 * (e - 1.0) ** 2))[col_w].T   # (N, M)
        S = md["n_species"]
        gwp, gg = np.zeros(S), np.zeros(S)
        sp = md["species"]
        for t, d in ((0, md["d_wp"]), (1, md["d_g"])):
            de = (d / md["eps_m"])[col_w].T                                  # (N, M)
            contrib = -np.imag(np.sum(ds_de * de * lp, axis=1))               # per particle
            out = gwp if t == 0 else gg
            for k in range(S):
                out[k] = float(np.sum(contrib[sp == k]))
        g = float(grad_out)
        dt = ctx.dtypes
        return (torch.tensor(gx / L0 * g, dtype=dt[0]), torch.tensor(ga / L0 * g, dtype=dt[1]),
                torch.tensor(gwp * g, dtype=dt[2]), torch.tensor(gg * g, dtype=dt[3]), None)


def extinction_loss(positions, radii, omega_p, gamma, *, box, omega, species, eps_inf, eps_m=1.0,
                    eps_const=None, E0=((1.0, 0.0, 0.0),), wavenumber=None, xi=0.5, tol=1e-6,
                    field_type="ewald", solve_tol=1e-11, maxiter=2000, length_scale=None):
    """Summed extinction cross-section with adjoint gradients.

    positions (N, 3), radii (N,): torch float64 tensors (any length unit);
    omega_p, gamma (S,): Drude parameters of the S species (torch tensors, in
    the units of ``omega``); species (N,) int: a particle's Drude species, or
    -1 for a constant permittivity ``eps_const[i]``; eps_inf (S,);
    wavenumber (W,): k_w in inverse length units (default 1);
    field_type: "ewald" (periodic ``box``) or "direct" (open boundaries).
    """
    species = np.asarray(species, dtype=np.int64)
    N = len(species)
    omega = np.asarray(omega, dtype=np.float64)
    cfg = dict(box=np.asarray(box, dtype=np.float64), omega=omega, species=species,
               eps_inf=np.asarray(eps_inf, dtype=np.float64), eps_m=float(eps_m),
               eps_const=np.zeros(N, complex) if eps_const is None else np.asarray(eps_const, dtype=np.complex128),
               E0=[np.asarray(e, dtype=np.complex128) for e in E0],
               wavenumber=np.ones(len(omega)) if wavenumber is None else np.asarray(wavenumber, dtype=np.float64),
               xi=float(xi), tol=float(tol), field_type=field_type, solve_tol=float(solve_tol), maxiter=int(maxiter),
               length_scale=length_scale)
    if field_type not in ("ewald", "direct"):
        raise ValueError("field_type must be 'ewald' or 'direct'")
    return _Extinction.apply(positions, radii, omega_p, gamma, cfg)
