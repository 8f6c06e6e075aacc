"""CPU oracle of the reference's EELS solve (electron energy loss of a
particle assembly under a moving electron beam), dipoles only.

TEST INFRASTRUCTURE ONLY, like ``mpm_oracle``: a float64 numpy restatement
of ``src/cpp/eels_solver.cu`` (``EELS_Solver::compute``, :386-881) used as a
checker; the product never imports it.  What it restates:

* non-dimensionalisation by the smallest radius and by eps_m (:241-263);
  the beam's Lorentz factor is taken after it, with eps_m = 1 (:482);
* the beam field at each particle (:519-578): soft-core distance
  sqrt(r_perp^2 + sigma^2) with sigma = 0.5 nm, K1 in-plane and K0 along the
  beam, phase exp(2 pi i omega z / v); with the Brillouin-zone sum (ASM),
  periodic images within 12 decay lengths and a Bloch phase per image
  (:491-509, 569-572);
* the reference's own K0/K1 of complex argument (:56-93): the real-argument
  function when the imaginary part vanishes or when both parts are nonzero,
  the Hankel form on the imaginary axis;
* self coefficients -3 / (4 pi (1 - eps)) without the radius factor
  (:638-642);
* the loss probability by reciprocity, sum_p Im(p . conj(E_inc)) / (2 pi^2)
  (:796-838), and the Brillouin-zone average (:847-859).

The solve itself is the oracle's operator (direct, monodisperse or
polydisperse Ewald, with the Bloch wavevector for ASM) and its GMRES to a
tight tolerance, so the result is the converged solution the reference's
Krylov solve approaches; the reference's initial-guess heuristics change
only how it gets there.  Not restated: particle splitting near the beam
(``eels.py``), quadrupoles (surface-averaged beam gradients, :580-634).
Pinned by the reference's golden vector ``tests/data/ref_eels_vs_python_module.npz``.
"""
import math

import numpy as np
from scipy import special

from . import mpm_oracle as O

PI = math.pi


def eval_k(n, z):
    """K_n(z), n in {0, 1}, as the reference evaluates it (:56-93)."""
    z = complex(z)
    if abs(z.imag) < 1e-12:
        return complex(special.kv(n, z.real))
    if abs(z.real) < 1e-12:
        y = z.imag
        yy = -y if y < 0.0 else y
        j, yn = special.jv(n, yy), special.yv(n, yy)
        v = complex(-PI / 2.0 * yn, -PI / 2.0 * j) if n == 0 else complex(-PI / 2.0 * j, PI / 2.0 * yn)
        return v.conjugate() if y < 0.0 else v
    return complex(special.kv(n, z.real))


def beam_field(pos, epos, omega, v, gamma, length_scale, box=None, k=(0.0, 0.0), asm=False):
    """E_inc (N, 3) of the beam at scaled positions for one scaled omega."""
    pos = np.asarray(pos, dtype=np.float64)
    N = len(pos)
    E = np.zeros((N, 3), dtype=np.complex128)
    rx_max = ry_max = 0
    if asm:
        r_decay = 12.0 * abs((v * gamma) / (2.0 * PI * omega))
        rx_max = int(math.ceil(r_decay / box[0]))
        ry_max = int(math.ceil(r_decay / box[1]))
    sigma = 0.5 / length_scale
    for ix in range(-rx_max, rx_max + 1):
        for iy in range(-ry_max, ry_max + 1):
            Rx = ix * box[0] if asm else 0.0
            Ry = iy * box[1] if asm else 0.0
            for p in range(N):
                dx = pos[p, 0] - epos[0] - Rx
                dy = pos[p, 1] - epos[1] - Ry
                r_safe = math.sqrt(dx * dx + dy * dy + sigma * sigma)
                xv = (2.0 * PI * omega * r_safe) / (v * gamma)
                pref = omega / (v * v * gamma) * np.exp(1j * 2.0 * PI * omega * pos[p, 2] / v)
                k0, k1 = eval_k(0, xv), eval_k(1, xv)
                e = np.array([-pref * k1 * dx / r_safe, -pref * k1 * dy / r_safe, pref * 1j / gamma * k0])
                if asm:
                    e = e * np.exp(1j * (k[0] * (pos[p, 0] - Rx) + k[1] * (pos[p, 1] - Ry)))
                E[p] += e
    return E


class EELSOracle:
    """``EELS_Solver`` for dipoles: ``compute(epos, positions)`` per beam
    position; ``eels`` (beams, W), ``dipoles`` (beams, W, N, 3) in scaled
    units (the reference's ``physical=False``)."""

    def __init__(self, box, eps_p, omega, v, eps_m=1.0, radius=1.0, xi=0.5, tol=1e-3, field_type="auto",
                 asm=False, asm_n=(1, 1), solve_tol=1e-11):
        self.box = np.asarray(box, dtype=np.float64)
        self.omega = np.asarray(omega, dtype=np.float64)
        self.eps_p = np.asarray(eps_p, dtype=np.complex128)
        self.v, self.eps_m, self.radius = float(v), float(eps_m), radius
        self.xi, self.tol, self.field_type = float(xi), float(tol), field_type
        self.asm, self.asm_n, self.solve_tol = bool(asm), asm_n, solve_tol
        self.eels, self.dipoles = [], []

    def _eps(self, N):
        W = len(self.omega)
        e = self.eps_p
        if e.ndim == 0 or e.size == 1:
            return np.full((W, N), complex(e.ravel()[0]))
        if e.ndim == 1:
            return np.repeat(e[:, None], N, axis=1) if e.size == W else np.tile(e, (W, 1))
        return np.broadcast_to(e, (W, N)).copy()

    def _field(self, box_s, radius_s, k):
        mono = all(r == radius_s[0] for r in radius_s)
        if self.field_type == "direct":
            return O.DirectOperator(radius_s, True)
        if self.field_type == "polydisperse" or (self.field_type == "auto" and not mono):
            return O.PolyEwaldOperator(box_s, self.tol, self.xi, radius_s, True, bloch=k)
        return O.MonoEwaldOperator(box_s, self.tol, self.xi, True, bloch=k)

    def compute(self, epos, positions):
        pos = np.asarray(positions, dtype=np.float64)
        N = len(pos)
        radius = list(np.atleast_1d(np.asarray(self.radius, dtype=np.float64)))
        if len(radius) == 1:
            radius = radius * N
        ls = min(radius)
        box_s = self.box / ls
        radius_s = [r / ls for r in radius]
        omega_s = self.omega * ls
        eps = self._eps(N) / self.eps_m
        gamma = 1.0 / np.sqrt(complex(1.0 - 1.0 * self.v * self.v))
        gamma = gamma.real if abs(gamma.imag) < 1e-300 else gamma
        pos_s = pos / ls
        e_s = np.asarray(epos, dtype=np.float64) / ls
        W = len(omega_s)
        nx, ny = self.asm_n if self.asm else (1, 1)
        dkx = 2.0 * PI / (box_s[0] * nx) if self.asm else 0.0
        dky = 2.0 * PI / (box_s[1] * ny) if self.asm else 0.0
        eels = np.zeros(W)
        dips = np.zeros((W, N, 3), dtype=np.complex128)
        for ix in range(nx):
            for iy in range(ny):
                k = (-PI / box_s[0] + (ix + 0.5) * dkx, -PI / box_s[1] + (iy + 0.5) * dky) if self.asm else (0.0, 0.0)
                F = self._field(box_s, radius_s, k)
                F.set_positions(pos_s)
                for w in range(W):
                    E = beam_field(pos_s, e_s, omega_s[w], self.v, gamma, ls, box_s, k, self.asm)
                    sc = -3.0 / (4.0 * PI * (1.0 - eps[w]))
                    b = E.ravel()
                    M = O.jacobi_inverse(sc, N)
                    sol, _ = O.gmres(lambda x: F.apply(x, sc), b, np.zeros_like(b), self.solve_tol, M)
                    p = sol.reshape(N, 3)
                    eels[w] += np.sum(np.imag(np.sum(p * np.conj(E), axis=1))) / (2.0 * PI * PI)
                    dips[w] += p
        if self.asm:
            frac = (dkx * dky) / ((2.0 * PI / box_s[0]) * (2.0 * PI / box_s[1]))
            eels *= frac
            dips *= frac
        self.eels.append(eels)
        self.dipoles.append(dips)
        return eels, dips
