"""Electron energy loss (EELS) of a particle assembly under a moving
electron beam, on the device batched solve.

Drop-in for the reference's ``cuMPM.EELS`` (``src/cuMPM/eels.py``,
``src/cpp/eels_solver.cu``) for dipoles.  Per beam position, every
frequency is one right-hand side of one batched Krylov solve on the GPU:

* host: non-dimensionalisation by the smallest radius and by eps_m
  (eels_solver.cu:241-263), the beam field at each particle (:519-578):
  soft-core distance sqrt(r_perp^2 + sigma^2) with sigma = 0.5 nm, K1 across
  and K0 along the beam, phase exp(2 pi i omega z / v), Lorentz factor
  1/sqrt(1 - v^2) (taken after eps_m is scaled to 1, :482); self
  coefficients -3 / (4 pi (1 - eps)) without the radius factor (:638-642);
* device: ``capi.Field.batch_solve`` of A(omega_w) p_w = E_inc(omega_w)
  for all w at once (the field and its precalcs built once per frame);
* host: the loss by reciprocity, sum_p Im(p . conj(E_inc)) / (2 pi^2)
  (:796-838).

Particles closer to the beam than ``split_dist`` (with ``N_split`` > 1) are
split into sub-dipoles on a cubic, Fibonacci or fcc lattice in the unit
sphere that keep the particle's volume (``eels.py:177-320``); each beam
position then solves its own split system.

With ``asm_flag`` (an infinite array: the Brillouin-zone sum,
eels_solver.cu:495-881) the solve runs once per point of an asm_Nx x
asm_Ny midpoint grid over the zone: the device field takes the point's
Bloch wavevector (``capi.Field.set_bloch``; a direct field has none, as in
the reference), the beam field sums the periodic images within 12 decay
lengths with the Bloch phase, and loss and dipoles are averaged over the
points (the sum times dk_x dk_y over the zone area).

Not available yet (it raises ``RuntimeError`` naming the gap): quadrupoles.
"""
import math

import numpy as np

from . import capi

_PI = math.pi


def _bessel_k(n, z):
    """K_n(z), n in {0, 1}, by the reference's rules (eels_solver.cu:56-93):
    the real-argument function unless z lies on the imaginary axis, where
    the Hankel form applies."""
    from scipy import special

    z = np.asarray(z, dtype=np.complex128)
    out = special.kv(n, z.real).astype(np.complex128)
    axis = (np.abs(z.imag) >= 1e-12) & (np.abs(z.real) < 1e-12)
    if np.any(axis):
        y = np.abs(z.imag[axis])
        j, yn = special.jv(n, y), special.yv(n, y)
        v = (-_PI / 2 * yn - 1j * _PI / 2 * j) if n == 0 else (-_PI / 2 * j + 1j * _PI / 2 * yn)
        out[axis] = np.where(z.imag[axis] < 0.0, np.conj(v), v)
    return out


def beam_field(pos, epos, omega, v, gamma, length_scale, box=None, k=(0.0, 0.0), asm=False):
    """Beam field (N, 3) at scaled positions, for one scaled frequency.
    With ``asm``: the sum over the beam's periodic images (R_x, R_y) within
    12 decay lengths |v gamma / (2 pi omega)|, each times the Bloch phase
    exp(i (k_x (x - R_x) + k_y (y - R_y))) (eels_solver.cu:519-578)."""
    pos = np.asarray(pos, dtype=np.float64)
    sigma = 0.5 / length_scale
    pref = omega / (v * v * gamma) * np.exp(1j * 2.0 * _PI * omega * pos[:, 2] / v)
    nx = ny = 0
    if asm:
        r_decay = 12.0 * abs((v * gamma) / (2.0 * _PI * omega))
        nx = int(math.ceil(r_decay / box[0]))
        ny = int(math.ceil(r_decay / box[1]))
    E = np.zeros((len(pos), 3), dtype=np.complex128)
    for ix in range(-nx, nx + 1):
        for iy in range(-ny, ny + 1):
            Rx = ix * box[0] if asm else 0.0
            Ry = iy * box[1] if asm else 0.0
            dx = pos[:, 0] - epos[0] - Rx
            dy = pos[:, 1] - epos[1] - Ry
            r = np.sqrt(dx * dx + dy * dy + sigma * sigma)
            x = (2.0 * _PI * omega * r) / (v * gamma)
            k0, k1 = _bessel_k(0, x), _bessel_k(1, x)
            e = np.stack([-pref * k1 * dx / r, -pref * k1 * dy / r, pref * 1j / gamma * k0], axis=1)
            if asm:
                e = e * np.exp(1j * (k[0] * (pos[:, 0] - Rx) + k[1] * (pos[:, 1] - Ry)))[:, None]
            E += e
    return E


def unit_offsets(method, n_split):
    """Sub-dipole offsets inside the unit sphere (eels.py:177-258).

    * cubic: the n^3 cell centres of [-1, 1]^3, n the smallest integer with
      n^3 >= n_split, those within distance 1 kept;
    * fibonacci: n_split golden-angle directions on the sphere times
      cube-root shell radii ((i + 1/2)/n)^(1/3), the radii shuffled by the
      generator of seed 0;
    * fcc: points of even index sum on a cubic lattice of step h within
      distance 1, h = (2 pi / 3n)^(1/3) shrunk by 2 % until at least n_split
      points fit.
    """
    if method == "cubic":
        n = int(np.ceil(n_split ** (1.0 / 3.0)))
        while n ** 3 < n_split:
            n += 1
        h = 2.0 / n
        c = np.linspace(-1.0 + h / 2.0, 1.0 - h / 2.0, n)
        g = np.stack([a.ravel() for a in np.meshgrid(c, c, c, indexing="ij")], axis=1)
        return g[np.linalg.norm(g, axis=1) <= 1.0]
    if method == "fibonacci":
        n = int(n_split)
        i = np.arange(n, dtype=np.float64)
        y = 1.0 - (i / float(n - 1)) * 2.0
        t = np.pi * (3.0 - np.sqrt(5.0)) * i
        s = np.sqrt(np.maximum(0.0, 1.0 - y * y))
        dirs = np.stack([np.cos(t) * s, y, np.sin(t) * s], axis=1)
        shells = ((i + 0.5) / n) ** (1.0 / 3.0)
        np.random.default_rng(0).shuffle(shells)
        return shells[:, None] * dirs
    if method == "fcc":
        n = max(1, int(n_split))

        def lattice(step):
            m = int(np.ceil(1.0 / step))
            k = np.arange(-m, m + 1)
            gx, gy, gz = np.meshgrid(k, k, k, indexing="ij")
            even = (gx + gy + gz) % 2 == 0
            g = np.stack([gx[even], gy[even], gz[even]], axis=1) * step
            return g[np.linalg.norm(g, axis=1) <= 1.0]

        h = ((2.0 * np.pi) / (3.0 * n)) ** (1.0 / 3.0)
        pts = lattice(h)
        while len(pts) < n and h > 1e-4:
            h *= 0.98
            pts = lattice(h)
        return pts
    raise ValueError(f"Unknown split_method: {method}")


def split_near_beam(positions, e_pos, radii, eps, split_dist, offsets):
    """Particles within split_dist of the beam (in the plane across it)
    replaced by sub-dipoles at position + R * offset of radius
    R / M^(1/3), M = len(offsets), each with its particle's permittivity;
    the others first, in order (eels.py:261-320).  eps is (W, N)."""
    positions = np.asarray(positions, dtype=np.float64)
    d = np.linalg.norm(positions[:, :2] - np.asarray(e_pos, dtype=np.float64)[None, :], axis=1)
    close = d < split_dist
    if not np.any(close):
        return positions.copy(), np.asarray(radii, dtype=np.float64).copy(), np.asarray(eps).copy()
    keep = np.nonzero(~close)[0]
    M = len(offsets)
    frac = 1.0 / (M ** (1.0 / 3.0))
    pos_out = [positions[keep]]
    rad_out = [np.asarray(radii, dtype=np.float64)[keep]]
    eps_out = [np.asarray(eps)[:, keep]]
    for i in np.nonzero(close)[0]:
        R = float(radii[i])
        pos_out.append(positions[i] + offsets * R)
        rad_out.append(np.full(M, R * frac))
        eps_out.append(np.repeat(np.asarray(eps)[:, i:i + 1], M, axis=1))
    return np.concatenate(pos_out), np.concatenate(rad_out), np.concatenate(eps_out, axis=1)


class EELS:
    """EELS probability spectrum and induced dipoles (see the module
    docstring); same constructor, ``compute``, ``get_eels``,
    ``get_dipoles`` and ``get_positions`` as the reference's class."""

    def __init__(self, box, eps_p, omega, v, eps_m=1.0, radius=1.0, xi=0.5, tol=1e-3, quiet=False,
                 guess_type="derivative", solver_type="gmres", field_type="auto", split_dist=None, N_split=None,
                 integration_step=0.05, split_method="cubic", solve_quadrupoles=False, quad_idxs=None,
                 asm_flag=False, asm_Nx=1, asm_Ny=1, precision=None):
        if split_method not in ("cubic", "fibonacci", "fcc"):
            raise ValueError("split_method must be 'cubic', 'fibonacci', or 'fcc', got " + repr(split_method))
        if (split_dist is None) != (N_split is None):
            raise ValueError("Both split_dist and N_split must be specified, or both left as None.")
        if field_type not in ("auto", "monodisperse", "polydisperse", "direct"):
            raise ValueError(f"field_type must be 'auto', 'monodisperse', 'polydisperse', or 'direct', got {field_type}")
        if len(np.atleast_1d(box)) != 3:
            raise ValueError("box must have length 3")
        if solver_type not in ("gmres", "bicgstab"):
            raise ValueError(f"Unknown solver_type: {solver_type}")
        self.split_dist = 0.0 if split_dist is None else float(split_dist)
        self.N_split = 0 if N_split is None else int(N_split)
        self.split_method = split_method
        if solve_quadrupoles or (quad_idxs is not None and len(quad_idxs)):
            raise RuntimeError("EELS quadrupoles are not available in this build")
        self.asm = bool(asm_flag)
        self.asm_n = (int(asm_Nx), int(asm_Ny)) if self.asm else (1, 1)
        if self.asm and min(self.asm_n) < 1:
            raise ValueError("asm_Nx and asm_Ny must be at least 1")
        from .solver import _parse_precision

        prec = _parse_precision(precision)
        self._fp64 = str(prec).upper().endswith("DOUBLE")
        self.box = np.asarray(box, dtype=np.float64)
        self.omega = np.atleast_1d(np.asarray(omega, dtype=np.float64))
        self.eps_p = eps_p
        self.v, self.eps_m, self.radius = float(v), float(eps_m), radius
        self.xi, self.tol, self.quiet = float(xi), float(tol), bool(quiet)
        self.solver_type, self.field_type = solver_type, field_type
        self.use_jacobi_precond = True
        self._N = 0
        self._F = None
        self._eels, self._dips = [], []
        self._split_pos, self._dip_scale = [], []
        self._precision = precision
        self.positions = None

    # -- set-up (eels_solver.cu:202-263) -----------------------------------
    def _eps_matrix(self, N):
        W = len(self.omega)
        e = np.asarray(self.eps_p, dtype=np.complex128)
        if e.ndim == 0 or e.size == 1:
            return np.full((W, N), complex(e.ravel()[0]))
        if e.ndim == 1:
            if e.size != W:
                raise ValueError("1D eps_p must have length equal to num_wavevectors")
            return np.repeat(e[:, None], N, axis=1)
        if e.shape[0] != W:
            raise ValueError("First dimension of 2D eps_p must be equal to num_wavevectors")
        if e.shape[1] == 1:
            return np.repeat(e, N, axis=1)
        if e.shape[1] != N:
            raise RuntimeError("The number of particles is inconsistent with eps_p provided.")
        return e.copy()

    def _setup(self, N):
        rad = np.atleast_1d(np.asarray(self.radius, dtype=np.float64))
        if rad.size == 1:
            rad = np.full(N, float(rad[0]))
        elif rad.size != N:
            raise RuntimeError("The number of particles is inconsistent with the number of radii provided.")
        mono = bool(np.all(rad == rad[0]))
        if self.field_type == "monodisperse" and not mono:
            raise RuntimeError("field_type was set to 'monodisperse' but radii are not identical.")
        self._ls = float(rad.min())
        self._eps = self._eps_matrix(N) / self.eps_m
        self._rad_s = rad / self._ls
        box_s = self.box / self._ls
        if self.field_type == "direct":
            self._F = capi.Field(capi.FIELD_DIRECT, radius=self._rad_s)
        elif self.field_type == "polydisperse" or (self.field_type == "auto" and not mono):
            self._F = capi.Field(capi.FIELD_POLY, box_s, self.tol, self.xi, radius=self._rad_s)
        else:
            self._F = capi.Field(capi.FIELD_MONO, box_s, self.tol, self.xi)
        self._N = N

    # -- one beam position (eels_solver.cu:386-881) ------------------------
    def _frame(self, epos, pos_s):
        import torch

        N, W = self._N, len(self.omega)
        om = self.omega * self._ls
        gamma = 1.0 / math.sqrt(1.0 - self.v * self.v)
        e_s = np.asarray(epos, dtype=np.float64) / self._ls
        box_s = self.box / self._ls
        S = (-3.0 / (4.0 * _PI * (1.0 - self._eps))).T.copy()          # (N, W)
        dev = torch.device("cuda")
        St = torch.tensor(S, device=dev)
        method = capi.METHOD_BICGSTAB if self.solver_type == "bicgstab" else capi.METHOD_GMRES
        nx, ny = self.asm_n
        dkx = 2.0 * _PI / (box_s[0] * nx) if self.asm else 0.0
        dky = 2.0 * _PI / (box_s[1] * ny) if self.asm else 0.0
        eels = np.zeros(W)
        dips = np.zeros((W, N, 3), dtype=np.complex128)
        for ix in range(nx):
            for iy in range(ny):
                k = ((-_PI / box_s[0] + (ix + 0.5) * dkx, -_PI / box_s[1] + (iy + 0.5) * dky) if self.asm
                     else (0.0, 0.0))
                if self.asm and self._F.kind != capi.FIELD_DIRECT:
                    self._F.set_bloch(*k)
                B = np.empty((3 * N, W), dtype=np.complex128)
                for w in range(W):
                    B[:, w] = beam_field(pos_s, e_s, om[w], self.v, gamma, self._ls, box_s, k, self.asm).ravel()
                Bt = torch.tensor(B, device=dev)
                X = torch.zeros_like(Bt)
                self._F.batch_solve(Bt, X, St, tol=self.tol, method=method, jacobi=self.use_jacobi_precond,
                                    recip_fp32=not self._fp64, refine=not self._fp64)
                p = X.cpu().numpy()
                eels += np.imag(np.sum(p * np.conj(B), axis=0)) / (2.0 * _PI * _PI)
                dips += p.T.reshape(W, N, 3)
        if self.asm:
            # the average over the zone points (eels_solver.cu:847-862)
            frac = (dkx * dky) / ((2.0 * _PI / box_s[0]) * (2.0 * _PI / box_s[1]))
            eels *= frac
            dips *= frac
        return eels, dips

    def compute(self, epos, positions):
        positions = np.asarray(positions, dtype=np.float64)
        if positions.ndim != 2 or positions.shape[1] != 3:
            raise ValueError("positions must be of shape (num_particles, 3)")
        epos = np.asarray(epos, dtype=np.float64)
        if epos.ndim == 1:
            if epos.shape[0] != 2:
                raise ValueError("epos must be of shape (2,) or (num_epos, 2)")
            epos = epos[np.newaxis, :]
        elif epos.ndim != 2 or epos.shape[1] != 2:
            raise ValueError("epos must be of shape (2,) or (num_epos, 2)")
        N = len(positions)
        if N == 0:
            return
        if self._splitting():
            self._compute_split(epos, positions)
            return
        if self._N == 0:
            self._setup(N)
        elif N != self._N:
            raise RuntimeError("The number of particles has changed!")
        self.positions = positions
        pos_s = positions / self._ls
        self._F.set_positions(pos_s)
        for e in epos:
            if not self.quiet:
                print("  [EELS] impact parameter", e)
            eels, dips = self._frame(e, pos_s)
            self._eels.append(eels)
            self._dips.append(dips)

    # -- splitting near the beam (eels.py:381-478) --------------------------
    def _splitting(self):
        return self.split_dist > 0.0 and self.N_split > 1

    def _compute_split(self, epos, positions):
        N, W = len(positions), len(self.omega)
        rad = np.atleast_1d(np.asarray(self.radius, dtype=np.float64))
        if rad.size == 1:
            rad = np.full(N, float(rad[0]))
        elif rad.size != N:
            raise ValueError("The number of particles is inconsistent with the number of radii provided.")
        eps = self._eps_matrix(N)
        offsets = unit_offsets(self.split_method, self.N_split)
        self.positions = positions
        for e in epos:
            if not self.quiet:
                print("  [EELS] impact parameter", e)
            sp, sr, se = split_near_beam(positions, e, rad, eps, self.split_dist, offsets)
            sub = EELS(self.box, se, self.omega, self.v, eps_m=self.eps_m, radius=sr, xi=self.xi, tol=self.tol,
                       quiet=True, solver_type=self.solver_type, field_type=self.field_type,
                       asm_flag=self.asm, asm_Nx=self.asm_n[0], asm_Ny=self.asm_n[1], precision=self._precision)
            sub.use_jacobi_precond = self.use_jacobi_precond
            sub.compute(e, sp)
            self._eels.append(sub._eels[0])
            self._dips.append(sub._dips[0])
            self._split_pos.append(sp)
            # physical dipoles of a split system scale by the first particle's
            # radius, as the reference does (eels.py:469)
            self._dip_scale.append(self.eps_m * sr[0] ** 3)

    @staticmethod
    def _stack(items):
        if len(items) == 1:
            return np.squeeze(items[0])
        try:
            return np.squeeze(np.stack(items))
        except ValueError:
            return [np.squeeze(a) for a in items]

    def get_eels(self):
        """Loss probability, (num_epos, num_wavelengths), squeezed."""
        return np.squeeze(np.array(self._eels))

    def get_dipoles(self, physical=True):
        """Induced dipoles, (num_epos, num_wavelengths, N, 3), squeezed
        (a list when split systems differ in size); physical units multiply
        by eps_m * a_min^3 (eels_solver.h:155-160)."""
        if self._splitting():
            if not self._dips:
                return []
            d = [a * f for a, f in zip(self._dips, self._dip_scale)] if physical else list(self._dips)
            return self._stack(d)
        d = np.array(self._dips)
        if physical:
            d = d * (self.eps_m * self._ls ** 3)
        return np.squeeze(d)

    def get_quadrupoles(self, physical=True):
        raise RuntimeError("EELS quadrupoles are not available in this build")

    def get_positions(self):
        """Positions used: the split systems of every beam position when
        splitting, else the particles."""
        if self._splitting():
            return self._stack(self._split_pos) if self._split_pos else []
        return self.positions
