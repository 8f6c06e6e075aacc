"""``dipole_solver`` / ``drude_dielectric``: the reference Python API.

Same signatures, argument normalisation, error types and messages as the
reference ``src/cuMPM/solver.py`` (``drude_dielectric`` :4-51,
``dipole_solver`` :53-271), running on the B200 extension ``_cuMPM`` built
in this package.  Positions and permittivities may also be given as
PyTorch tensors (moved to host memory on entry); results are numpy arrays as
in the reference.
"""
from __future__ import annotations

import numpy as np

from . import _load

_cuMPM = _load.extension()


def _to_numpy(a):
    if hasattr(a, "detach") and hasattr(a, "cpu"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def _as_1d(value, message):
    if not np.iterable(value):
        return np.asarray([value])
    arr = np.asarray(value)
    if arr.ndim != 1:
        raise ValueError(message)
    return arr


def drude_dielectric(omega, gamma, omega_p, eps_inf):
    """Complex Drude permittivity eps_inf - omega_p^2 / (omega^2 + i omega gamma).

    Returns an array of shape (num_omega, num_materials), squeezed.
    """
    omega = _as_1d(_to_numpy(omega) if hasattr(omega, "cpu") else omega,
                   "omega must be a scalar or a 1-D array of wavenumbers")
    gamma = _as_1d(gamma, "gamma must be a scalar or a 1-D array of damping coefficients")
    omega_p = _as_1d(omega_p, "omega_p must be a scalar or a 1-D array of plasma frequencies")
    eps_inf = _as_1d(eps_inf, "eps_inf must be a scalar or a 1-D array of high frequency permitivities")
    if np.any(len(eps_inf) != np.array([len(gamma), len(omega_p)])):
        raise ValueError("eps_inf, gamma, and omega_p must all have the same number of values applied")
    eps = eps_inf[None, :] - omega_p[None, :] ** 2 / (omega[:, None] ** 2 + 1j * omega[:, None] * gamma[None, :])
    return np.squeeze(eps.astype(np.complex128))


_PRECISION_NAMES = {
    "mixed": "MIXED", "fp32": "MIXED", "float32": "MIXED", "single": "MIXED",
    "double": "DOUBLE", "fp64": "DOUBLE", "double64": "DOUBLE",
    "auto": "AUTO",
}


def _parse_precision(precision):
    if precision is None:
        return _cuMPM.PrecisionMode.AUTO
    if isinstance(precision, _cuMPM.PrecisionMode):
        return precision
    if isinstance(precision, str):
        key = precision.lower()
        if key not in _PRECISION_NAMES:
            raise ValueError(f"Unknown precision mode: {precision}")
        return getattr(_cuMPM.PrecisionMode, _PRECISION_NAMES[key])
    raise ValueError(f"Invalid precision type: {type(precision)}")


def _parse_E0(E0):
    if E0 is None:
        return []
    arr = _to_numpy(E0)
    if arr.ndim == 1:
        if arr.size % 3 != 0:
            raise ValueError("E0 size must be divisible by 3")
        return [[complex(v) for v in arr[i:i + 3]] for i in range(0, arr.size, 3)]
    if arr.ndim == 2:
        if arr.shape[1] % 3 != 0:
            raise ValueError("Each vector in E0 must be 3-dimensional or have a size that is a multiple of 3")
        return [[complex(v) for v in row] for row in arr]
    if arr.ndim == 3:
        if arr.shape[2] != 3:
            raise ValueError("The last dimension of E0 must be 3")
        return [[complex(v) for v in block.ravel()] for block in arr]
    raise ValueError("E0 must be a 1D, 2D, or 3D array")


class dipole_solver:
    """Self-consistent induced dipoles (and optionally quadrupoles) of N spheres.

    Drop-in for the reference ``cuMPM.dipole_solver``: restarted GMRES or
    BiCGSTAB with Jacobi preconditioning around a spectral-Ewald (periodic)
    or direct (open boundary) field operator, all on the GPU.  The
    polarisations of each frequency are solved as one batch.
    """

    def __init__(self, box, eps_p, radius=1.0, eps_m=1.0, xi=0.5, tol=1e-3, quiet=False,
                 guess_type="derivative", solver_type="gmres", field_type="auto", E0=None,
                 quadrupoles=False, precision=None):
        if field_type not in ("auto", "monodisperse", "polydisperse", "direct"):
            raise ValueError(
                f"field_type must be 'auto', 'monodisperse', 'polydisperse', or 'direct', got {field_type}")
        prec = _parse_precision(precision)
        box_list = [float(v) for v in _to_numpy(box).ravel()] if np.iterable(box) else [float(box)]
        if len(box_list) != 3:
            raise ValueError("box must have length 3")
        radius_list = [float(r) for r in np.ravel(_to_numpy(radius))] if np.iterable(radius) else [float(radius)]
        E0_list = _parse_E0(E0)
        if isinstance(quadrupoles, bool):
            solve_q, quad_idxs = quadrupoles, []
        elif np.iterable(quadrupoles):
            solve_q, quad_idxs = True, [int(i) for i in quadrupoles]
        else:
            raise TypeError("quadrupoles must be a boolean or a list/iterable of particle indices")
        eps = _to_numpy(eps_p)
        # the run's inputs, kept for result files (cumpm_b200.io.save_solution)
        self._args = {"box": np.array(box_list), "eps_p": np.asarray(eps, dtype=np.complex128),
                      "radius": np.array(radius_list), "eps_m": float(eps_m), "xi": float(xi), "tol": float(tol),
                      "E0": np.array(E0_list, dtype=np.complex128) if E0_list else np.eye(3, dtype=np.complex128)}
        args = (radius_list, float(eps_m), float(xi), float(tol), bool(quiet), guess_type, solver_type,
                field_type, E0_list, solve_q, quad_idxs, prec)
        if eps.ndim == 0 or (eps.ndim == 1 and eps.size == 1):
            self._solver = _cuMPM.Dipole_Solver(box_list, complex(eps.reshape(-1)[0]), *args)
        elif eps.ndim == 1:
            self._solver = _cuMPM.Dipole_Solver(box_list, [complex(v) for v in eps], *args)
        elif eps.ndim == 2:
            self._solver = _cuMPM.Dipole_Solver(box_list, [[complex(v) for v in row] for row in eps], *args)
        else:
            raise ValueError("eps_p must be a scalar, 1D array, or 2D array")

    def compute(self, positions):
        """Solve for positions of shape (N, 3) or (num_frames, N, 3)."""
        pos = _to_numpy(positions)
        if pos.ndim == 2:
            pos = pos[np.newaxis, ...]
        if pos.ndim != 3 or pos.shape[-1] != 3:
            raise ValueError("positions must be of shape (num_particles, 3) or (num_frames, num_particles, 3)")
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        if getattr(self, "_autotune_pending", False):
            self.autotune(pos[0])
        for frame in pos:
            self._solver.compute(np.ascontiguousarray(frame[:, 0]), np.ascontiguousarray(frame[:, 1]),
                                 np.ascontiguousarray(frame[:, 2]))

    def get_eff_polarizability(self, physical=True):
        """Frame- and particle-averaged dipole per polarisation, (W, K, 3) squeezed."""
        return np.squeeze(self._solver.get_eff_polarizability(physical))

    def get_dipoles(self, physical=True):
        """Dipoles, (frames, W, N, K, 3) squeezed."""
        return np.squeeze(self._solver.get_dipoles(physical))

    def get_quadrupoles(self, physical=True):
        """Quadrupoles of the quadrupole subset, (frames, W, Nq, K, 5) squeezed."""
        return np.squeeze(self._solver.get_quadrupoles(physical))

    def get_cap_dip(self):
        """Deprecated alias returning (get_eff_polarizability(), get_dipoles())."""
        return self.get_eff_polarizability(), self.get_dipoles()

    @property
    def use_jacobi_precond(self) -> bool:
        return self._solver.isUsingJacobiPrecond()

    @use_jacobi_precond.setter
    def use_jacobi_precond(self, enable: bool):
        self._solver.setUseJacobiPrecond(bool(enable))

    # ---- extensions beyond the reference API --------------------------------
    def set_solver_options(self, restart=50, maxiter=1000, batch_all=False, refine=False, inner_tol=1e-4,
                           real_fp32=False, autotune=False):
        """GMRES restart/maxiter, all-frequency batching, mixed-precision refinement.

        Each fp32 inner solve of the refinement reduces a column's residual by
        at most inner_tol and stops earlier once that column's residual is
        below half the outer tolerance.  ``autotune=True`` tunes the field on
        the next frame's positions before solving it (see ``autotune``).
        """
        self._solver.set_solver_options(restart, maxiter, batch_all, refine, inner_tol, real_fp32)
        self._autotune_pending = bool(autotune)

    def autotune(self, positions):
        """Tune the Ewald field for these positions (N, 3) and this solver's
        batch width and arithmetic: the splitting parameter xi, the grid, the
        Gaussian support and the spread tile are measured on the device and
        the fastest setting whose operator error stays within
        max(tol, the error of the reference's rule setting) is kept for
        every later frame.  Returns the pick (xi non-dimensional, zeros =
        the rule) with its timings and errors."""
        pos = np.ascontiguousarray(_to_numpy(positions), dtype=np.float64)
        if pos.ndim != 2 or pos.shape[-1] != 3:
            raise ValueError("positions must be of shape (num_particles, 3)")
        out = self._solver.autotune(pos[:, 0].tolist(), pos[:, 1].tolist(), pos[:, 2].tolist())
        self._autotune_pending = False
        return dict(out)

    def set_tuning(self, xi, grid=(0, 0, 0), support=0, tile=(0, 0)):
        """Use this field setting (xi non-dimensional; zeros keep the rule)."""
        self._solver.set_tuning(float(xi), tuple(int(g) for g in grid), int(support), tuple(int(t) for t in tile))
        self._autotune_pending = False

    def get_iterations(self):
        """Krylov steps of every right-hand side solved so far (solve order)."""
        return list(self._solver.get_iterations())
