"""Stand-alone field operators: the reference's `cuMPM.dev` classes
(src/cuMPM/dev/electric_field.py: DirectElectricField :29,
MonodisperseEwaldElectricField :430, PolydisperseEwaldElectricField :845)
on this build's C-ABI field (`capi.Field`, include/cumpm_b200.h
mpm_field_*).

Same constructors, update / calculate / get_epoint_host methods and field
splits (`compute_real_field`, `compute_inverse_field`) as the reference;
`calculate()` is the reference's `Electric_Field::calculate()`: in
SOLVER_AX mode the interaction field plus the self terms set by
`set_self_coef`, in INTERACTION_FIELD mode the field at the field points.
The reference's accessors of its internal device buffers (`dev_*`,
`get_*_precalcs_host`, neighbour-list and table getters) have no
counterpart: this build's data layout is different.  Bloch wavevectors
(`set_bloch_wavevector`, ewald_electric_field_base.h:132-138) are taken for
dipoles; with quadrupoles they raise RuntimeError naming the gap.
"""
from __future__ import annotations

import numpy as np

from . import capi
from ._cuMPM import FieldCalcMode, PrecisionMode

__all__ = ["DirectElectricField", "MonodisperseEwaldElectricField", "PolydisperseEwaldElectricField",
           "FieldCalcMode", "PrecisionMode"]


def _vec(v):
    return np.atleast_1d(np.asarray(v, dtype=np.float64)).ravel()


def _parse_precision(precision):
    """The reference's rule (dev/electric_field.py:13-27)."""
    if precision is None:
        return PrecisionMode.AUTO
    if isinstance(precision, str):
        p = precision.lower()
        if p == "auto":
            return PrecisionMode.AUTO
        if p in ("mixed", "fp32", "single"):
            return PrecisionMode.MIXED
        if p in ("double", "fp64"):
            return PrecisionMode.DOUBLE
        raise ValueError(f"Unknown precision mode string: '{precision}'. Must be 'auto', 'mixed', or 'double'.")
    return precision


def _mode(m, default=FieldCalcMode.SOLVER_AX):
    if m is None:
        return default
    if isinstance(m, bool):
        return FieldCalcMode.SOLVER_AX if m else FieldCalcMode.INTERACTION_FIELD
    return m


class _Field:
    """State shared by the three field classes: host copies of the inputs,
    the device operator built on first use, the last result."""

    def __init__(self, kind, box, errortol, xi, mode, radius, solve_quadrupoles, quad_idxs, precision):
        self._kind = kind
        self._box = np.asarray(box, dtype=np.float64) if box is not None else None
        self._errortol = float(errortol)
        self._xi = float(xi)
        self._mode = mode
        self._radius = None if radius is None else _vec(radius)
        self._solve_quads = bool(solve_quadrupoles)
        self._quad_idxs = [int(i) for i in (quad_idxs or [])]
        self._prec = _parse_precision(precision)
        self._pos = np.zeros((0, 3))
        self._fpts = None
        self._dip = None
        self._quad = None
        self._self = None
        self._F = None
        self._built_for = None
        self._E = None
        self._bloch = (0.0, 0.0)

    # ---------------------------------------------------------- inputs --
    def update_particle_coordinates(self, x_part, y_part, z_part):
        self._pos = np.stack([_vec(x_part), _vec(y_part), _vec(z_part)], axis=1)

    def update_field_coordinates(self, x_field, y_field, z_field):
        self._fpts = np.stack([_vec(x_field), _vec(y_field), _vec(z_field)], axis=1)

    def update_dipoles(self, dip_x, dip_y, dip_z):
        self._dip = np.stack([_vec(dip_x), _vec(dip_y), _vec(dip_z)], axis=1).astype(complex)

    def update_dipoles_complex(self, dip_xr, dip_xi, dip_yr, dip_yi, dip_zr, dip_zi):
        self._dip = np.stack([_vec(dip_xr) + 1j * _vec(dip_xi), _vec(dip_yr) + 1j * _vec(dip_yi),
                              _vec(dip_zr) + 1j * _vec(dip_zi)], axis=1)

    def update_quadrupoles(self, quad_1, quad_2, quad_3, quad_4, quad_5):
        self._quad = np.stack([_vec(q) for q in (quad_1, quad_2, quad_3, quad_4, quad_5)], axis=1).astype(complex)

    def update_quadrupoles_complex(self, quad_1r, quad_1i, quad_2r, quad_2i, quad_3r, quad_3i, quad_4r, quad_4i,
                                   quad_5r, quad_5i):
        parts = (quad_1r, quad_1i, quad_2r, quad_2i, quad_3r, quad_3i, quad_4r, quad_4i, quad_5r, quad_5i)
        self._quad = np.stack([_vec(parts[2 * c]) + 1j * _vec(parts[2 * c + 1]) for c in range(5)], axis=1)

    def set_self_coef(self, self_coef_r, self_coef_i=None):
        n = self.num_particles
        r = _vec(self_coef_r) if np.iterable(self_coef_r) else np.full(n, float(self_coef_r))
        if self_coef_i is None:
            i = np.zeros(len(r))
        else:
            i = _vec(self_coef_i) if np.iterable(self_coef_i) else np.full(n, float(self_coef_i))
        self._self = r + 1j * i

    def set_bloch_wavevector(self, kx, ky):
        """Bloch wavevector (k_x, k_y) of the periodic images: the k-space
        Green tensor at k - b and a phase on every real-space pair
        (dipoles only in this build)."""
        if self._kind == capi.FIELD_DIRECT:
            raise RuntimeError("a direct field has no Bloch wavevector")
        if self._solve_quads and (kx != 0.0 or ky != 0.0):
            raise RuntimeError("Bloch wavevectors with quadrupoles are not available in this build")
        self._bloch = (float(kx), float(ky))

    # ------------------------------------------------------------ sizes --
    @property
    def num_particles(self) -> int:
        return len(self._pos)

    @property
    def num_field_points(self) -> int:
        return 0 if self._fpts is None else len(self._fpts)

    @property
    def solve_quadrupoles(self) -> bool:
        return self._solve_quads

    @property
    def num_quads(self) -> int:
        if not self._solve_quads:
            return 0
        return len(self._quad_idxs) if self._quad_idxs else self.num_particles

    @property
    def mode(self):
        return self._mode

    @property
    def errortol(self) -> float:
        return self._errortol

    @property
    def xi(self) -> float:
        return self._xi

    # ------------------------------------------------------------ solve --
    def _fp32(self):
        return self._prec in (PrecisionMode.MIXED, PrecisionMode.FP32)

    def _operator(self):
        n = self.num_particles
        if n == 0:
            raise RuntimeError("update_particle_coordinates before calculate")
        inter = self._mode == FieldCalcMode.INTERACTION_FIELD
        key = (n, None if self._fpts is None else len(self._fpts))
        if self._F is None or self._built_for != key:
            qi = None
            if self._solve_quads:
                qi = self._quad_idxs or list(range(n))
            self._F = capi.Field(self._kind, self._box, self._errortol, self._xi,
                                 mode=capi.MODE_INTERACTION if inter else capi.MODE_SOLVER_AX,
                                 radius=self._radius, quad_idxs=qi, solve_quads=self._solve_quads)
            self._built_for = key
        if inter:
            if self._fpts is None:
                raise RuntimeError("update_field_coordinates before calculate in INTERACTION_FIELD mode")
            self._F.set_field_points(self._fpts)
        self._F.set_positions(self._pos)
        self._F.set_bloch(*self._bloch)
        return self._F

    def _inputs(self):
        """(X, self terms) as CUDA tensors; every size is checked on the host
        first, so a mismatch never reaches a device call."""
        import torch

        n = self.num_particles
        dip = self._dip if self._dip is not None else np.zeros((n, 3), complex)
        if dip.shape != (n, 3):
            raise ValueError("dipoles must have one entry per particle")
        parts = [dip.ravel()]
        if self._solve_quads:
            nq = self.num_quads
            q = self._quad if self._quad is not None else np.zeros((nq, 5), complex)
            if q.shape != (nq, 5):
                raise ValueError("quadrupoles must have one entry per quadrupole index")
            parts.append(q.ravel())
        s = None
        if self._mode != FieldCalcMode.INTERACTION_FIELD:
            s = self._self if self._self is not None else np.zeros(n, complex)
            if len(s) != n:
                raise ValueError("self coefficients must have one entry per particle")
        X = torch.tensor(np.concatenate(parts).reshape(-1, 1), dtype=torch.complex128, device="cuda")
        sc = None if s is None else torch.tensor(np.asarray(s, dtype=complex).reshape(-1, 1), device="cuda")
        return X, sc

    def calculate(self):
        F = self._operator()
        X, sc = self._inputs()
        self._E = F.apply(X, self_coef=sc, recip_fp32=self._fp32(), real_fp32=self._fp32()).cpu().numpy()[:, 0]

    def clear_epoint(self):
        self._E = None

    def compute_real_field(self):
        """Real-space (pair and self) part of the field (the reference's
        clear_epoint + real_space); for the direct field, the whole field."""
        F = self._operator()
        X, sc = self._inputs()
        if self._kind == capi.FIELD_DIRECT:
            self._E = F.apply(X, self_coef=sc, recip_fp32=self._fp32()).cpu().numpy()[:, 0]
        else:
            self._E = F.apply_part(X, 1, self_coef=sc, recip_fp32=self._fp32(),
                                   real_fp32=self._fp32()).cpu().numpy()[:, 0]
        return self.get_epoint_host()

    def compute_inverse_field(self):
        """Total field minus its real-space part (the reference's definition)."""
        self.calculate()
        total = self.get_epoint_host()
        real = self.compute_real_field()
        if isinstance(total, tuple):
            return total[0] - real[0], total[1] - real[1]
        return total - real

    def get_epoint_host(self, reshape=True):
        if self._E is None:
            raise RuntimeError("calculate before get_epoint_host")
        raw = np.asarray(self._E, dtype=np.complex128)
        if not reshape:
            return raw
        nf = self.num_field_points if self._mode == FieldCalcMode.INTERACTION_FIELD else 0
        if nf == 0:
            nf = self.num_particles
        if self._solve_quads and self.num_quads > 0:
            return raw[:nf * 3].reshape((nf, 3)), raw[nf * 3:].reshape((self.num_quads, 5))
        return raw.reshape((nf, 3))

    def get_dipoles_host(self):
        d = self._dip if self._dip is not None else np.zeros((self.num_particles, 3), complex)
        return tuple(np.real(d[:, c]).copy() for c in range(3))

    def get_dipoles_complex_host(self):
        d = self._dip if self._dip is not None else np.zeros((self.num_particles, 3), complex)
        out = []
        for c in range(3):
            out += [np.real(d[:, c]).copy(), np.imag(d[:, c]).copy()]
        return tuple(out)


class DirectElectricField(_Field):
    """Open-boundary all-pairs field (dev/electric_field.py:29-428)."""

    def __init__(self, radius=None, mode=None, solve_quadrupoles=False, quad_idxs=None, precision=None):
        super().__init__(capi.FIELD_DIRECT, None, 1e-3, 0.5, _mode(mode),
                         None if radius is None or len(np.atleast_1d(radius)) == 0 else radius,
                         solve_quadrupoles, quad_idxs, precision)

    @property
    def is_using_fp32(self) -> bool:
        return self._fp32()

    @property
    def precision_mode(self):
        return self._prec


class _EwaldField(_Field):
    @property
    def is_using_recip_fp32(self) -> bool:
        return self._fp32()

    @property
    def recip_precision_mode(self):
        return self._prec

    @property
    def box_x(self) -> float:
        return float(self._box[0])

    @property
    def box_y(self) -> float:
        return float(self._box[1])

    @property
    def box_z(self) -> float:
        return float(self._box[2])


class MonodisperseEwaldElectricField(_EwaldField):
    """Spectral-Ewald field of equal spheres (dev/electric_field.py:430-843).
    Lengths are in units of the particle radius, as in the reference."""

    def __init__(self, box_x, box_y, box_z, errortol, xi, calc_inter_dipole, radius=1.0, solve_quadrupoles=False,
                 quad_idxs=None, precision=None):
        if float(radius) != 1.0:
            raise ValueError("the monodisperse field works in units of the particle radius (radius=1.0); "
                             "use PolydisperseEwaldElectricField for other radii")
        super().__init__(capi.FIELD_MONO, (box_x, box_y, box_z), errortol, xi, _mode(calc_inter_dipole), None,
                         solve_quadrupoles, quad_idxs, precision)


class PolydisperseEwaldElectricField(_EwaldField):
    """Spectral-Ewald field of spheres of different radii
    (dev/electric_field.py:845-1292), dipoles."""

    def __init__(self, box_x, box_y, box_z, errortol, xi, calc_inter_dipole, particle_radii, solve_quadrupoles=False,
                 quad_idxs=None, precision=None):
        super().__init__(capi.FIELD_POLY, (box_x, box_y, box_z), errortol, xi, _mode(calc_inter_dipole),
                         particle_radii, solve_quadrupoles, quad_idxs, precision)
