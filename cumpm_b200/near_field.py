"""``Near_Field``: intensity |E_ind + E0|^2 at arbitrary points.

Same API as the reference ``src/cuMPM/near_field.py`` (:4-126), evaluated by
the B200 field operator in INTERACTION_FIELD mode.
"""
from __future__ import annotations

import numpy as np

from . import _load

_cuMPM = _load.extension()


class Near_Field:
    def __init__(self, box, E0, radius=1.0, dip=None, dip_pos=None, field_points=None, xi=0.5, errortol=1e-3,
                 field_type="auto"):
        self.box = [float(x) for x in box]
        self.E0 = [complex(x) for x in E0]
        self.radius_list = [float(r) for r in radius] if np.iterable(radius) else [float(radius)]
        self.xi = float(xi)
        self.errortol = float(errortol)
        self.field_type = field_type
        self._near_field = _cuMPM.Near_Field(self.box, self.E0, self.radius_list, self.xi, self.errortol,
                                             self.field_type)
        if dip is not None:
            self.set_dipoles(dip)
        if dip_pos is not None:
            self.set_dipole_positions(dip_pos)
        if field_points is not None:
            self.set_field_points(field_points)

    def set_dipoles(self, dip):
        if dip is None:
            raise ValueError("dipoles can't be set to None")
        arr = np.asarray(dip, dtype=complex)
        self._near_field.set_dipoles(arr.ravel().tolist())

    def set_dipole_positions(self, dip_pos):
        if dip_pos is None:
            raise ValueError("dipole positions can't be set to None")
        p = np.asarray(dip_pos, dtype=float)
        self._near_field.set_dipole_positions(p[:, 0].tolist(), p[:, 1].tolist(), p[:, 2].tolist())

    def set_field_points(self, field_points):
        if field_points is None:
            raise ValueError("field points can't be set to None")
        p = np.asarray(field_points, dtype=float)
        self._near_field.set_field_points(p[:, 0].tolist(), p[:, 1].tolist(), p[:, 2].tolist())

    def calculate(self):
        return np.array(self._near_field.calculate())
