"""cumpm_b200: B200-native self-consistent dipole/quadrupole solve.

Drop-in for the reference ``cuMPM`` package (``dipole_solver``,
``drude_dielectric``, ``Near_Field``, ``EELS``, ``dev``) on hand-written
sm_100a kernels.
"""
from .solver import dipole_solver, drude_dielectric  # noqa: F401
from .near_field import Near_Field  # noqa: F401
from .eels import EELS  # noqa: F401
from . import capi  # noqa: F401
from . import dev  # noqa: F401
from . import io  # noqa: F401
from ._load import extension as _extension

_cuMPM = _extension()

__all__ = ["dipole_solver", "drude_dielectric", "Near_Field", "EELS", "dev", "capi", "io"]
