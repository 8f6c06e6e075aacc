"""CPU oracle for the cuMPM self-consistent dipole/quadrupole solve.

TEST INFRASTRUCTURE ONLY.  This module is a float64 numpy restatement of the
reference algorithm (cuMPM, ``src/cpp``) used as the checker for the CUDA
path in ``cumpm_b200``.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it; the product never does.

What it restates (reference ``file:line``):

* monodisperse spectral-Ewald operator
  - parameters: ``electric_field/monodisperse_ewald_electric_field.cu:546-616``
  - real-space tables: ``...monodisperse_ewald_electric_field.cu:92-542``
  - table interpolation: ``...monodisperse_ewald_electric_field.cu:668-685``
  - Gaussian spread / contract weights: ``...:687-816, 960-1069``
  - reciprocal scale coefficients: ``...:1300-1404``
  - scale (dipole and joint dipole/quadrupole): ``...:1406-1486``
  - contraction: ``...:1488-1587``
  - real-space self and pair terms: ``...:1589-1869``
  - stage order and INTERACTION_FIELD sign: ``...:2211-2411``
* neighbour search (minimum image, ``d^2 <= rc^2``):
  ``electric_field/neighbor_list.cu:186-223``
* polydisperse spectral-Ewald dipole operator
  (``electric_field/polydisperse_ewald_electric_field.cu``): radius classes
  ``:39-84``, parameters ``:2039-2112``, pair functions ``:1434-1627``,
  table nodes and interpolation ``:170-187, 1629-1687``, spread weights
  ``:189-350``, scale ``:565-651``, contraction ``:653-693``, real space
  ``:352-441, 695-826``, stage order ``:2553-2730``
* polydisperse quadrupoles on the same scalar grid: radius-1 quadrupole
  tables ``:1690-2035`` (gq2 and gq3 are the polydisperse field's own
  expressions), point-Gaussian weights ``:828-922, 2114-2278``, joint scale
  ``:565-638, 925-962``, spread and G contraction ``:964-1146``, joint self
  and pair terms ``:1148-1428``.  Pinned by the shared tables against the
  reference CPU operator's fixtures and by the reference's own solver-level
  checks (equal radii against the monodisperse quadrupole solve, mixed radii
  in a large box against the direct sum); not yet against the reference
  build's polydisperse quadrupole field.
* Bloch wavevector (k_x, k_y) in both Ewald operators: shifted k in the
  scales (``monodisperse...cu:1329-1330``, ``polydisperse...cu:592-593``)
  and a phase exp(-i(k_x r_x + k_y r_y)) on every pair term
  (``monodisperse...cu:1749-1858``, ``polydisperse...cu:799-806,
  1339-1419``); pinned by the reference's mono/poly Bloch check
  (``tests/test_electric_fields.py:226-284``)
* open-boundary direct sum: ``electric_field/direct_electric_field.cu:42-324``
* Krylov solvers: ``numerical_solver/gmres_solver.cu:56-208``,
  ``numerical_solver/bicgstab_solver.cu:58-192``, Jacobi
  ``numerical_solver/numerical_solver.cu:207-242``
* driver: ``dipole_solver.cu:131-647``
* near field: ``near_field.cu:78-213``

Parity is pinned by ``tests/test_oracle_golden.py`` against the reference's
own golden vectors (``tests/data/*.npz`` of the reference, re-saved under
``tests/golden``) and against fixtures produced by the reference's CPU
operator ``tests/quadrupole_field.py`` (generator script:
``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import math
import numpy as np
from scipy.special import erfc

PI = math.pi

# ---------------------------------------------------------------------------
# small helpers
# ---------------------------------------------------------------------------


def c_round(x):
    """C ``round()``: halves away from zero (numpy rounds halves to even)."""
    x = np.asarray(x, dtype=np.float64)
    return (np.sign(x) * np.floor(np.abs(x) + 0.5)).astype(np.int64)


def _combo(r, xi, ep, em, e0, fp, fm, f0, reg):
    """exp/erfc combination shared by every real-space table entry."""
    x2 = xi * xi
    out = (ep * np.exp(-(r + 2.0) ** 2 * x2) + fp * erfc((r + 2.0) * xi)
           + em * np.exp(-(r - 2.0) ** 2 * x2) + fm * erfc((r - 2.0) * xi)
           + e0 * np.exp(-r * r * x2) + f0 * erfc(r * xi))
    return out + np.where(r < 2.0, reg, 0.0)


# ---------------------------------------------------------------------------
# Monodisperse Ewald parameters (monodisperse_ewald_electric_field.cu:546-616)
# ---------------------------------------------------------------------------


class MonoParams:
    def __init__(self, box, errortol, xi):
        box = np.asarray(box, dtype=np.float64)
        self.box = box
        self.errortol = float(errortol)
        self.xi = float(xi)
        rc = math.sqrt(-math.log(errortol)) / xi
        if rc < 2.0:
            rc = 2.0
        if rc > box[0] / 2.0 or rc > box[1] / 2.0 or rc > box[2] / 2.0:
            raise RuntimeError("Real space cutoff (%f) larger than half the box length." % rc)
        self.rc = rc
        kcut = 2.0 * xi * xi * rc
        self.num_grid = np.array([int(math.ceil(1.0 + b * kcut / PI)) for b in box])
        self.h = box / self.num_grid
        self.P = int(math.ceil(-2.0 * math.log(errortol) / PI))
        self.eta = self.P * (self.h * xi) ** 2 / PI
        off = self.P // 2
        self.offsets = np.arange(-off, off + 1)


# ---------------------------------------------------------------------------
# Real-space tables (monodisperse_ewald_electric_field.cu:92-542)
# ---------------------------------------------------------------------------

TABLE_STEPS = 9000
TABLE_DR = 0.001


def mono_real_tables(xi, r=None, variant="mono"):
    """Return (r_table, dict name->values, selfo, self_grad).

    Entry 0 is r=0 (the self value); entries 1.. are r = 1 + k*0.001, 9000
    of them unless ``r`` gives the nodes (the polydisperse field sizes its
    table by the cutoff, polydisperse_ewald_electric_field.cu:1629-1645).
    Names: fd1 (perp), fd2 (para), fq1, fq2, fq3, gq1..gq4.

    ``variant="poly"`` gives the radius-1 quadrupole tables the polydisperse
    field builds for itself (:1697-2035): fq1-fq3, gq1 and gq4 are the
    monodisperse expressions, gq2 is a different expression and gq3 carries
    the opposite sign on the r^5 and r^4 terms of its exp(-(r+2)^2 xi^2)
    coefficient.
    """
    if variant not in ("mono", "poly"):
        raise ValueError("variant must be 'mono' or 'poly'")
    if r is None:
        r = 1.0 + np.arange(TABLE_STEPS) * TABLE_DR
    r = np.asarray(r, dtype=np.float64)
    x = xi
    x2, x4, x6, x8, x10 = x ** 2, x ** 4, x ** 6, x ** 8, x ** 10
    x5, x7, x9 = x ** 5, x ** 7, x ** 9
    sp = PI ** 1.5
    r2, r3, r4, r5, r6 = r ** 2, r ** 3, r ** 4, r ** 5, r ** 6
    r7, r8, r9, r10 = r ** 7, r ** 8, r ** 9, r ** 10
    t = {}

    # field_dip_1 (:132-165)
    ep = (4 * x4 * r5 - 8 * x4 * r4 + 8 * x2 * (2 - 7 * x2) * r3 - 8 * x2 * (3 + 2 * x2) * r2
          + (3 - 12 * x2 + 32 * x4) * r + 2 * (3 + 4 * x2 - 32 * x4)) / (1024 * sp * x5 * r3)
    em = (4 * x4 * r5 + 8 * x4 * r4 + 8 * x2 * (2 - 7 * x2) * r3 + 8 * x2 * (3 + 2 * x2) * r2
          + (3 - 12 * x2 + 32 * x4) * r - 2 * (3 + 4 * x2 - 32 * x4)) / (1024 * sp * x5 * r3)
    e0 = (-4 * x4 * r4 - 8 * x2 * (2 - 9 * x2) * r2 - 3 + 36 * x2) / (512 * sp * x5 * r2)
    fp = (-8 * x6 * r6 - 36 * x4 * (1 - 4 * x2) * r4 + 256 * x6 * r3 - 18 * x2 * (1 - 8 * x2) * r2
          + 3 - 36 * x2 + 256 * x6) / (2048 * PI * x6 * r3)
    fm = (-8 * x6 * r6 - 36 * x4 * (1 - 4 * x2) * r4 - 256 * x6 * r3 - 18 * x2 * (1 - 8 * x2) * r2
          + 3 - 36 * x2 + 256 * x6) / (2048 * PI * x6 * r3)
    f0 = (8 * x6 * r6 + 36 * x4 * (1 - 4 * x2) * r4 + 18 * x2 * (1 - 8 * x2) * r2 - 3 + 36 * x2) / (1024 * PI * x6 * r3)
    reg = -1.0 / (4 * PI * r3) + (1.0 - 9.0 * r / 16.0 + r3 / 32.0) / (4 * PI)
    t["fd1"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)

    # field_dip_2 (:167-197)
    ep = (8 * x4 * r5 - 16 * x4 * r4 + 2 * x2 * (7 - 20 * x2) * r3 - 4 * x2 * (3 - 4 * x2) * r2
          - (3 - 12 * x2 + 32 * x4) * r - 2 * (3 + 4 * x2 - 32 * x4)) / (512 * sp * x5 * r3)
    em = (8 * x4 * r5 + 16 * x4 * r4 + 2 * x2 * (7 - 20 * x2) * r3 + 4 * x2 * (3 - 4 * x2) * r2
          - (3 - 12 * x2 + 32 * x4) * r + 2 * (3 + 4 * x2 - 32 * x4)) / (512 * sp * x5 * r3)
    e0 = (-8 * x4 * r4 - 2 * x2 * (7 - 36 * x2) * r2 + 3 - 36 * x2) / (256 * sp * x5 * r2)
    fp = (-16 * x6 * r6 - 36 * x4 * (1 - 4 * x2) * r4 + 128 * x6 * r3 - 3 + 36 * x2 - 256 * x6) / (1024 * PI * x6 * r3)
    fm = (-16 * x6 * r6 - 36 * x4 * (1 - 4 * x2) * r4 - 128 * x6 * r3 - 3 + 36 * x2 - 256 * x6) / (1024 * PI * x6 * r3)
    f0 = (16 * x6 * r6 + 36 * x4 * (1 - 4 * x2) * r4 + 3 - 36 * x2) / (512 * PI * x6 * r3)
    reg = 1.0 / (2 * PI * r3) + (1.0 - 9.0 * r / 8.0 + r3 / 8.0) / (4 * PI)
    t["fd2"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)

    # field_quad_1 (:199-234)
    c = 15.0 / (16384 * sp * x7 * r4)
    ep = c * (-24 * x6 * r7 - 4 * x4 * (9 - 8 * x2) * r5 + 8 * x4 * (3 - 8 * x2) * r4 + 48 * x6 * r6
              + 2 * x2 * (21 - 80 * x2 + 64 * x4) * r3 - 4 * x2 * (3 - 8 * x2) ** 2 * r2
              - (45 - 120 * x2 + 192 * x4 - 512 * x6) * r - 2 * (45 + 24 * x2 - 64 * x4 + 512 * x6))
    em = c * (-24 * x6 * r7 - 4 * x4 * (9 - 8 * x2) * r5 - 8 * x4 * (3 - 8 * x2) * r4 - 48 * x6 * r6
              + 2 * x2 * (21 - 80 * x2 + 64 * x4) * r3 + 4 * x2 * (3 - 8 * x2) ** 2 * r2
              - (45 - 120 * x2 + 192 * x4 - 512 * x6) * r + 2 * (45 + 24 * x2 - 64 * x4 + 512 * x6))
    e0 = 15.0 / (8192 * sp * x7 * r3) * (24 * x6 * r6 + 4 * x4 * (9 - 32 * x2) * r4
                                          - 2 * x2 * (21 - 128 * x2) * r2 + 45 - 480 * x2)
    c = 15.0 / (32768 * PI * x8 * r4)
    fp = c * (48 * x8 * r8 + 32 * x6 * (3 - 8 * x2) * r6 - 24 * x4 * (3 - 16 * x2) * r4
              + 72 * x2 * (1 - 8 * x2) * r2 - 45 + 480 * x2 + 4096 * x8)
    fm = fp
    f0 = 15.0 / (16384 * PI * x8 * r4) * (-48 * x8 * r8 - 32 * x6 * (3 - 8 * x2) * r6
                                          + 24 * x4 * (3 - 16 * x2) * r4 - 72 * x2 * (1 - 8 * x2) * r2
                                          + 45 - 480 * x2)
    reg = -15.0 / (4 * PI * r4) + 15.0 * r2 / (64 * PI) * (1.0 - 3.0 * r2 / 16.0)
    t["fq1"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)

    # field_quad_2 (:236-273)
    c = 3.0 / (16384 * sp * x7 * r4)
    ep = c * (-40 * x6 * r7 + 80 * x6 * r6 - 20 * x4 * (11 - 24 * x2) * r5 + 8 * x4 * (45 + 8 * x2) * r4
              - 2 * x2 * (45 - 80 * x2 + 64 * x4) * r3 - 4 * x2 * (15 + 48 * x2 - 64 * x4) * r2
              + (45 - 120 * x2 + 192 * x4 - 512 * x6) * r + 2 * (45 + 24 * x2 - 64 * x4 + 512 * x6))
    em = c * (-40 * x6 * r7 - 80 * x6 * r6 - 20 * x4 * (11 - 24 * x2) * r5 - 8 * x4 * (45 + 8 * x2) * r4
              - 2 * x2 * (45 - 80 * x2 + 64 * x4) * r3 + 4 * x2 * (15 + 48 * x2 - 64 * x4) * r2
              + (45 - 120 * x2 + 192 * x4 - 512 * x6) * r - 2 * (45 + 24 * x2 - 64 * x4 + 512 * x6))
    e0 = 15.0 / (8192 * sp * x7 * r3) * (8 * x6 * r6 + 4 * x4 * (11 - 32 * x2) * r4
                                          + 2 * x2 * (9 - 64 * x2) * r2 - 9 + 96 * x2)
    c = 3.0 / (32768 * PI * x8 * r4)
    fp = c * (80 * x8 * r8 + 160 * x6 * (3 - 8 * x2) * r6 - 2048 * x8 * r5 + 120 * x4 * (3 - 16 * x2) * r4
              - 120 * x2 * (1 - 8 * x2) * r2 + 45 - 480 * x2 - 4096 * x8)
    fm = c * (80 * x8 * r8 + 160 * x6 * (3 - 8 * x2) * r6 + 2048 * x8 * r5 + 120 * x4 * (3 - 16 * x2) * r4
              - 120 * x2 * (1 - 8 * x2) * r2 + 45 - 480 * x2 - 4096 * x8)
    f0 = 15.0 / (16384 * PI * x8 * r4) * (-16 * x8 * r8 - 32 * x6 * (3 - 8 * x2) * r6
                                          - 24 * x4 * (3 - 16 * x2) * r4 + 24 * x2 * (1 - 8 * x2) * r2
                                          - 9 + 96 * x2)
    reg = 3.0 / (4 * PI * r4) - 3.0 * r / (8 * PI) * (1.0 - 5.0 * r / 8.0 + 5.0 * r3 / 128.0)
    t["fq2"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)

    # field_quad_3 (:275-299)
    c = 5.0 / (1024 * sp * x5 * r2)
    ep = c * (4 * x4 * r5 - 8 * x4 * r4 + 16 * x2 * (1 - 2 * x2) * r3 - 24 * x2 * r2 + 3 * r + 6)
    em = c * (4 * x4 * r5 + 8 * x4 * r4 + 16 * x2 * (1 - 2 * x2) * r3 + 24 * x2 * r2 + 3 * r - 6)
    e0 = 5.0 / (512 * sp * x5 * r) * (-4 * x4 * r4 - 16 * x2 * (1 - 3 * x2) * r2 - 3 + 24 * x2)
    c = 5.0 / (2048 * PI * x6 * r2)
    fp = c * (-8 * x6 * r6 - 12 * x4 * (3 - 8 * x2) * r4 + 128 * x6 * r3 - 6 * x2 * (3 - 16 * x2) * r2 + 3 - 24 * x2)
    fm = c * (-8 * x6 * r6 - 12 * x4 * (3 - 8 * x2) * r4 - 128 * x6 * r3 - 6 * x2 * (3 - 16 * x2) * r2 + 3 - 24 * x2)
    f0 = 5.0 / (1024 * PI * x6 * r2) * (8 * x6 * r6 + 12 * x4 * (3 - 8 * x2) * r4
                                        + 6 * x2 * (3 - 16 * x2) * r2 - 3 + 24 * x2)
    reg = 5.0 * r / (8 * PI) * (1.0 - 3.0 * r / 4.0 + r3 / 16.0)
    t["fq3"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)

    # grad_quad_1 (:301-330)
    c = 75.0 / (16384 * sp * x7 * r3)
    ep = c * (8 * x6 * r7 - 16 * x6 * r6 + (44 * x4 - 32 * x6) * r5 - (72 * x4 - 64 * x6) * r4
              + (18 * x2 + 32 * x4) * r3 + (12 * x2 - 64 * x4) * r2 - (9 + 24 * x2) * r - (18 - 48 * x2))
    em = c * (8 * x6 * r7 + 16 * x6 * r6 + (44 * x4 - 32 * x6) * r5 + (72 * x4 - 64 * x6) * r4
              + (18 * x2 + 32 * x4) * r3 - (12 * x2 - 64 * x4) * r2 - (9 + 24 * x2) * r + (18 - 48 * x2))
    e0 = -75.0 / (8192 * sp * x7 * r2) * (8 * x6 * r6 + (44 * x4 - 64 * x6) * r4
                                          + (18 * x2 - 64 * x4 + 128 * x6) * r2 - 9 + 48 * x2 - 192 * x4)
    poly = (16 * x8 * r8 + (96 * x6 - 128 * x8) * r6 + (72 * x4 - 192 * x6 + 256 * x8) * r4
            - (24 * x2 - 96 * x4 + 256 * x6) * r2 + 9 - 48 * x2 + 192 * x4)
    fp = -75.0 / (32768 * PI * x8 * r3) * poly
    fm = fp
    f0 = 75.0 / (16384 * PI * x8 * r3) * poly
    reg = 75.0 * r * (4.0 - r2) ** 2 / (1024 * PI)
    t["gq1"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)

    # grad_quad_2 (:332-373)
    c = 3.0 / (32768 * sp * x9 * r5)
    ep = c * (-48 * x8 * r9 + 96 * x8 * r8 - (576 * x6 - 608 * x8) * r7 + (1056 * x6 - 1216 * x8) * r6
              - (1536 * x4 - 2576 * x6 + 3968 * x8) * r5 + (2160 * x4 - 4320 * x6 - 256 * x8) * r4
              - (360 * x2 + 360 * x4 + 640 * x6 - 512 * x8) * r3
              - (360 * x2 - 1680 * x4 - 768 * x6 + 1024 * x8) * r2
              + (135 + 180 * x2 + 480 * x4 - 768 * x6 + 2048 * x8) * r
              + (270 - 1080 * x2 - 192 * x4 + 512 * x6 - 4096 * x8))
    em = c * (-48 * x8 * r9 - 96 * x8 * r8 - (576 * x6 - 608 * x8) * r7 - (1056 * x6 - 1216 * x8) * r6
              - (1536 * x4 - 2576 * x6 + 3968 * x8) * r5 - (2160 * x4 - 4320 * x6 - 256 * x8) * r4
              - (360 * x2 + 360 * x4 + 640 * x6 - 512 * x8) * r3
              + (360 * x2 - 1680 * x4 - 768 * x6 + 1024 * x8) * r2
              + (135 + 180 * x2 + 480 * x4 - 768 * x6 + 2048 * x8) * r
              - (270 - 1080 * x2 - 192 * x4 + 512 * x6 - 4096 * x8))
    e0 = 1.0 / (16384 * sp * x9 * r4) * (144 * x8 * r8 + (1728 * x6 - 2400 * x8) * r6
                                         + (4608 * x4 - 13200 * x6 + 19200 * x8) * r4
                                         + (1080 * x2 - 5400 * x4 + 19200 * x6) * r2
                                         - 405 + 2700 * x2 - 14400 * x4)
    base = (288 * x10 * r10 + (3600 * x8 - 4800 * x10) * r8
            + (10800 * x6 - 28800 * x8 + 38400 * x10) * r6
            + (5400 * x4 - 21600 * x6 + 57600 * x8) * r4
            - (1350 * x2 - 7200 * x4 + 28800 * x6) * r2 + 405 - 2700 * x2 + 14400 * x4)
    fp = (base + 49152 * x10 * r5 + 49152 * x10) / (65536 * PI * x10 * r5)
    fm = (base - 49152 * x10 * r5 + 49152 * x10) / (65536 * PI * x10 * r5)
    f0 = -base / (32768 * PI * x10 * r5)
    reg = -3.0 / (2 * PI) * (1.0 / r5 - 1.0 + 25.0 * r / 32.0 - 25.0 * r3 / 256.0 + 3.0 * r5 / 512.0)
    t["gq2"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)
    if variant == "poly":
        # polydisperse grad_quad_2 (:1890-1924): odd and even parts of the
        # exp(-(r -+ 2)^2 xi^2) polynomials, one erfc polynomial
        c = -15.0 / (16384 * sp * x7 * r3)
        odd = (24 * x6 * r7 + (148 * x4 - 96 * x6) * r5 + (90 * x2 + 72 * x4 + 256 * x8) * r3
               - (45 + 120 * x2 - 192 * x4 + 512 * x6) * r)
        even = (-48 * x6 * r6 - (264 * x4 - 192 * x6) * r4 + (60 * x2 - 144 * x4 + 512 * x8) * r2
                - 2 * (45 + 24 * x2 - 64 * x4 + 512 * x6))
        ep, em = c * (odd + even), c * (odd - even)
        e0 = 75.0 / (8192 * sp * x7 * r2) * (8 * x6 * r6 + (44 * x4 - 64 * x6) * r4
                                             + (18 * x2 - 48 * x4 + 128 * x6) * r2 - 9 + 40 * x2 - 192 * x4)
        base = (48 * x8 * r8 + (288 * x6 - 384 * x8) * r6 + (216 * x4 - 576 * x6 + 768 * x8) * r4
                - (72 * x2 - 288 * x4 + 768 * x6) * r2 + 45 - 240 * x2 + 960 * x4)
        fp = -15.0 / (32768 * PI * x8 * r3) * (base - 4096 * x8 * r5 - 8192 * x8)
        fm = -15.0 / (32768 * PI * x8 * r3) * (base + 4096 * x8 * r5 - 8192 * x8)
        f0 = 15.0 / (16384 * PI * x8 * r3) * base
        reg = -45.0 * r / (32 * PI) * (1.0 - 5.0 * r2 / 12.0 + r4 / 16.0)
        t["gq2"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)

    # grad_quad_3 (:375-416)
    c = -15.0 / (65536 * sp * x9 * r5)
    s54 = -1.0 if variant == "poly" else 1.0
    ep = c * (48 * x8 * r9 - 96 * x8 * r8 + (336 * x6 - 288 * x8) * r7 - 576 * (x6 - x8) * r6
              + s54 * ((216 * x4 + 144 * x6 + 128 * x8) * r5 - (480 * x6 + 256 * x8) * r4)
              - (180 * x2 - 120 * x4 + 640 * x6 - 512 * x8) * r3
              + (720 * x4 + 768 * x6 - 1024 * x8) * r2
              + (135 + 180 * x2 + 480 * x4 - 768 * x6 + 2048 * x8) * r
              - (-270 + 1080 * x2 + 192 * x4 - 512 * x6 + 4096 * x8))
    em = c * (48 * x8 * r9 + 96 * x8 * r8 + (336 * x6 - 288 * x8) * r7 + 576 * (x6 - x8) * r6
              + (216 * x4 + 144 * x6 + 128 * x8) * r5 + (480 * x6 + 256 * x8) * r4
              - (180 * x2 - 120 * x4 + 640 * x6 - 512 * x8) * r3
              - (720 * x4 + 768 * x6 - 1024 * x8) * r2
              + (135 + 180 * x2 + 480 * x4 - 768 * x6 + 2048 * x8) * r
              + (-270 + 1080 * x2 + 192 * x4 - 512 * x6 + 4096 * x8))
    e0 = 15.0 / (32768 * sp * x9 * r4) * (48 * x8 * r8 + (336 * x6 - 480 * x8) * r6
                                          + (216 * x4 - 720 * x6 + 1280 * x8) * r4
                                          - (180 * x2 - 840 * x4 + 2560 * x6) * r2
                                          + 135 - 900 * x2 + 4800 * x4)
    base = (-96 * x10 * r10 + (-720 * x8 + 960 * x10) * r8
            - (720 * x6 - 1920 * x8 + 2560 * x10) * r6
            + (360 * x4 - 1440 * x6 + 3840 * x8) * r4
            - (270 * x2 - 1440 * x4 + 5760 * x6) * r2 + 135 - 900 * x2 + 4800 * x4)
    fp = -15.0 / (131072 * PI * x10 * r5) * (base + 16384 * x10)
    fm = fp
    f0 = 15.0 / (65536 * PI * x10 * r5) * base
    reg = -15.0 * (r2 - 4.0) ** 3 * (3.0 * r4 + 6.0 * r2 + 8.0) / (2048 * PI * r5)
    t["gq3"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)

    # grad_quad_4 (:418-459)
    c = -15.0 / (65536 * sp * x9 * r5)
    ep = c * (144 * x8 * r9 - 288 * x8 * r8 + (288 * x6 + 96 * x8) * r7 - (288 * x6 + 192 * x8) * r6
              - (432 * x4 - 912 * x6 + 896 * x8) * r5 + (720 * x4 - 480 * x6 + 1792 * x8) * r4
              + (720 * x2 - 2280 * x4 + 4480 * x6 - 3584 * x8) * r3
              - (1080 * x2 + 2160 * x4 + 5376 * x6 - 7168 * x8) * r2
              - (945 + 1260 * x2 + 3360 * x4 - 5376 * x6 + 14336 * x8) * r
              - (1890 - 7560 * x2 - 1344 * x4 + 3584 * x6 - 28672 * x8))
    em = c * (144 * x8 * r9 + 288 * x8 * r8 + (288 * x6 + 96 * x8) * r7 + (288 * x6 + 192 * x8) * r6
              - (432 * x4 - 912 * x6 + 896 * x8) * r5 - (720 * x4 - 480 * x6 + 1792 * x8) * r4
              + (720 * x2 - 2280 * x4 + 4480 * x6 - 3584 * x8) * r3
              + (1080 * x2 + 2160 * x4 + 5376 * x6 - 7168 * x8) * r2
              - (945 + 1260 * x2 + 3360 * x4 - 5376 * x6 + 14336 * x8) * r
              + (1890 - 7560 * x2 - 1344 * x4 + 3584 * x6 - 28672 * x8))
    e0 = 15.0 / (32768 * sp * x9 * r4) * (144 * x8 * r8 + (288 * x6 - 480 * x8) * r6
                                          - (432 * x4 - 1200 * x6 + 1280 * x8) * r4
                                          + (720 * x2 - 3000 * x4 + 6400 * x6) * r2
                                          - 945 + 6300 * x2 - 33600 * x4)
    base = (288 * x10 * r10 + (720 * x8 - 960 * x10) * r8
            - (720 * x6 - 1920 * x8 + 2560 * x10) * r6
            + (1080 * x4 - 4320 * x6 + 11520 * x8) * r4
            - (1350 * x2 - 7200 * x4 + 28800 * x6) * r2 + 945 - 6300 * x2 + 33600 * x4)
    fp = 15.0 / (131072 * PI * x10 * r5) * (base + 114688 * x10)
    fm = fp
    f0 = -15.0 / (65536 * PI * x10 * r5) * base
    reg = -15.0 * (3584.0 - 80.0 * r6 - 30.0 * r8 + 9.0 * r10) / (2048 * PI * r5)
    t["gq4"] = _combo(r, x, ep, em, e0, fp, fm, f0, reg)

    # self values (:462-467)
    selfo = ((-1.0 + 6.0 * x2 + (1.0 - 2.0 * x2) * math.exp(-4.0 * x2)) / (16.0 * sp * x ** 3)
             + math.erfc(2.0 * x) / (4.0 * PI))
    self_grad = 0.5 / PI * (3.0 * (3.0 - 10.0 * x2 + 20.0 * x4) / (8.0 * math.sqrt(PI) * x5)
                            - 3.0 * (3.0 + 2.0 * x2 + 4.0 * x4) * math.exp(-4.0 * x2) / (8.0 * math.sqrt(PI) * x5)
                            + 3.0 * math.erfc(2.0 * x))
    r_table = np.concatenate([[0.0], r])
    head = {"fd1": selfo, "fd2": selfo, "fq1": 0.0, "fq2": 0.0, "fq3": 0.0,
            "gq1": self_grad, "gq2": self_grad, "gq3": self_grad, "gq4": self_grad}
    tables = {k: np.concatenate([[head[k]], v]) for k, v in t.items()}
    return r_table, tables, selfo, self_grad


def interp_table(r, r_table, y):
    """Linear table lookup (monodisperse_ewald_electric_field.cu:668-685)."""
    r = np.asarray(r, dtype=np.float64)
    n = len(r_table)
    out = np.empty_like(r)
    lo = r <= 0.0
    hi = (~lo) & (r >= r_table[n - 1])
    sub = (~lo) & (~hi) & (r < 1.0)
    mid = (~lo) & (~hi) & (~sub)
    out[lo] = y[0]
    out[hi] = y[n - 1]
    out[sub] = y[0] * (1.0 - r[sub]) + y[1] * r[sub]
    rm = r[mid]
    idx = 1 + ((rm - 1.0) / TABLE_DR).astype(np.int64)
    over = idx >= n - 1
    idx_c = np.minimum(idx, n - 2)
    r0 = r_table[idx_c]
    r1 = r_table[idx_c + 1]
    tt = (rm - r0) / (r1 - r0)
    val = y[idx_c] * (1.0 - tt) + y[idx_c + 1] * tt
    val = np.where(over, y[n - 1], val)
    out[mid] = val
    return out


# ---------------------------------------------------------------------------
# Reciprocal space (monodisperse_ewald_electric_field.cu:1300-1404)
# ---------------------------------------------------------------------------


def _freqs(n):
    i = np.arange(n)
    return np.where(i <= (n - 1) // 2, i, i - n).astype(np.float64)


def mono_scale(params: MonoParams, quads=False, bloch=(0.0, 0.0)):
    Nx, Ny, Nz = params.num_grid
    L = params.box
    xi = params.xi
    fx, fy, fz = _freqs(Nx), _freqs(Ny), _freqs(Nz)
    Gx = fx * 2 * PI / L[0]
    Gy = fy * 2 * PI / L[1]
    Gz = fz * 2 * PI / L[2]
    kx = (Gx - bloch[0])[:, None, None]
    ky = (Gy - bloch[1])[None, :, None]
    kz = Gz[None, None, :]
    ksq = kx ** 2 + ky ** 2 + kz ** 2
    kmag = np.sqrt(ksq)
    zero = kmag < 1e-12
    ks = np.where(zero, 1.0, kmag)
    ksq_s = np.where(zero, 1.0, ksq)
    khat = np.stack(np.broadcast_arrays(kx / ks, ky / ks, kz / ks), axis=-1)
    khat[zero] = 0.0
    etaksq = ksq - (Gx[:, None, None] ** 2 * params.eta[0] + Gy[None, :, None] ** 2 * params.eta[1]
                    + Gz[None, None, :] ** 2 * params.eta[2])
    term = np.sin(ks) / ks - np.cos(ks)
    exp_part = np.exp(-etaksq / (4 * xi * xi))
    V = float(Nx * Ny * Nz)
    scale = 9.0 * term * term * exp_part / (ksq_s * ksq_s) / V
    scale[zero] = 0.0
    out = {"scale": scale, "khat": khat}
    if quads:
        j1 = term / ks
        j2 = (3.0 / ksq_s - 1.0) * np.sin(ks) / ks - 3.0 * np.cos(ks) / ksq_s
        expk2 = exp_part / ksq_s
        sQ = -22.5 * j1 * j2 * expk2 / V
        sGP = 45.0 * j1 * j2 * expk2 / V
        sGQ = 112.5 * j2 * j2 * expk2 / V
        for a in (sQ, sGP, sGQ):
            a[zero] = 0.0
        k0, k1, k2 = khat[..., 0], khat[..., 1], khat[..., 2]
        qf = np.stack([k0 * k0 - 1.0 / 3.0, k0 * k1, k0 * k2, k1 * k1 - 1.0 / 3.0, k1 * k2], axis=-1)
        qd = np.stack([k0 * k0 - k2 * k2, 2 * k0 * k1, 2 * k0 * k2, k1 * k1 - k2 * k2, 2 * k1 * k2], axis=-1)
        qf[zero] = 0.0
        qd[zero] = 0.0
        out.update(sQ=sQ, sGP=sGP, sGQ=sGQ, qf=qf, qd=qd)
    return out


def gaussian_stencil(params: MonoParams, pos, with_volume=False):
    """Per-point grid indices and weights (monodisperse_...cu:687-816).

    Returns (ix, iy, iz, w): index arrays of shape (n, P, P, P) (wrapped into
    the grid) and weights of the same shape.
    """
    pos = np.asarray(pos, dtype=np.float64)
    h = params.h
    xi = params.xi
    g = c_round(pos / h)  # (n,3)
    d = g * h - pos
    o = params.offsets
    const = (2.0 * xi * xi / PI) ** 1.5 * math.sqrt(1.0 / np.prod(params.eta))
    if with_volume:
        const *= float(np.prod(h))
    wx = np.exp(-2 * xi * xi * (d[:, 0:1] + o[None, :] * h[0]) ** 2 / params.eta[0])
    wy = np.exp(-2 * xi * xi * (d[:, 1:2] + o[None, :] * h[1]) ** 2 / params.eta[1])
    wz = np.exp(-2 * xi * xi * (d[:, 2:3] + o[None, :] * h[2]) ** 2 / params.eta[2])
    # the reference evaluates exp of the summed exponent; same value to rounding
    w = const * wx[:, :, None, None] * wy[:, None, :, None] * wz[:, None, None, :]
    N = params.num_grid
    ix = np.mod(g[:, 0:1] + o[None, :], N[0])[:, :, None, None]
    iy = np.mod(g[:, 1:2] + o[None, :], N[1])[:, None, :, None]
    iz = np.mod(g[:, 2:3] + o[None, :], N[2])[:, None, None, :]
    ix, iy, iz = np.broadcast_arrays(ix, iy, iz)
    return ix, iy, iz, w


# ---------------------------------------------------------------------------
# Neighbour pairs (neighbor_list.cu:186-223, minimum image)
# ---------------------------------------------------------------------------


def neighbor_pairs(src, tgt, box, rc, exclude_self):
    """All (source i, target j, r = x_i - x_j minimum image) with |r|^2 <= rc^2."""
    src = np.asarray(src, dtype=np.float64)
    tgt = np.asarray(tgt, dtype=np.float64)
    box = np.asarray(box, dtype=np.float64)
    I, J, R = [], [], []
    chunk = max(1, 2_000_000 // max(1, len(tgt)))
    for s in range(0, len(src), chunk):
        rr = src[s:s + chunk, None, :] - tgt[None, :, :]
        rr = rr - box * c_round(rr / box)
        d2 = np.sum(rr * rr, axis=-1)
        m = d2 <= rc * rc
        if exclude_self:
            ii = np.arange(s, min(s + chunk, len(src)))
            ok = ii < len(tgt)
            m[np.arange(len(ii))[ok], ii[ok]] = False
        a, b = np.nonzero(m)
        I.append(a + s)
        J.append(b)
        R.append(rr[a, b])
    if not I:
        return np.zeros(0, int), np.zeros(0, int), np.zeros((0, 3))
    return np.concatenate(I), np.concatenate(J), np.concatenate(R)


# ---------------------------------------------------------------------------
# Monodisperse Ewald operator
# ---------------------------------------------------------------------------


def _bloch_phase(bloch, r):
    """exp(i phase), phase = -(k_x r_x + k_y r_y) per pair (r = source -
    target, minimum image); None without a Bloch wavevector."""
    kx, ky = bloch
    if kx == 0.0 and ky == 0.0:
        return None
    ph = -(kx * r[:, 0] + ky * r[:, 1])
    return np.cos(ph) + 1j * np.sin(ph)


class MonoEwaldOperator:
    """Monodisperse spectral-Ewald field (SOLVER_AX or INTERACTION_FIELD).

    Moments layout follows the reference: ``[N*3 dipoles][Nq*5 quadrupoles]``
    (``base_electric_field.cu:235``).
    """

    def __init__(self, box, errortol, xi, solver_ax=True, quad_idxs=None, fft_workers=None, bloch=(0.0, 0.0)):
        self.fft_workers = fft_workers
        self.p = MonoParams(box, errortol, xi)
        self.solver_ax = solver_ax
        self.quad_idxs = None if quad_idxs is None else np.asarray(quad_idxs, dtype=int)
        self.r_table, self.tables, self.selfo, self.self_grad = mono_real_tables(xi)
        # Bloch wavevector (k_x, k_y): shifted k in the scale, a phase on
        # every pair term (monodisperse_ewald_electric_field.cu:1329-1330,
        # 1749-1756, 1778-1785, 1851-1858)
        self.bloch = (float(bloch[0]), float(bloch[1]))
        self.sc = mono_scale(self.p, quads=self.quad_idxs is not None, bloch=self.bloch)

    def set_positions(self, pos, field_points=None):
        self.pos = np.asarray(pos, dtype=np.float64)
        self.fp = self.pos if field_points is None else np.asarray(field_points, dtype=np.float64)
        N = len(self.pos)
        if self.quad_idxs is not None:
            qm = -np.ones(N, dtype=int)
            qm[self.quad_idxs] = np.arange(len(self.quad_idxs))
            self.quad_map = qm
        self.sp = gaussian_stencil(self.p, self.pos)
        self.ct = gaussian_stencil(self.p, self.fp, with_volume=True)
        i, j, r = neighbor_pairs(self.pos, self.fp, self.p.box, self.p.rc, self.solver_ax)
        d = np.sqrt(np.sum(r * r, axis=1))
        keep = d < self.p.rc
        self.pi_, self.pj, self.pr, self.pd = i[keep], j[keep], r[keep], d[keep]
        self.phase = _bloch_phase(self.bloch, self.pr)

    # -- stages --------------------------------------------------------------
    def _fftn(self, a):
        if self.fft_workers:
            import scipy.fft
            return scipy.fft.fftn(a, axes=(1, 2, 3), workers=self.fft_workers)
        return np.fft.fftn(a, axes=(1, 2, 3))

    def _ifftn(self, a):
        if self.fft_workers:
            import scipy.fft
            return scipy.fft.ifftn(a, axes=(1, 2, 3), workers=self.fft_workers)
        return np.fft.ifftn(a, axes=(1, 2, 3))

    def reciprocal(self, p, Q=None):
        Nx, Ny, Nz = self.p.num_grid
        ix, iy, iz, w = self.sp
        grid = np.zeros((3, Nx, Ny, Nz), dtype=np.complex128)
        for c in range(3):
            np.add.at(grid[c], (ix, iy, iz), w * p[:, c][:, None, None, None])
        F = self._fftn(grid)
        kh = self.sc["khat"]
        dot = F[0] * kh[..., 0] + F[1] * kh[..., 1] + F[2] * kh[..., 2]
        if Q is None:
            Edot = dot * self.sc["scale"]
        else:
            gq = np.zeros((5, Nx, Ny, Nz), dtype=np.complex128)
            qi = self.quad_idxs
            for c in range(5):
                np.add.at(gq[c], (ix[qi], iy[qi], iz[qi]), w[qi] * Q[:, c][:, None, None, None])
            FG = np.fft.fftn(gq, axes=(1, 2, 3))
            gdot = sum(FG[c] * self.sc["qd"][..., c] for c in range(5))
            Edot = dot * self.sc["scale"] + gdot * (1j * self.sc["sQ"])
            Gdot = dot * (1j * self.sc["sGP"]) + gdot * self.sc["sGQ"]
            FG = np.stack([Gdot * self.sc["qf"][..., c] for c in range(5)])
        F = np.stack([Edot * kh[..., c] for c in range(3)])
        Es = self._ifftn(F) * float(Nx * Ny * Nz)
        cx, cy, cz, cw = self.ct
        E = np.stack([np.sum(cw * Es[c][cx, cy, cz], axis=(1, 2, 3)) for c in range(3)], axis=1)
        G = None
        if Q is not None:
            Gs = np.fft.ifftn(FG, axes=(1, 2, 3)) * float(Nx * Ny * Nz)
            qi = self.quad_idxs
            Gp = np.stack([np.sum(cw * Gs[c][cx, cy, cz], axis=(1, 2, 3)) for c in range(5)], axis=1)
            G = Gp[qi]
        return E, G

    def real_space(self, p, Q=None, self_coef=None):
        """Pair sum plus (SOLVER_AX) self term, before any INTERACTION negation."""
        M = len(self.fp)
        E = np.zeros((M, 3), dtype=np.complex128)
        G = None if Q is None else np.zeros((len(self.quad_idxs), 5), dtype=np.complex128)
        sign = 1.0 if self.solver_ax else -1.0
        if self.solver_ax and self_coef is not None:
            E += (self_coef + self.selfo)[:, None] * p
            if Q is not None:
                sc = self_coef[self.quad_idxs]
                G += (2.5 * sc + 0.5 * self.self_grad)[:, None] * Q
        if len(self.pi_) == 0:
            return E, G
        deff = np.maximum(self.pd, 1.0)
        dl = self.pr / deff[:, None]
        perp = interp_table(deff, self.r_table, self.tables["fd1"])
        para = interp_table(deff, self.r_table, self.tables["fd2"])
        P = p[self.pi_]
        rP = np.sum(P * dl, axis=1)
        Ed = (P - rP[:, None] * dl) * perp[:, None] + (rP[:, None] * dl) * para[:, None]
        if Q is not None:
            qm = self.quad_map
            qs = qm[self.pi_]
            has = qs >= 0
            Qs = np.zeros((len(self.pi_), 5), dtype=np.complex128)
            Qs[has] = Q[qs[has]]
            dx, dy, dz = dl[:, 0], dl[:, 1], dl[:, 2]
            q0, q1, q2, q3, q4 = (Qs[:, c] for c in range(5))
            Qr = np.stack([q0 * dx + q1 * dy + q2 * dz,
                           q1 * dx + q3 * dy + q4 * dz,
                           q2 * dx + q4 * dy - (q0 + q3) * dz], axis=1)
            rr_ = np.stack([dx * dx - dz * dz, 2 * dx * dy, 2 * dx * dz, dy * dy - dz * dz, 2 * dy * dz], axis=1)
            Qrr = np.sum(Qs * rr_, axis=1)
            Q1 = interp_table(deff, self.r_table, self.tables["fq1"])
            Q2 = interp_table(deff, self.r_table, self.tables["fq2"])
            Q3 = interp_table(deff, self.r_table, self.tables["fq3"])
            Eq = 0.5 * (Qrr[:, None] * (Q1[:, None] * dl) + Qr * (2.0 * Q2[:, None]))
            Eq[~has] = 0.0
            Ed = Ed - Eq
            if self.phase is not None:
                Ed = Ed * self.phase[:, None]
            # contributions to G of quadrupole targets
            tq = qm[self.pj] if self.pj.max(initial=-1) < len(qm) else -np.ones_like(self.pj)
            tgt = tq >= 0
            if np.any(tgt):
                rs = np.stack([dx * dx, dx * dy, dx * dz, dy * dy, dy * dz], axis=1)
                I5 = np.array([1.0, 0.0, 0.0, 1.0, 0.0])
                px, py, pz = P[:, 0], P[:, 1], P[:, 2]
                Pr = np.stack([2 * px * dx, px * dy + py * dx, px * dz + pz * dx, 2 * py * dy,
                               py * dz + pz * dy], axis=1)
                Gd = rP[:, None] * (Q1[:, None] * rs + (Q2 + Q3)[:, None] * I5[None, :]) + Pr * Q2[:, None]
                G1 = interp_table(deff, self.r_table, self.tables["gq1"])
                G2 = interp_table(deff, self.r_table, self.tables["gq2"])
                G3 = interp_table(deff, self.r_table, self.tables["gq3"])
                G4 = interp_table(deff, self.r_table, self.tables["gq4"])
                Qrr2 = np.sum(Qr * dl, axis=1)
                QrrQ = np.stack([Qr[:, 0] * 2 * dx, Qr[:, 0] * dy + Qr[:, 1] * dx, Qr[:, 0] * dz + Qr[:, 2] * dx,
                                 Qr[:, 1] * 2 * dy, Qr[:, 1] * dz + Qr[:, 2] * dy], axis=1)
                Gq = 0.5 * (Qrr2[:, None] * ((G1 + G3)[:, None] * I5[None, :] + G4[:, None] * rs)
                            + Qs * G2[:, None] + QrrQ * (2.0 * G3[:, None]))
                Gq[~has] = 0.0
                Gt = (Gd + Gq) * sign
                if self.phase is not None:
                    Gt = Gt * self.phase[:, None]
                np.add.at(G, tq[tgt], Gt[tgt])
        elif self.phase is not None:
            Ed = Ed * self.phase[:, None]
        np.add.at(E, self.pj, Ed * sign)
        return E, G

    def apply(self, moments, self_coef=None, split=False):
        """Full field for flat moments ``[N*3 (+ Nq*5)]``; returns flat E."""
        N = len(self.pos)
        moments = np.asarray(moments, dtype=np.complex128)
        p = moments[:3 * N].reshape(N, 3)
        Q = None
        if self.quad_idxs is not None:
            Q = moments[3 * N:].reshape(len(self.quad_idxs), 5)
        Er, Gr = self.reciprocal(p, Q)
        Es, Gs = self.real_space(p, Q, self_coef)
        E = Er + Es
        G = None if Q is None else Gr + Gs
        if not self.solver_ax:
            E = -E
            G = None if G is None else -G
        out = E.ravel() if G is None else np.concatenate([E.ravel(), G.ravel()])
        if split:
            return out, (Er, Es, Gr, Gs)
        return out


# ---------------------------------------------------------------------------
# Polydisperse spectral-Ewald operator (polydisperse_ewald_electric_field.cu)
# ---------------------------------------------------------------------------


def poly_unique_radii(radii, tol=1e-5):
    """Radius classes (polydisperse_ewald_electric_field.cu:39-84).

    A radius joins the first class whose value is within ``tol``; the class
    values are then sorted and every particle is mapped to the first sorted
    class within ``tol``.
    """
    uniq = []
    for r in radii:
        if not any(abs(u - r) < tol for u in uniq):
            uniq.append(float(r))
    uniq.sort()
    ridx = np.array([next(k for k, u in enumerate(uniq) if abs(u - r) < tol) for r in radii], dtype=np.int64)
    return np.array(uniq), ridx


class PolyParams:
    """Grid, support and splitting (polydisperse_ewald_electric_field.cu:2039-2112)."""

    def __init__(self, box, errortol, xi, radii):
        box = np.asarray(box, dtype=np.float64)
        self.box = box
        self.errortol = float(errortol)
        self.xi = float(xi)
        self.unique, self.ridx = poly_unique_radii(list(map(float, radii)))
        rc = math.sqrt(-math.log(errortol)) / xi
        rc_min = 2.0 * self.unique[-1]
        if rc < rc_min:
            rc = rc_min
        if rc > box[0] / 2.0 or rc > box[1] / 2.0 or rc > box[2] / 2.0:
            raise RuntimeError("Real space cutoff (%f) larger than half the box length." % rc)
        self.rc = rc
        kcut = 2.0 * xi * xi * rc
        self.num_grid = np.array([int(math.ceil(1.0 + b * kcut / PI)) for b in box])
        self.h = box / self.num_grid
        mean_h = (self.h[0] + self.h[1] + self.h[2]) / 3.0
        self.P = int(math.ceil(2.0 / mean_h - 2.0 * math.log(errortol) / PI))
        self.eta = self.P * (mean_h * xi) ** 2 / PI
        off_min = -int(math.floor((self.P - 1) / 2.0))
        self.offsets = np.arange(off_min, off_min + self.P)
        # table nodes (computeRealSpaceTables, :1629-1645): r=0 then 1 + k*0.001
        rc_val = max(rc, 1.001)
        nsteps = int(math.ceil((rc_val - 1.0) / 0.001))
        self.r_table = np.concatenate([[0.0], 1.0 + np.arange(nsteps) * 0.001])


def poly_pair_functions(r, ai, aj, xi):
    """Perpendicular/parallel real-space pair functions of two radii and the
    self value (helper_compute_pair_tables,
    polydisperse_ewald_electric_field.cu:1434-1627), term by term."""
    r = np.asarray(r, dtype=np.float64)
    a, b, x = float(ai), float(aj), float(xi)
    x2, x3 = x * x, x ** 3
    x4, x5, x6 = x2 * x2, x ** 5, x ** 6
    r2, r3 = r * r, r ** 3
    r4, r5, r6 = r2 * r2, r ** 5, r ** 6
    a3, b3 = a ** 3, b ** 3
    p15 = PI ** 1.5
    k5 = 1.0 / (1024.0 * p15 * a3 * b3 * r3 * x5)
    k6 = 1.0 / (2048.0 * PI * a3 * b3 * r3 * x6)
    s, t = a + b, a - b
    cA = 4 * a3 - 3 * a * a * b - 3 * a * b * b + 4 * b3      # 4a^3-3a^2b-3ab^2+4b^3
    cB = 4 * a3 + 3 * a * a * b - 3 * a * b * b - 4 * b3      # 4a^3+3a^2b-3ab^2-4b^3
    qm = a * a - 4 * a * b + b * b
    qp = a * a + 4 * a * b + b * b
    f1 = k5 * (4 * r5 * x4 - 4 * s * r4 * x4 + r3 * (16 * x2 + 8 * (-4 * a * a + a * b - 4 * b * b) * x4)
               + r2 * (-12 * s * x2 - 8 * cA * x4) + r * (3 - 12 * (a * a - a * b + b * b) * x2 - 4 * s ** 2 * qm * x4)
               + 3 * s + 4 * cA * x2 + 4 * s ** 3 * qm * x4)
    f2 = k5 * (4 * r5 * x4 + 4 * s * r4 * x4 + r3 * (16 * x2 + 8 * (-4 * a * a + a * b - 4 * b * b) * x4)
               + r2 * (12 * s * x2 + 8 * cA * x4) + r * (3 - 12 * (a * a - a * b + b * b) * x2 - 4 * s ** 2 * qm * x4)
               - 3 * s - 4 * cA * x2 - 4 * s ** 3 * qm * x4)
    f3 = k5 * (-4 * r5 * x4 + 4 * (-a + b) * r4 * x4 + r3 * (-16 * x2 + 8 * (4 * a * a + a * b + 4 * b * b) * x4)
               + r2 * (12 * (-a + b) * x2 - 8 * cB * x4) + r * (-3 + 12 * (a * a + a * b + b * b) * x2 + 4 * t ** 2 * qp * x4)
               + 3 * t + 4 * cB * x2 + 4 * t ** 3 * qp * x4)
    f4 = k5 * (-4 * r5 * x4 + 4 * t * r4 * x4 + r3 * (-16 * x2 + 8 * (4 * a * a + a * b + 4 * b * b) * x4)
               + r2 * (12 * t * x2 + 8 * cB * x4) + r * (-3 + 12 * (a * a + a * b + b * b) * x2 + 4 * t ** 2 * qp * x4)
               + 3 * (-a + b) - 4 * cB * x2 - 4 * t ** 3 * qp * x4)
    sq2 = a * a + b * b
    dq2 = (a * a - b * b) ** 2
    f5 = k6 * (-8 * r6 * x6 + 36 * r4 * x4 * (-1 + 2 * sq2 * x2) + 128 * (a3 + b3) * r3 * x6
               + r2 * (-18 * x2 + 72 * sq2 * x4 + 72 * dq2 * x6) + 3 - 18 * sq2 * x2 - 36 * dq2 * x4 - 8 * s ** 4 * qm * x6)
    f6 = k6 * (-8 * r6 * x6 + 36 * r4 * x4 * (-1 + 2 * sq2 * x2) - 128 * (a3 + b3) * r3 * x6
               + r2 * (-18 * x2 + 72 * sq2 * x4 + 72 * dq2 * x6) + 3 - 18 * sq2 * x2 - 36 * dq2 * x4 - 8 * s ** 4 * qm * x6)
    f7 = k6 * (8 * r6 * x6 + 36 * r4 * x4 * (1 - 2 * sq2 * x2) + 128 * (a3 - b3) * r3 * x6
               + r2 * (18 * x2 - 72 * sq2 * x4 - 72 * dq2 * x6) - 3 + 18 * sq2 * x2 + 36 * dq2 * x4 + 8 * t ** 4 * qp * x6)
    f8 = k6 * (8 * r6 * x6 + 36 * r4 * x4 * (1 - 2 * sq2 * x2) - 128 * (a3 - b3) * r3 * x6
               + r2 * (18 * x2 - 72 * sq2 * x4 - 72 * dq2 * x6) - 3 + 18 * sq2 * x2 + 36 * dq2 * x4 + 8 * t ** 4 * qp * x6)
    ov = (r < s) & (r >= abs(t))
    reg1 = np.where(ov, (s - r) ** 3 / (128 * PI * a3 * b3 * r3)
                    * (-r3 - 3 * s * r2 + 3 * qm * r + a3 - 3 * a * a * b - 3 * a * b * b + b3),
                    np.where(r < b - a, (r3 - b3) / (4 * PI * b3 * r3),
                             np.where(r < a - b, (r3 - a3) / (4 * PI * a3 * r3), 0.0)))
    ep, em = np.exp(-(r + s) ** 2 * x2), np.exp(-(r - s) ** 2 * x2)
    e3, e4 = np.exp(-(r - a + b) ** 2 * x2), np.exp(-(r + a - b) ** 2 * x2)
    cp, cm = erfc((r + s) * x), erfc((r - s) * x)
    c3, c4 = erfc((r - a + b) * x), erfc((r + a - b) * x)
    fd1 = f1 * ep + f2 * em + f3 * e3 + f4 * e4 + f5 * cp + f6 * cm + f7 * c3 + f8 * c4 + reg1

    j5 = 1.0 / (512.0 * p15 * a3 * b3 * r3 * x5)
    j6 = 1.0 / (1024.0 * PI * a3 * b3 * r3 * x6)
    cC = a3 - 3 * a * a * b - 3 * a * b * b + b3                # a^3-3a^2b-3ab^2+b^3
    cD = a3 + 3 * a * a * b - 3 * a * b * b - b3                # a^3+3a^2b-3ab^2-b^3
    g1 = j5 * (8 * r5 * x4 - 8 * s * r4 * x4 + r3 * (14 * x2 - 4 * (7 * a * a - 4 * a * b + 7 * b * b) * x4)
               + r2 * (-6 * s * x2 - 4 * cC * x4) + r * (-3 + 12 * (a * a - a * b + b * b) * x2 + 4 * s ** 2 * qm * x4)
               - 3 * s - 4 * cA * x2 - 4 * s ** 3 * qm * x4)
    g2 = j5 * (8 * r5 * x4 + 8 * s * r4 * x4 + r3 * (14 * x2 - 4 * (7 * a * a - 4 * a * b + 7 * b * b) * x4)
               + r2 * (6 * s * x2 + 4 * cC * x4) + r * (-3 + 12 * (a * a - a * b + b * b) * x2 + 4 * s ** 2 * qm * x4)
               + 3 * s + 4 * cA * x2 + 4 * s ** 3 * qm * x4)
    g3 = j5 * (-8 * r5 * x4 + 8 * (-a + b) * r4 * x4 + r3 * (-14 * x2 + 4 * (7 * a * a + 4 * a * b + 7 * b * b) * x4)
               + r2 * (6 * (-a + b) * x2 - 4 * cD * x4) + r * (3 - 12 * (a * a + a * b + b * b) * x2 - 4 * t ** 2 * qp * x4)
               + 3 * (-a + b) - 4 * cB * x2 - 4 * t ** 3 * qp * x4)
    # the reference's fourth term carries +4 (a-b)^2 (...) xi^4 in its r^1
    # coefficient where the symmetry of the other terms gives -4
    g4 = j5 * (-8 * r5 * x4 + 8 * t * r4 * x4 + r3 * (-14 * x2 + 4 * (7 * a * a + 4 * a * b + 7 * b * b) * x4)
               + r2 * (6 * t * x2 + 4 * cD * x4) + r * (3 - 12 * (a * a + a * b + b * b) * x2 + 4 * t ** 2 * qp * x4)
               + 3 * t + 4 * cB * x2 + 4 * t ** 3 * qp * x4)
    g5 = j6 * (-16 * r6 * x6 + 36 * r4 * x4 * (-1 + 2 * sq2 * x2) + 64 * (a3 + b3) * r3 * x6
               - 3 + 18 * sq2 * x2 + 36 * dq2 * x4 + 8 * s ** 4 * qm * x6)
    g6 = j6 * (-16 * r6 * x6 + 36 * r4 * x4 * (-1 + 2 * sq2 * x2) - 64 * (a3 + b3) * r3 * x6
               - 3 + 18 * sq2 * x2 + 36 * dq2 * x4 + 8 * s ** 4 * qm * x6)
    g7 = j6 * (16 * r6 * x6 + 36 * r4 * x4 * (1 - 2 * sq2 * x2) + 64 * (a3 - b3) * r3 * x6
               + 3 - 18 * sq2 * x2 - 36 * dq2 * x4 - 8 * t ** 4 * qp * x6)
    g8 = j6 * (16 * r6 * x6 + 36 * r4 * x4 * (1 - 2 * sq2 * x2) + 64 * (-a3 + b3) * r3 * x6
               + 3 - 18 * sq2 * x2 - 36 * dq2 * x4 - 8 * t ** 4 * qp * x6)
    reg2 = np.where(ov, -1.0 / (64 * PI * a3 * b3 * r3) * (s ** 4 * qm - 8 * (a3 + b3) * r3 + 9 * sq2 * r4 - 2 * r6),
                    np.where(r < b - a, (r3 + 2 * b3) / (4 * PI * b3 * r3),
                             np.where(r < a - b, (r3 + 2 * a3) / (4 * PI * a3 * r3), 0.0)))
    fd2 = g1 * ep + g2 * em + g3 * e3 + g4 * e4 + g5 * cp + g6 * cm + g7 * c3 + g8 * c4 + reg2

    from scipy.special import erf
    selfv = (1.0 / (16 * p15 * a3 * b3 * x3)
             * ((1 - 2 * a * a * x2 + 2 * a * b * x2 - 2 * b * b * x2) * math.exp(-s * s * x2)
                + (-1 + 2 * a * a * x2 + 2 * a * b * x2 + 2 * b * b * x2) * math.exp(-t * t * x2))
             + 1.0 / (8 * PI * a3 * b3) * ((a3 - b3) * erf(t * x) - (a3 + b3) * erf(s * x))
             + min(a3, b3) / (4 * PI * a3 * b3))
    return fd1, fd2, float(selfv)


def poly_table_lookup(d, ai, aj, xi, r_table):
    """Linear interpolation in the (ai, aj) pair table at distance d
    (interpolate_table_gpu_polydisperse, :170-187), evaluating only the two
    table nodes the lookup reads.  Returns (perp, para)."""
    d = np.atleast_1d(np.asarray(d, dtype=np.float64))
    n = len(r_table)
    idx = np.where(d < 1.0, 0, 1 + ((d - 1.0) / TABLE_DR).astype(np.int64))
    idx = np.clip(idx, 0, n - 2)
    out = []
    fd1s, fd2s, selfv = poly_pair_functions(np.array([1.0]), ai, aj, xi)
    for which in (0, 1):
        y0 = np.empty_like(d)
        y1 = np.empty_like(d)
        lo_nodes = r_table[idx]
        hi_nodes = r_table[idx + 1]
        v_lo = np.where(idx == 0, selfv, poly_pair_functions(np.where(idx == 0, 1.0, lo_nodes), ai, aj, xi)[which])
        v_hi = poly_pair_functions(hi_nodes, ai, aj, xi)[which]
        last = poly_pair_functions(np.array([r_table[-1]]), ai, aj, xi)[which][0]
        y0[:] = v_lo
        y1[:] = v_hi
        val = np.empty_like(d)
        lo = d <= 0.0
        hi = (~lo) & (d >= r_table[-1])
        sub = (~lo) & (~hi) & (d < 1.0)
        mid = (~lo) & (~hi) & (~sub)
        val[lo] = selfv
        val[hi] = last
        val[sub] = selfv * (1.0 - d[sub]) + y1[sub] * d[sub]
        k = 1 + ((d[mid] - 1.0) / TABLE_DR).astype(np.int64)
        over = k >= n - 1
        t = (d[mid] - r_table[np.minimum(k, n - 2)]) / (r_table[np.minimum(k, n - 2) + 1] - r_table[np.minimum(k, n - 2)])
        vm = y0[mid] * (1.0 - t) + y1[mid] * t
        val[mid] = np.where(over, last, vm)
        out.append(val)
    return out[0], out[1]


def poly_weights(params: PolyParams, pos, radius):
    """Per-point grid indices and 3-vector weights of the smoothed-sphere
    spreading (spread_precalcs_kernel_polydisperse, :189-263; the contraction
    uses the same weights, :265-350).  Returns (idx (n,P^3) flat voxel index,
    w (n,P^3,3))."""
    pos = np.asarray(pos, dtype=np.float64)
    radius = np.asarray(radius, dtype=np.float64)
    h, xi, eta = params.h, params.xi, params.eta
    N = params.num_grid
    g = c_round(pos / h)
    d0 = g * h - pos
    o = params.offsets
    ox, oy, oz = np.meshgrid(o, o, o, indexing="ij")
    off = np.stack([ox.ravel(), oy.ravel(), oz.ravel()], axis=1)      # (P^3, 3), x slowest
    gd = d0[:, None, :] + off[None, :, :] * h[None, None, :]
    dist = np.sqrt(np.sum(gd * gd, axis=-1))
    a = radius[:, None]
    x2 = xi * xi
    with np.errstate(divide="ignore", invalid="ignore"):
        k = 3.0 / (8.0 * math.sqrt(2.0) * PI ** 1.5 * a ** 3.0 * math.sqrt(eta) * xi * dist * dist)
        tp = (eta + 4.0 * a * x2 * dist) * np.exp(-2.0 * (dist + a) ** 2 * x2 / eta)
        tm = (eta - 4.0 * a * x2 * dist) * np.exp(-2.0 * (dist - a) ** 2 * x2 / eta)
        cs = k * (tp - tm)
        wfar = cs[..., None] * (gd / dist[..., None])
    kn = 8.0 * math.sqrt(2.0) * xi ** 5 * np.exp(-2.0 * a * x2 / eta) / (PI ** 1.5 * eta ** 2.5)
    wnear = kn[..., None] * gd
    w = np.where((dist >= 1e-6)[..., None], wfar, wnear)
    gi = np.mod(g[:, None, :] + off[None, :, :], N[None, None, :])
    idx = (gi[..., 0] * N[1] + gi[..., 1]) * N[2] + gi[..., 2]
    return idx, w


def poly_scale(params: PolyParams, bloch=(0.0, 0.0)):
    """exp(-(1-eta) k^2 / 4 xi^2) / (k^2 V), 0 at k=0 (:565-638)."""
    Nx, Ny, Nz = params.num_grid
    L = params.box
    kx = (_freqs(Nx) * 2 * PI / L[0] - bloch[0])[:, None, None]
    ky = (_freqs(Ny) * 2 * PI / L[1] - bloch[1])[None, :, None]
    kz = (_freqs(Nz) * 2 * PI / L[2])[None, None, :]
    ksq = kx * kx + ky * ky + kz * kz
    zero = ksq < 1e-12
    ks = np.where(zero, 1.0, ksq)
    sc = np.exp(-(1.0 - params.eta) * ks / (4.0 * params.xi * params.xi)) / ks * (1.0 / float(Nx * Ny * Nz))
    return np.where(zero, 0.0, sc)


def poly_point_weights(params: PolyParams, pos):
    """Point-Gaussian weights of the quadrupole grid, (2 xi^2/pi)^1.5 h^3
    exp(-2 xi^2 |g|^2) on the same stencil and voxel indices as
    :func:`poly_weights` (spread_precalcs_kernel_point, :828-874, and
    contract_precalcs_kernel_point, :876-922; the constant from :2145 and
    :2227).  Returns (idx (n,P^3), w (n,P^3))."""
    pos = np.asarray(pos, dtype=np.float64)
    h, xi, N = params.h, params.xi, params.num_grid
    g = c_round(pos / h)
    d0 = g * h - pos
    o = params.offsets
    ox, oy, oz = np.meshgrid(o, o, o, indexing="ij")
    off = np.stack([ox.ravel(), oy.ravel(), oz.ravel()], axis=1)
    gd = d0[:, None, :] + off[None, :, :] * h[None, None, :]
    const = (2.0 * xi * xi / PI) ** 1.5 * float(np.prod(h))
    w = const * np.exp(-2.0 * xi * xi * np.sum(gd * gd, axis=-1))
    gi = np.mod(g[:, None, :] + off[None, :, :], N[None, None, :])
    idx = (gi[..., 0] * N[1] + gi[..., 1]) * N[2] + gi[..., 2]
    return idx, w


def poly_quad_scale(params: PolyParams, bloch=(0.0, 0.0)):
    """k-space factors of the quadrupole coupling on the scalar grid
    (compute_scale_coefficients_polydisperse_kernel, :565-638): with
    e = exp(-(1-eta) k^2 / 4 xi^2) / V, sQ = -e/2, sGP = e, sGQ = -e k^2 / 2,
    the traceless projector qf and its dot form qd, all 0 at k=0."""
    Nx, Ny, Nz = params.num_grid
    L = params.box
    kx = (_freqs(Nx) * 2 * PI / L[0] - bloch[0])[:, None, None]
    ky = (_freqs(Ny) * 2 * PI / L[1] - bloch[1])[None, :, None]
    kz = (_freqs(Nz) * 2 * PI / L[2])[None, None, :]
    kx, ky, kz = np.broadcast_arrays(kx, ky, kz)
    ksq = kx * kx + ky * ky + kz * kz
    zero = ksq < 1e-12
    ks = np.where(zero, 1.0, ksq)
    e = np.exp(-(1.0 - params.eta) * ks / (4.0 * params.xi * params.xi)) / float(Nx * Ny * Nz)
    km = np.sqrt(ks)
    k0, k1, k2 = kx / km, ky / km, kz / km
    qf = np.stack([k0 * k0 - 1.0 / 3.0, k0 * k1, k0 * k2, k1 * k1 - 1.0 / 3.0, k1 * k2])
    qd = np.stack([k0 * k0 - k2 * k2, 2 * k0 * k1, 2 * k0 * k2, k1 * k1 - k2 * k2, 2 * k1 * k2])
    out = {"sQ": -0.5 * e, "sGP": e, "sGQ": -0.5 * e * ks, "qf": qf, "qd": qd}
    for a in out.values():
        a[..., zero] = 0.0
    return out


def poly_self_grad(a, xi):
    """Quadrupole self value of radius ``a`` (computeRealSpaceTables,
    :1690-1706): the radius-1 gradient self value at xi*a, over a^5."""
    xa = xi * a
    x2, x4, x5 = xa * xa, xa ** 4, xa ** 5
    v = 0.5 / PI * (3.0 * (3.0 - 10.0 * x2 + 20.0 * x4) / (8.0 * math.sqrt(PI) * x5)
                    - 3.0 * (3.0 + 2.0 * x2 + 4.0 * x4) * math.exp(-4.0 * x2) / (8.0 * math.sqrt(PI) * x5)
                    + 3.0 * math.erfc(2.0 * xa))
    return v / a ** 5


class PolyEwaldOperator:
    """Polydisperse spectral-Ewald field (SOLVER_AX or INTERACTION_FIELD),
    polydisperse_ewald_electric_field.cu: scalar grid, spread :443-562, scale
    :640-651, contract :653-693, real space :695-826, stage order and
    INTERACTION sign :2553-2730.

    With ``quad_idxs`` the quadrupoles ride along as the reference has them:
    five point-Gaussian component grids (:964-1087), the joint k-space scale
    coupling them with the dipole grid (:925-962), a G contraction at every
    field point copied out at the quadrupole particles (:1090-1146), and the
    joint self and pair terms (:1148-1428) with radius-1 quadrupole tables.
    Quadrupole q is spread on the stencil of particle q (the spread kernel
    indexes the particle stencils by q, :994-1005), which is particle
    quad_idxs[q] only when every particle carries a quadrupole."""

    def __init__(self, box, errortol, xi, radii, solver_ax=True, quad_idxs=None, bloch=(0.0, 0.0)):
        self.p = PolyParams(box, errortol, xi, radii)
        self.radii = np.asarray(radii, dtype=np.float64)
        self.solver_ax = solver_ax
        # Bloch wavevector: shifted k in the scales, a phase on every pair
        # term (:592-593, 799-806, 1339-1346, 1414-1419)
        self.bloch = (float(bloch[0]), float(bloch[1]))
        self.scale = poly_scale(self.p, self.bloch)
        u = self.p.unique
        self.self_perp = np.array([poly_pair_functions(np.array([1.0]), a, a, xi)[2] for a in u])
        self.quad_idxs = None if quad_idxs is None else np.asarray(quad_idxs, dtype=np.int64)
        if self.quad_idxs is not None:
            N = len(self.radii)
            self.quad_map = -np.ones(N, dtype=np.int64)
            for q, i in enumerate(self.quad_idxs):
                if 0 <= i < N:
                    self.quad_map[i] = q
            self.qsc = poly_quad_scale(self.p, self.bloch)
            _, tabs, _, sg = mono_real_tables(xi, self.p.r_table[1:], variant="poly")
            self.qtables = tabs
            self.self_G2 = np.array([poly_self_grad(a, xi) for a in u])

    def set_positions(self, pos, field_points=None):
        if self.quad_idxs is not None and field_points is not None:
            # the joint pair kernel writes quadrupole rows at an offset of
            # 3 x (particle count) into a field laid out by the field-point
            # count (:1265); only targets that are the particles are restated
            raise NotImplementedError("polydisperse quadrupoles are restated for targets at the particles only")
        self.pos = np.asarray(pos, dtype=np.float64)
        self.fp = self.pos if field_points is None else np.asarray(field_points, dtype=np.float64)
        N = len(self.pos)
        self.sp = poly_weights(self.p, self.pos, self.radii)
        # field points beyond the particles use the first particle's radius (:297)
        frad = np.array([self.radii[j] if j < N else self.radii[0] for j in range(len(self.fp))])
        self.ct = self.sp if field_points is None else poly_weights(self.p, self.fp, frad)
        if self.quad_idxs is not None:
            self.sq = poly_point_weights(self.p, self.pos)
            self.cq = self.sq if field_points is None else poly_point_weights(self.p, self.fp)
        i, j, r = neighbor_pairs(self.pos, self.fp, self.p.box, self.p.rc, self.solver_ax)
        d = np.sqrt(np.sum(r * r, axis=1))
        keep = d < self.p.rc
        self.pi_, self.pj, self.pr, self.pd = i[keep], j[keep], r[keep], d[keep]
        self.phase = _bloch_phase(self.bloch, self.pr)
        # per-pair table values (real_space_precalcs_kernel_polydisperse, :352-441)
        u, ridx = self.p.unique, self.p.ridx
        deff = np.maximum(self.pd, 1e-6)
        self.deff = deff
        ri = ridx[self.pi_]
        rj = np.where(self.pj < N, ridx[np.minimum(self.pj, N - 1)], 0)
        lo, hi = np.minimum(ri, rj), np.maximum(ri, rj)
        self.perp = np.zeros(len(deff))
        self.para = np.zeros(len(deff))
        for a_ in np.unique(lo):
            for b_ in np.unique(hi[lo == a_]):
                m = (lo == a_) & (hi == b_)
                pp, pa = poly_table_lookup(deff[m], u[a_], u[b_], self.p.xi, self.p.r_table)
                self.perp[m], self.para[m] = pp, pa
        if self.quad_idxs is not None:
            self.qpair = {k: interp_table(deff, self.p.r_table, v) for k, v in self.qtables.items()
                          if k in ("fq1", "fq2", "fq3", "gq1", "gq2", "gq3", "gq4")}

    def reciprocal(self, p, Q=None):
        """(E at the field points, G at the quadrupoles or None)."""
        Nx, Ny, Nz = self.p.num_grid
        V = Nx * Ny * Nz
        idx, w = self.sp
        vals = np.einsum("noc,nc->no", w, p)
        grid = np.zeros(V, dtype=np.complex128)
        np.add.at(grid, idx.ravel(), vals.ravel())
        F = np.fft.fftn(grid.reshape(Nx, Ny, Nz))
        cidx, cw = self.ct
        h3 = float(np.prod(self.p.h))
        if Q is None:
            Es = (np.fft.ifftn(F * self.scale) * float(V)).ravel()
            return h3 * np.einsum("noc,no->nc", cw, Es[cidx]), None
        Q = np.asarray(Q, dtype=np.complex128)
        sidx, sw = self.sq
        gq = np.zeros((5, V), dtype=np.complex128)
        for c in range(5):
            # quadrupole q on particle q's stencil (see the class docstring)
            np.add.at(gq[c], sidx[:len(Q)].ravel(), (sw[:len(Q)] * Q[:, c][:, None]).ravel())
        FG = np.fft.fftn(gq.reshape(5, Nx, Ny, Nz), axes=(1, 2, 3))
        k = self.qsc
        gdot = np.sum(FG * k["qd"], axis=0)
        Fs = F * self.scale + gdot * k["sQ"]
        Gd = -(F * k["sGP"]) - gdot * k["sGQ"]
        Es = (np.fft.ifftn(Fs) * float(V)).ravel()
        Gs = (np.fft.ifftn(Gd[None] * k["qf"], axes=(1, 2, 3)) * float(V)).reshape(5, V)
        E = h3 * np.einsum("noc,no->nc", cw, Es[cidx])
        qidx, qw = self.cq
        Gp = np.stack([np.sum(qw * Gs[c][qidx], axis=1) for c in range(5)], axis=1)
        G = np.zeros((len(self.quad_idxs), 5), dtype=np.complex128)
        ok = (self.quad_idxs >= 0) & (self.quad_idxs < len(self.fp))
        G[ok] = Gp[self.quad_idxs[ok]]
        return E, G

    def real_space(self, p, Q=None, self_coef=None):
        """Pair sum (sign +1) plus, in SOLVER_AX, the self terms; returns
        (E, G or None)."""
        M = len(self.fp)
        E = np.zeros((M, 3), dtype=np.complex128)
        G = None if Q is None else np.zeros((len(self.quad_idxs), 5), dtype=np.complex128)
        if self.solver_ax and self_coef is not None:
            sc = np.asarray(self_coef)
            E += (sc + self.self_perp[self.p.ridx])[:, None] * p
            if Q is not None:
                for q, i in enumerate(self.quad_idxs):
                    a = self.radii[i]
                    f = 2.5 * sc[i] / (a * a) + 0.5 * self.self_G2[self.p.ridx[i]]
                    G[q] += f * Q[q]
        if len(self.pi_) == 0:
            return E, G
        dl = self.pr / self.deff[:, None]
        P = p[self.pi_]
        rP = np.sum(P * dl, axis=1)
        Ed = (P - rP[:, None] * dl) * self.perp[:, None] + (rP[:, None] * dl) * self.para[:, None]
        if Q is not None:
            t = self.qpair
            qs = self.quad_map[self.pi_]
            has = qs >= 0
            Qs = np.zeros((len(self.pi_), 5), dtype=np.complex128)
            Qs[has] = Q[qs[has]]
            dx, dy, dz = dl[:, 0], dl[:, 1], dl[:, 2]
            q0, q1, q2, q3, q4 = (Qs[:, c] for c in range(5))
            Qr = np.stack([q0 * dx + q1 * dy + q2 * dz,
                           q1 * dx + q3 * dy + q4 * dz,
                           q2 * dx + q4 * dy - (q0 + q3) * dz], axis=1)
            rr_ = np.stack([dx * dx - dz * dz, 2 * dx * dy, 2 * dx * dz, dy * dy - dz * dz, 2 * dy * dz], axis=1)
            Qrr = np.sum(Qs * rr_, axis=1)
            Eq = 0.5 * (Qrr[:, None] * (t["fq1"][:, None] * dl) + Qr * (2.0 * t["fq2"][:, None]))
            Eq[~has] = 0.0
            Ed = Ed - Eq
            N = len(self.pos)
            tq = np.where(self.pj < N, self.quad_map[np.minimum(self.pj, N - 1)], -1)
            tgt = tq >= 0
            if np.any(tgt):
                rs = np.stack([dx * dx, dx * dy, dx * dz, dy * dy, dy * dz], axis=1)
                I5 = np.array([1.0, 0.0, 0.0, 1.0, 0.0])
                px, py, pz = P[:, 0], P[:, 1], P[:, 2]
                Pr = np.stack([2 * px * dx, px * dy + py * dx, px * dz + pz * dx, 2 * py * dy,
                               py * dz + pz * dy], axis=1)
                Gd = (rP[:, None] * (t["fq1"][:, None] * rs + (t["fq2"] + t["fq3"])[:, None] * I5[None, :])
                      + Pr * t["fq2"][:, None])
                Qrr2 = np.sum(Qr * dl, axis=1)
                QrrQ = np.stack([Qr[:, 0] * 2 * dx, Qr[:, 0] * dy + Qr[:, 1] * dx, Qr[:, 0] * dz + Qr[:, 2] * dx,
                                 Qr[:, 1] * 2 * dy, Qr[:, 1] * dz + Qr[:, 2] * dy], axis=1)
                Gq = 0.5 * (Qrr2[:, None] * ((t["gq1"] + t["gq3"])[:, None] * I5[None, :] + t["gq4"][:, None] * rs)
                            + Qs * t["gq2"][:, None] + QrrQ * (2.0 * t["gq3"][:, None]))
                Gq[~has] = 0.0
                Gt = Gd + Gq
                if self.phase is not None:
                    Gt = Gt * self.phase[:, None]
                np.add.at(G, tq[tgt], Gt[tgt])
        if self.phase is not None:
            Ed = Ed * self.phase[:, None]
        np.add.at(E, self.pj, Ed)
        return E, G

    def apply(self, moments, self_coef=None, split=False):
        """Full field for flat moments ``[N*3 (+ Nq*5)]``; returns flat E
        (then G when quadrupoles are on)."""
        N = len(self.pos)
        moments = np.asarray(moments, dtype=np.complex128)
        p = moments[:3 * N].reshape(N, 3)
        Q = None
        if self.quad_idxs is not None:
            Q = moments[3 * N:3 * N + 5 * len(self.quad_idxs)].reshape(len(self.quad_idxs), 5)
        Er, Gr = self.reciprocal(p, Q)
        Es, Gs = self.real_space(p, Q, self_coef)
        # INTERACTION_FIELD: reciprocal part negated, pairs added with sign -1
        E = Er + Es if self.solver_ax else -(Er + Es)
        G = None
        if Q is not None:
            G = Gr + Gs if self.solver_ax else -(Gr + Gs)
        out = E.ravel() if G is None else np.concatenate([E.ravel(), G.ravel()])
        if split:
            return out, ((Er, Es) if G is None else (Er, Es, Gr, Gs))
        return out


# ---------------------------------------------------------------------------
# Direct (open boundary) operator (direct_electric_field.cu:42-324)
# ---------------------------------------------------------------------------


class DirectOperator:
    def __init__(self, radius, solver_ax=True, quad_idxs=None):
        self.radius = np.asarray(radius, dtype=np.float64)
        self.solver_ax = solver_ax
        self.quad_idxs = None if quad_idxs is None else np.asarray(quad_idxs, dtype=int)

    def set_positions(self, pos, field_points=None):
        self.pos = np.asarray(pos, dtype=np.float64)
        self.fp = self.pos if field_points is None else np.asarray(field_points, dtype=np.float64)
        N = len(self.pos)
        if self.quad_idxs is not None:
            qm = -np.ones(N, dtype=int)
            qm[self.quad_idxs] = np.arange(len(self.quad_idxs))
            self.quad_map = qm

    def apply(self, moments, self_coef=None):
        N = len(self.pos)
        M = len(self.fp)
        moments = np.asarray(moments, dtype=np.complex128)
        p = moments[:3 * N].reshape(N, 3)
        quads = self.quad_idxs is not None
        Qn = None
        if quads:
            Qn = moments[3 * N:].reshape(len(self.quad_idxs), 5)
        inv4pi = 1.0 / (4.0 * PI)
        k = inv4pi * (-1.0 if self.solver_ax else 1.0)
        E = np.zeros((M, 3), dtype=np.complex128)
        G = np.zeros((M, 5), dtype=np.complex128)
        for j in range(M):
            r = self.pos - self.fp[j][None, :]
            r2 = np.sum(r * r, axis=1)
            rs = self.radius.copy()
            mind2 = rs * rs
            ro = np.sqrt(r2)
            small = r2 < mind2
            scl = np.where(small & (ro > 1e-9), np.sqrt(mind2 / np.where(r2 > 0, r2, 1.0)), 1.0)
            r = r * scl[:, None]
            r2 = np.where(small, mind2, r2)
            valid = r2 >= 1e-18
            if self.solver_ax:
                valid &= np.arange(N) != j
            rr = np.sqrt(np.where(valid, r2, 1.0))
            u = r / rr[:, None]
            inv_r3 = 1.0 / rr ** 3
            pr = np.sum(p * u, axis=1)
            Ed = (pr[:, None] * 3 * u - p) * (k * inv_r3)[:, None]
            Ed[~valid] = 0
            E[j] += Ed.sum(0)
            if quads:
                qmap = self.quad_map
                qsrc = qmap
                Qs = np.zeros((N, 5), dtype=np.complex128)
                Qs[qsrc >= 0] = Qn[qsrc[qsrc >= 0]]
                q0, q1, q2, q3, q4 = (Qs[:, c] * f for c, f in enumerate([-1.0, -2.0, -2.0, -1.0, -2.0]))
                qzz = -(q0 + q3)
                ux, uy, uz = u[:, 0], u[:, 1], u[:, 2]
                Qx = q0 * ux + q1 * uy + q2 * uz
                Qy = q1 * ux + q3 * uy + q4 * uz
                Qz = q2 * ux + q4 * uy + qzz * uz
                Qrr = Qx * ux + Qy * uy + Qz * uz
                Eq = np.stack([Qrr * 2.5 * ux - Qx, Qrr * 2.5 * uy - Qy, Qrr * 2.5 * uz - Qz], axis=1)
                Eq *= (3.0 * k / rr ** 4)[:, None]
                Eq[~valid] = 0
                E[j] += Eq.sum(0)
                qt = qmap[j] if j < N else -1
                if qt >= 0:
                    px, py, pz = p[:, 0], p[:, 1], p[:, 2]
                    rs5 = [ux * ux, ux * uy, ux * uz, uy * uy, uy * uz]
                    Gd = [pr * (-5 * rs5[0] + 1) + px * 2 * ux,
                          pr * (-5 * rs5[1]) + (px * uy + py * ux),
                          pr * (-5 * rs5[2]) + (px * uz + pz * ux),
                          pr * (-5 * rs5[3] + 1) + py * 2 * uy,
                          pr * (-5 * rs5[4]) + (py * uz + pz * uy)]
                    gdf = -3.0 * k / rr ** 4
                    QQ = [Qx * 2 * ux, Qx * uy + Qy * ux, Qx * uz + Qz * ux, Qy * 2 * uy, Qy * uz + Qz * uy]
                    qp = [q0, q1, q2, q3, q4]
                    diag = [1, 0, 0, 1, 0]
                    f = -k / rr ** 5
                    for c in range(5):
                        Gq = qp[c] * -1.5 + Qrr * (52.5 * rs5[c] - 7.5 * diag[c]) - QQ[c] * 15.0
                        val = Gd[c] * gdf + Gq * f
                        val[~valid] = 0
                        G[j, c] += val.sum()
        if self.solver_ax and self_coef is not None:
            a = self.radius[:M]
            corr = inv4pi / a ** 3
            E += (self_coef + corr)[:, None] * p[:M]
            if quads:
                for j in range(M):
                    qt = self.quad_map[j]
                    if qt >= 0:
                        cq = 3.0 * corr[j] / a[j] ** 2
                        fsc = 2.5 / a[j] ** 2
                        G[j] += (fsc * self_coef[j] + cq) * Qn[qt]
        out = E.ravel()
        if quads:
            Gq = np.zeros((len(self.quad_idxs), 5), dtype=np.complex128)
            for j in range(min(M, N)):
                qt = self.quad_map[j]
                if qt >= 0:
                    Gq[qt] = G[j]
            out = np.concatenate([out, Gq.ravel()])
        return out


# ---------------------------------------------------------------------------
# Krylov solvers (gmres_solver.cu:56-208, bicgstab_solver.cu:58-192)
# ---------------------------------------------------------------------------


def jacobi_inverse(self_coef, N, quad_idxs=None):
    """diag(s)^-1 over the unknown layout (numerical_solver.cu:250-285)."""
    sc = np.asarray(self_coef, dtype=np.complex128)
    den = sc.real ** 2 + sc.imag ** 2
    inv = np.where(den > 1e-30, np.conj(sc) / np.where(den > 0, den, 1.0), 1.0 + 0j)
    d = np.repeat(inv, 3)
    if quad_idxs is not None and len(quad_idxs):
        d = np.concatenate([d, np.repeat(inv[np.asarray(quad_idxs)], 5)])
    return d


def gmres(A, b, x0, tol, M=None, restart=50, maxiter=1000):
    n = len(b)
    Mi = (lambda v: v) if M is None else (lambda v: M * v)
    bnorm = np.linalg.norm(b)
    if bnorm == 0.0:
        return np.zeros(n, dtype=np.complex128), 0
    m = min(n, restart)
    x = np.array(x0, dtype=np.complex128)
    it = 0
    while it < maxiter:
        r = Mi(b - A(x))
        rn = np.linalg.norm(r)
        if rn < tol * bnorm:
            break
        V = np.zeros((m + 1, n), dtype=np.complex128)
        H = np.zeros((m + 1, m), dtype=np.complex128)
        g = np.zeros(m + 1, dtype=np.complex128)
        cs = np.zeros(m)
        sn = np.zeros(m, dtype=np.complex128)
        g[0] = rn
        V[0] = r / rn
        k = 0
        while k < m and it < maxiter:
            w = Mi(A(V[k]))
            for i in range(k + 1):
                H[i, k] = np.vdot(V[i], w)
                w = w - H[i, k] * V[i]
            wn = np.linalg.norm(w)
            H[k + 1, k] = wn
            if wn > 0.0:
                V[k + 1] = w / wn
            for i in range(k):
                h1, h2 = H[i, k], H[i + 1, k]
                H[i, k] = cs[i] * h1 + np.conj(sn[i]) * h2
                H[i + 1, k] = -sn[i] * h1 + cs[i] * h2
            h1, h2 = H[k, k], H[k + 1, k]
            c, s = 1.0, 0.0 + 0j
            if h2 != 0.0:
                a1 = abs(h1)
                if a1 == 0.0:
                    c, s = 0.0, 1.0 + 0j
                else:
                    sv = a1 + abs(h2)
                    hh = sv * math.sqrt(abs(h1 / sv) ** 2 + abs(h2 / sv) ** 2)
                    c = a1 / hh
                    s = (np.conj(h1) / a1) * (h2 / hh)
            cs[k], sn[k] = c, s
            H[k, k] = c * h1 + np.conj(s) * h2
            H[k + 1, k] = 0.0
            g1, g2 = g[k], g[k + 1]
            g[k] = c * g1 + np.conj(s) * g2
            g[k + 1] = -s * g1 + c * g2
            k += 1
            it += 1
            if abs(g[k]) < tol * bnorm:
                break
        y = np.zeros(k, dtype=np.complex128)
        for i in range(k - 1, -1, -1):
            y[i] = (g[i] - np.dot(H[i, i + 1:k], y[i + 1:k])) / H[i, i]
        x = x + V[:k].T @ y
    return x, it


def bicgstab(A, b, x0, tol, M=None, maxiter=1000):
    Mi = (lambda v: v) if M is None else (lambda v: M * v)
    n = len(b)
    bnorm = np.linalg.norm(b)
    if bnorm == 0.0:
        return np.zeros(n, dtype=np.complex128), 0
    x = np.array(x0, dtype=np.complex128)
    r = Mi(b - A(x))
    if np.linalg.norm(r) < tol * bnorm:
        return x, 0
    r0 = r.copy()
    p = r.copy()
    rho = alpha = omega = 1.0 + 0j
    v = np.zeros(n, dtype=np.complex128)
    it = 0
    for it in range(maxiter):
        rho_new = np.sum(r0 * r)
        if abs(rho_new) < 1e-16:
            break
        if it > 0:
            beta = (rho_new / rho) * (alpha / omega)
            p = (p - omega * v) * beta + r
        rho = rho_new
        v = Mi(A(p))
        rv = np.sum(r0 * v)
        if abs(rv) < 1e-16:
            break
        alpha = rho / rv
        s = r - alpha * v
        if np.linalg.norm(s) < tol * bnorm:
            x = x + alpha * p
            break
        t = Mi(A(s))
        ts = np.vdot(t, s)
        tt = np.vdot(t, t)
        if abs(tt) < 1e-16:
            break
        omega = ts / tt.real
        x = x + alpha * p + omega * s
        r = s - omega * t
        if np.linalg.norm(r) < tol * bnorm:
            break
        if abs(omega) < 1e-16:
            break
    return x, it


# ---------------------------------------------------------------------------
# Driver (dipole_solver.cu:131-647)
# ---------------------------------------------------------------------------


class DipoleSolverOracle:
    """CPU restatement of ``Dipole_Solver`` (one frame loop per compute call)."""

    def __init__(self, box, eps_p, radius=(), eps_m=1.0, xi=0.5, tol=1e-3, guess_type="derivative",
                 solver_type="gmres", field_type="auto", E0=None, solve_quadrupoles=False, quad_idxs=(),
                 jacobi=True, solve_tol=None, matvec_hook=None):
        self.box = list(map(float, box))
        eps = np.asarray(eps_p, dtype=np.complex128)
        if eps.ndim == 0:
            eps = eps.reshape(1, 1)
        elif eps.ndim == 1:
            eps = eps[:, None]
        self.eps_p = eps
        self.radius = list(map(float, np.atleast_1d(radius))) if np.size(radius) else []
        self.eps_m = float(eps_m)
        self.xi = float(xi)
        self.tol = float(tol)
        self.solve_tol = self.tol if solve_tol is None else solve_tol
        self.guess_type = guess_type
        self.solver_type = solver_type
        self.field_type = field_type
        self.E0 = [np.asarray(e, dtype=np.complex128) for e in (E0 if E0 else np.eye(3))]
        self.solve_quadrupoles = bool(solve_quadrupoles)
        self.quad_idxs = list(quad_idxs)
        self.jacobi = jacobi
        self.num_particles = 0
        self.num_frames = 0
        self.avg_dips, self.dips, self.quads = [], [], []
        self.matvec_hook = matvec_hook
        self.iterations = []

    def _set_dims(self, n):
        self.num_particles = n
        self.num_quads = (n if not self.quad_idxs else len(self.quad_idxs)) if self.solve_quadrupoles else 0
        if not self.radius:
            self.radius = [1.0] * n
        elif len(self.radius) == 1:
            self.radius = self.radius * n
        elif len(self.radius) != n:
            raise RuntimeError("The number of particles is inconsistent with the number of radii provided.")
        mono = all(r == self.radius[0] for r in self.radius)
        if self.field_type == "monodisperse" and not mono:
            raise RuntimeError("field_type was set to 'monodisperse' but radii are not identical.")
        if self.eps_p.shape[1] == 1:
            self.eps_p = np.repeat(self.eps_p, n, axis=1)
        elif self.eps_p.shape[1] != n:
            raise RuntimeError("The number of particles is inconsistent with eps_p provided.")
        vs = 3 * n + 5 * self.num_quads
        for d, e in enumerate(self.E0):
            if e.size not in (3, 3 * n, vs):
                raise RuntimeError(f"Incident field E0[{d}] has size {e.size}, but expected 3, {3 * n}, or {vs}.")

    def _nondim(self):
        self.length_scale = min(self.radius)
        self.eps_scale = self.eps_m
        self.box = [b / self.length_scale for b in self.box]
        self.radius = [r / self.length_scale for r in self.radius]
        self.eps_p = self.eps_p / self.eps_scale
        s = sum(r ** 3 for r in self.radius)
        V = self.box[0] * self.box[1] * self.box[2]
        self.vol_frac = 0.0 if V == 0 else 4.0 / 3.0 * PI * s / V

    def _make_field(self):
        qi = None
        if self.solve_quadrupoles:
            qi = self.quad_idxs if self.quad_idxs else list(range(self.num_particles))
        self.qi = qi
        if self.field_type == "direct":
            return DirectOperator(self.radius, True, qi)
        mono = all(r == self.radius[0] for r in self.radius)
        if self.field_type == "polydisperse" or (self.field_type == "auto" and not mono):
            return PolyEwaldOperator(self.box, self.tol, self.xi, self.radius, True, qi)
        return MonoEwaldOperator(self.box, self.tol, self.xi, True, qi)

    def _mean_field(self, w):
        K = len(self.E0)
        N, Nq = self.num_particles, self.num_quads
        g = np.zeros(N * K * 3 + Nq * K * 5, dtype=np.complex128)
        for p in range(N):
            beta = (self.eps_p[w, p] - 1.0) / (self.eps_p[w, p] + 2.0)
            val = 4.0 * PI * self.radius[p] ** 3 * beta / (1.0 - beta * self.vol_frac)
            for d in range(K):
                e = self.E0[d]
                for c in range(3):
                    g[p * K * 3 + d * 3 + c] = val * (e[p * 3 + c] if e.size > 3 else e[c])
        return g

    def _guess(self, fd, fq, w):
        K = len(self.E0)
        N, Nq = self.num_particles, self.num_quads
        gt = self.guess_type
        if gt in ("mean_field", "mean-field") or (gt in ("previous", "derivative") and w < 1):
            return self._mean_field(w)
        if gt == "previous" or (gt == "derivative" and w < 2):
            g = np.zeros(N * K * 3 + Nq * K * 5, dtype=np.complex128)
            g[:N * K * 3] = fd[(w - 1) * N * K * 3:w * N * K * 3]
            if Nq:
                g[N * K * 3:] = fq[(w - 1) * Nq * K * 5:w * Nq * K * 5]
            return g
        if gt != "derivative":
            raise RuntimeError("Guess type " + gt + " not supported.")

        def X(e):
            return 0.0 if e - 1.0 == 0.0 else (e + 2.0) / (e - 1.0)

        g = np.zeros(N * K * 3 + Nq * K * 5, dtype=np.complex128)
        for p in range(N):
            run = X(self.eps_p[w - 1, p]) - X(self.eps_p[w - 2, p])
            new = X(self.eps_p[w, p]) - X(self.eps_p[w - 1, p])
            if abs(run) < 1e-12:
                run, new = 1.0, 0.0
            a1 = fd[(w - 1) * N * K * 3 + p * K * 3:(w - 1) * N * K * 3 + (p + 1) * K * 3]
            a2 = fd[(w - 2) * N * K * 3 + p * K * 3:(w - 2) * N * K * 3 + (p + 1) * K * 3]
            g[p * K * 3:(p + 1) * K * 3] = a1 + new * (a1 - a2) / run
        for q in range(Nq):
            p = q if not self.quad_idxs else self.quad_idxs[q]
            run = X(self.eps_p[w - 1, p]) - X(self.eps_p[w - 2, p])
            new = X(self.eps_p[w, p]) - X(self.eps_p[w - 1, p])
            if abs(run) < 1e-12:
                run, new = 1.0, 0.0
            a1 = fq[(w - 1) * Nq * K * 5 + q * K * 5:(w - 1) * Nq * K * 5 + (q + 1) * K * 5]
            a2 = fq[(w - 2) * Nq * K * 5 + q * K * 5:(w - 2) * Nq * K * 5 + (q + 1) * K * 5]
            g[N * K * 3 + q * K * 5:N * K * 3 + (q + 1) * K * 5] = a1 + new * (a1 - a2) / run
        return g

    def compute(self, positions):
        pos = np.asarray(positions, dtype=np.float64)
        n = len(pos)
        if n == 0:
            return
        if self.num_particles == 0:
            self._set_dims(n)
            self._nondim()
            self.EF = self._make_field()
        elif n != self.num_particles:
            raise RuntimeError("The number of particles has changed!")
        self.num_frames += 1
        self.EF.set_positions(pos / self.length_scale)
        K = len(self.E0)
        N, Nq = self.num_particles, self.num_quads
        W = self.eps_p.shape[0]
        if self.num_frames == 1:
            init = self._mean_field(0)
        else:
            prev = self.num_frames - 2
            init = np.zeros(N * K * 3 + Nq * K * 5, dtype=np.complex128)
            off = prev * W * N * K * 3
            init[:N * K * 3] = self.dips_flat()[off:off + N * K * 3]
            if Nq:
                qoff = prev * W * Nq * K * 5
                init[N * K * 3:] = np.concatenate(self.quads)[qoff:qoff + Nq * K * 5]
        fcap = np.zeros(W * K * 3, dtype=np.complex128)
        fd = np.zeros(W * N * K * 3, dtype=np.complex128)
        fq = np.zeros(W * Nq * K * 5, dtype=np.complex128)
        vs = 3 * N + 5 * Nq
        for w in range(W):
            diff = 1.0 - self.eps_p[w]
            diff = np.where(np.abs(diff) < 1e-12, 1e-12, diff)
            sc = -3.0 / (4.0 * PI * diff) / np.asarray(self.radius) ** 3
            guess = init if w == 0 else self._guess(fd, fq, w)
            Mj = jacobi_inverse(sc, N, self.qi) if self.jacobi else None

            def A(v, sc=sc):
                if self.matvec_hook is not None:
                    self.matvec_hook()
                return self.EF.apply(v, sc)

            for d in range(K):
                e = self.E0[d]
                b = np.zeros(vs, dtype=np.complex128)
                if e.size == 3 * N:
                    b[:3 * N] = e
                elif e.size == 3:
                    b[:3 * N] = np.tile(e, N)
                else:
                    b[:] = e
                x0 = np.zeros(vs, dtype=np.complex128)
                for p in range(N):
                    x0[p * 3:p * 3 + 3] = guess[p * K * 3 + d * 3:p * K * 3 + d * 3 + 3]
                for q in range(Nq):
                    x0[3 * N + q * 5:3 * N + q * 5 + 5] = guess[N * K * 3 + q * K * 5 + d * 5:N * K * 3 + q * K * 5 + d * 5 + 5]
                if self.solver_type == "bicgstab":
                    sol, it = bicgstab(A, b, x0, self.solve_tol, Mj)
                else:
                    sol, it = gmres(A, b, x0, self.solve_tol, Mj)
                self.iterations.append(it)
                for p in range(N):
                    fd[w * N * K * 3 + p * K * 3 + d * 3:w * N * K * 3 + p * K * 3 + d * 3 + 3] = sol[p * 3:p * 3 + 3]
                for q in range(Nq):
                    fq[w * Nq * K * 5 + q * K * 5 + d * 5:w * Nq * K * 5 + q * K * 5 + d * 5 + 5] = \
                        sol[3 * N + q * 5:3 * N + q * 5 + 5]
                fcap[w * K * 3 + d * 3:w * K * 3 + d * 3 + 3] = sol[:3 * N].reshape(N, 3).sum(0) / N
        self.avg_dips.append(fcap)
        self.dips.append(fd)
        if Nq:
            self.quads.append(fq)

    def dips_flat(self):
        return np.concatenate(self.dips)

    def get_eff_polarizability(self, physical=True):
        K = len(self.E0)
        W = self.eps_p.shape[0]
        f = self.eps_scale * self.length_scale ** 3 if physical else 1.0
        a = np.mean(np.stack(self.avg_dips), axis=0) * f
        return a.reshape(W, K, 3)

    def get_dipoles(self, physical=True):
        K = len(self.E0)
        W = self.eps_p.shape[0]
        f = self.eps_scale * self.length_scale ** 3 if physical else 1.0
        return (self.dips_flat() * f).reshape(self.num_frames, W, self.num_particles, K, 3)

    def get_quadrupoles(self, physical=True):
        K = len(self.E0)
        W = self.eps_p.shape[0]
        f = self.eps_scale * self.length_scale ** 4 if physical else 1.0
        if not self.quads:
            return np.zeros((self.num_frames, W, 0, K, 5), dtype=np.complex128)
        return (np.concatenate(self.quads) * f).reshape(self.num_frames, W, self.num_quads, K, 5)


def near_field_intensity(box, E0, radius, dip, dip_pos, field_points, xi=0.5, errortol=1e-3, field_type="auto"):
    """|E_point + E0|^2 at field points (near_field.cu:78-213)."""
    dip = np.asarray(dip, dtype=np.complex128).reshape(-1, 3)
    N = len(dip)
    rad = list(np.atleast_1d(radius).astype(float))
    if len(rad) == 1:
        rad = rad * N
    ls = rad[0]
    sbox = np.asarray(box, dtype=np.float64) / ls
    srad = np.asarray(rad) / ls
    pos = np.asarray(dip_pos, dtype=np.float64) / ls
    fp = np.asarray(field_points, dtype=np.float64) / ls
    mono = all(r == rad[0] for r in rad)
    if field_type == "direct":
        op = DirectOperator(srad, solver_ax=False)
    elif field_type == "polydisperse" or (field_type == "auto" and not mono):
        # polydisperse field on the radii scaled by the first one (:98-135)
        op = PolyEwaldOperator(sbox, errortol, xi, srad, solver_ax=False)
    else:
        op = MonoEwaldOperator(sbox, errortol, xi, solver_ax=False)
    op.set_positions(pos, fp)
    E = op.apply(dip.ravel(), np.zeros(N)).reshape(-1, 3)
    f = E + np.asarray(E0, dtype=np.complex128)[None, :]
    return np.sum(np.abs(f) ** 2, axis=1)
