"""Stand-alone on-disk result files (numpy ``.npz``).

Two formats:

* the extinction-spectrum file the reference's examples write
  (examples/mpm_hex_monolayer_sweep.py:131-135): keys ``wavenumber_cm``,
  ``energy_ev`` (wavenumber / 8065.54, the example's conversion),
  ``extinction_cs`` and ``extinction_cs_single``;
* a solution file: the physical dipoles, effective polarisability and (when
  solved) quadrupoles of a ``dipole_solver``, with the inputs that define
  the run (box, eps_p, radius, eps_m, xi, tol, E0, positions), so that a
  result can be reloaded and compared without the solver.

``extinction_cross_section`` is the example's C_ext = 4 pi k sum_i
Im(E0^* . p_i) (examples/mpm_hex_monolayer_sweep.py:116-118) for dipoles of
shape (N, 3) or (..., N, 3).
"""
from __future__ import annotations

import os
from typing import Dict, Optional

import numpy as np

__all__ = ["save_spectrum", "load_spectrum", "save_solution", "load_solution", "extinction_cross_section",
           "CM_PER_EV"]

CM_PER_EV = 8065.54   # wavenumber (cm^-1) per eV, as the reference's examples convert


def extinction_cross_section(dipoles, E0, k):
    """C_ext = 4 pi k sum_i Im(conj(E0_i) . p_i); dipoles (..., N, 3),
    E0 (3,) or (..., N, 3) broadcast against them, k the wavenumber."""
    p = np.asarray(dipoles)
    e = np.asarray(E0)
    proj = np.sum(np.conj(e) * p, axis=-1)
    return 4.0 * np.pi * np.asarray(k) * np.sum(np.imag(proj), axis=-1)


def save_spectrum(path, wavenumber_cm, extinction_cs, extinction_cs_single=None):
    """Write an extinction spectrum in the examples' file layout."""
    w = np.asarray(wavenumber_cm, dtype=np.float64)
    c = np.asarray(extinction_cs, dtype=np.float64)
    if c.shape != w.shape:
        raise ValueError(f"extinction_cs has shape {c.shape}, expected {w.shape} (one value per wavenumber)")
    single = np.full_like(w, np.nan) if extinction_cs_single is None else np.asarray(extinction_cs_single,
                                                                                    dtype=np.float64)
    if single.shape != w.shape:
        raise ValueError(f"extinction_cs_single has shape {single.shape}, expected {w.shape}")
    np.savez(path, wavenumber_cm=w, energy_ev=w / CM_PER_EV, extinction_cs=c, extinction_cs_single=single)


def load_spectrum(path) -> Dict[str, np.ndarray]:
    with np.load(path, allow_pickle=False) as z:
        missing = {"wavenumber_cm", "energy_ev", "extinction_cs", "extinction_cs_single"} - set(z.files)
        if missing:
            raise ValueError(f"{os.fspath(path)} is not a spectrum file (missing {sorted(missing)})")
        return {k: z[k] for k in z.files}


_SOLUTION_FORMAT = "cumpm_b200.solution/1"


def save_solution(path, solver, positions, *, box=None, eps_p=None, radius=None, eps_m=None, xi=None, tol=None,
                  E0=None, extra: Optional[Dict[str, np.ndarray]] = None):
    """Write a solved ``dipole_solver``'s physical results and the run's
    inputs.  The inputs default to what the solver was built with; the
    positions (N, 3) or frames (F, N, 3) are the caller's."""
    a = getattr(solver, "_args", {})
    out = {
        "format": np.array(_SOLUTION_FORMAT),
        "positions": np.asarray(positions, dtype=np.float64),
        "dipoles": np.asarray(solver.get_dipoles()),
        "eff_polarizability": np.asarray(solver.get_eff_polarizability()),
    }
    quads = None
    try:
        quads = solver.get_quadrupoles()
    except Exception:   # solved without quadrupoles
        quads = None
    if quads is not None and np.size(quads):
        out["quadrupoles"] = np.asarray(quads)
    for key, val in (("box", box), ("eps_p", eps_p), ("radius", radius), ("eps_m", eps_m), ("xi", xi), ("tol", tol),
                     ("E0", E0)):
        v = a.get(key) if val is None else val
        if v is not None:
            out[key] = np.asarray(v)
    for key, val in (extra or {}).items():
        if key in out:
            raise ValueError(f"extra key {key!r} collides with a result key")
        out[key] = np.asarray(val)
    np.savez(path, **out)


def load_solution(path) -> Dict[str, np.ndarray]:
    with np.load(path, allow_pickle=False) as z:
        if "format" not in z.files or str(z["format"]) != _SOLUTION_FORMAT:
            raise ValueError(f"{os.fspath(path)} is not a solution file")
        return {k: z[k] for k in z.files if k != "format"}
