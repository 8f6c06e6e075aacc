"""C ABI library: loads, exports what the header declares, host-only entry
points agree with the oracle.  No GPU needed."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import mpm_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "cumpm_b200.h")).read()
    return sorted(set(re.findall(r"MPM_API\s+[\w\s\*]*?\b(mpm_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from cumpm_b200 import capi

    L = capi.lib()
    names = header_symbols()
    assert len(names) >= 25
    assert sorted(capi.EXPORTS) == names
    for n in names:
        assert hasattr(L, n), n
        assert isinstance(getattr(L, n), ctypes._CFuncPtr)


def test_extension_module_surface():
    from cumpm_b200 import _cuMPM

    for name in ("Dipole_Solver", "Near_Field", "PrecisionMode", "FieldCalcMode"):
        assert hasattr(_cuMPM, name)
    assert _cuMPM.PrecisionMode.FP32 == _cuMPM.PrecisionMode.MIXED
    assert _cuMPM.PrecisionMode.FP64 == _cuMPM.PrecisionMode.DOUBLE
    for meth in ("compute", "get_eff_polarizability", "get_dipoles", "get_quadrupoles", "get_num_frames",
                 "get_num_particles", "get_num_quads", "get_num_wavevectors", "get_num_incident_polarizations",
                 "isUsingJacobiPrecond", "setUseJacobiPrecond"):
        assert hasattr(_cuMPM.Dipole_Solver, meth)


@pytest.mark.parametrize("xi", [0.3, 0.5, 0.8])
def test_cpp_tables_match_oracle(xi):
    from cumpm_b200 import capi

    r, T, so, sg = capi.mono_tables(xi)
    ro, To, soo, sgo = O.mono_real_tables(xi)
    np.testing.assert_array_equal(r, ro)
    for k in To:
        np.testing.assert_allclose(T[k], To[k], rtol=1e-9, atol=1e-12 * np.abs(To[k]).max())
    assert abs(so - soo) < 1e-15 and abs(sg - sgo) < 1e-14


@pytest.mark.parametrize("box,tol,xi", [((20, 20, 20), 1e-6, 0.5), ((308.4, 66.52, 200.0), 1e-6, 0.5),
                                        ((50, 60, 70), 1e-3, 0.5), ((100, 100, 100), 1e-8, 0.4),
                                        ((40, 40, 40), 1e-4, 0.45)])
def test_ewald_geometry_matches_oracle(box, tol, xi):
    from cumpm_b200 import capi

    g = capi.ewald_geometry(box, tol, xi)
    p = O.MonoParams(box, tol, xi)
    assert g["grid"] == list(p.num_grid)
    assert g["stencil"] == len(p.offsets)
    assert abs(g["rc"] - p.rc) < 1e-12
    np.testing.assert_allclose(g["h"], p.h, rtol=1e-15)
    np.testing.assert_allclose(g["eta"], p.eta, rtol=1e-14)


def test_host_errors_map_to_exceptions():
    from cumpm_b200 import capi

    with pytest.raises(RuntimeError, match="Real space cutoff .* larger than half the box length"):
        capi.ewald_geometry((10, 10, 10), 1e-6, 0.5)
    with pytest.raises(ValueError):
        capi.ewald_geometry((10, 10, 10), 0.0, 0.5)
    with pytest.raises(ValueError):
        capi.mono_tables(-1.0)
