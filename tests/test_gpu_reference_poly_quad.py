"""The oracle's polydisperse quadrupole field against the reference build
itself (oracle/_ref, the reference's Polydisperse_Ewald_Electric_Field with
quadrupoles, run on the GPU).  This pins the oracle's restatement of the
polydisperse quadrupole tables, the point-Gaussian grids, the joint scale and
the spread of quadrupole q on particle q's stencil; the device field is
compared with the same reference field directly (first run of that device
path: marked first_gpu_run).  Skipped when the
reference build is not present."""
import glob
import os
import sys

import numpy as np
import pytest

from oracle import mpm_oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.first_gpu_run]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


@pytest.fixture(scope="module")
def ref():
    if not glob.glob(os.path.join(REF_DIR, "_cuMPM*.so")):
        pytest.skip("reference build oracle/_ref not present")
    sys.path.insert(0, REF_DIR)
    try:
        import _cuMPM as R
    finally:
        sys.path.remove(REF_DIR)
    return R


def _flat(E):
    if isinstance(E, tuple) or np.asarray(E).dtype == object:
        return np.concatenate([np.ravel(np.asarray(e)) for e in E])
    return np.ravel(np.asarray(E))


@pytest.mark.parametrize("radii,qi", [([1.0] * 6, [0, 1, 2, 3, 4, 5]),
                                      ([1.0, 1.3, 1.0, 1.6, 1.3, 1.0], [0, 3, 4]),
                                      ([1.0, 1.3, 1.0, 1.6, 1.3, 1.0], [2])])
def test_polydisperse_quadrupole_field_vs_reference(ref, radii, qi):
    box = (26.0, 24.0, 28.0)
    pos = np.array([[2, 2, 2], [8, 3, 4], [14, 9, 5], [3, 15, 12], [18, 18, 18], [10, 20, 7.0]])
    rng = np.random.default_rng(51)
    N, Nq = len(pos), len(qi)
    P = rng.standard_normal((N, 3)) + 1j * rng.standard_normal((N, 3))
    Q = rng.standard_normal((Nq, 5)) + 1j * rng.standard_normal((Nq, 5))
    sc = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    ef = ref.Polydisperse_Ewald_Electric_Field(box[0], box[1], box[2], 1e-6, 0.5, ref.FieldCalcMode.SOLVER_AX,
                                               list(map(float, radii)), True, list(qi), ref.PrecisionMode.DOUBLE)
    ef.updateParticleCoordinates(*[list(pos[:, d]) for d in range(3)])
    ef.updateDipolesComplex(*[list(f(P[:, d])) for d in range(3) for f in (np.real, np.imag)])
    ef.updateQuadrupolesComplex(*[list(f(Q[:, c])) for c in range(5) for f in (np.real, np.imag)])
    ef.setSelfCoef(list(sc.real), list(sc.imag))
    ef.calculate()
    E_ref = _flat(ef.getEPointHost())
    op = O.PolyEwaldOperator(box, 1e-6, 0.5, radii, True, qi)
    op.set_positions(pos)
    X = np.concatenate([P.ravel(), Q.ravel()])
    E = op.apply(X, sc)
    assert E_ref.shape == E.shape
    np.testing.assert_allclose(E, E_ref, rtol=1e-8, atol=1e-9 * np.abs(E_ref).max())
    # the device operator against the reference build
    import torch
    from cumpm_b200 import capi
    F = capi.Field(capi.FIELD_POLY, box, 1e-6, 0.5, radius=radii, quad_idxs=qi, solve_quads=True)
    F.set_positions(pos)
    Y = F.apply(torch.tensor(X.reshape(-1, 1), device="cuda"),
                self_coef=torch.tensor(sc.reshape(-1, 1), device="cuda")).cpu().numpy()[:, 0]
    np.testing.assert_allclose(Y, E_ref, rtol=1e-8, atol=1e-9 * np.abs(E_ref).max())
