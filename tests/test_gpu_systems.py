"""Several independent systems solved through cumpm_b200.systems give, system
by system, what a dipole_solver of each gives on its own."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _packing(rng, n, box, a):
    pos = []
    while len(pos) < n:
        p = rng.uniform(0, box, 3)
        if all(np.linalg.norm((p - q) - box * np.round((p - q) / box)) >= 2.2 * a for q in pos):
            pos.append(p)
    return np.array(pos)


def _hex(rows, cols, d):
    return np.array([[(i + 0.5 * (j % 2)) * d, j * np.sqrt(3) / 2 * d, 0.0] for j in range(rows) for i in range(cols)])


def _systems():
    from cumpm_b200.systems import System

    rng = np.random.default_rng(41)
    omega = np.linspace(0.3, 0.9, 3)
    eps = 4.0 - 1.8 ** 2 / (omega ** 2 + 1j * omega * 0.1)
    # 10 x 8 monolayer; every box edge above twice the real-space cutoff
    # (about 8 radii at tol 1e-7)
    hexa = _hex(10, 8, 12.0)
    box_h = [8 * 12.0, 10 * np.sqrt(3) / 2 * 12.0, 200.0]
    out = [
        System(box=box_h, positions=hexa, eps_p=eps, radius=5.0, eps_m=1.77, tol=1e-7, quadrupoles=True,
               precision="double"),
        System(box=[40.0] * 3, positions=_packing(rng, 24, 40.0, 2.0), eps_p=eps, radius=2.0, eps_m=1.77, tol=1e-7,
               quadrupoles=[0, 5, 7], precision="double"),
        System(box=[50.0] * 3, positions=_packing(rng, 20, 50.0, 3.0), eps_p=eps,
               radius=list(rng.uniform(1.0, 3.0, 20)), eps_m=1.77, tol=1e-7, field_type="polydisperse",
               precision="double"),
    ]
    return out


def test_systems_match_their_own_solvers():
    from cumpm_b200 import systems as S

    syst = _systems()
    res = S.solve_systems(syst)
    for s, r in zip(syst, res):
        ref = S.solve_one(s)
        assert set(r) == set(ref)
        for k in ref:
            np.testing.assert_allclose(r[k], ref[k], rtol=1e-12, atol=1e-14 * np.abs(ref[k]).max())
    assert "quadrupoles" in res[0] and res[1]["quadrupoles"].shape[-1] == 5 and "quadrupoles" not in res[2]


def test_frequency_blocks_concatenate_to_the_whole_sweep():
    """solve_sharded's pieces: the sweep solved as two frequency blocks
    (what two ranks would each solve) and concatenated equals the whole
    sweep solved at once, to the solves' tolerance; one process is the whole
    sweep itself."""
    from cumpm_b200 import systems as S

    syst = _systems()[0]
    omega = np.linspace(0.3, 0.9, 5)
    syst.eps_p = 4.0 - 1.8 ** 2 / (omega ** 2 + 1j * omega * 0.1)
    syst.options = {"batch_all": True, "refine": True}
    syst.precision = None
    whole = S.solve_one_unsqueezed(syst)
    blocks = []
    for idx in S.frequency_shards(5, 2):
        sub = S.System(**{**syst.__dict__, "eps_p": np.asarray(syst.eps_p)[idx]})
        blocks.append(S.solve_one_unsqueezed(sub))
    # the quadrupoles are a small part of the solution vector, so the same
    # solve tolerance leaves them a larger relative difference
    for key, axis, lim in (("dipoles", 1, 1e-5), ("eff_polarizability", 0, 1e-5), ("quadrupoles", 1, 2e-3)):
        cat = np.concatenate([b[key] for b in blocks], axis=axis)
        assert cat.shape == whole[key].shape
        err = np.linalg.norm(cat - whole[key]) / np.linalg.norm(whole[key])
        assert err < lim, (key, err)
    one = S.solve_sharded(syst)
    assert one["dipoles"].shape == np.squeeze(whole["dipoles"]).shape


@pytest.mark.first_gpu_run
def test_concurrent_systems_match_serial():
    """Three systems solved at once from host threads (each with its own
    device stream) give what they give one after another."""
    from cumpm_b200 import systems as S

    syst = _systems()
    serial = S.solve_systems(syst)
    conc = S.solve_systems(syst, concurrency=3)
    for a, b in zip(conc, serial):
        assert set(a) == set(b)
        for k in b:
            np.testing.assert_allclose(a[k], b[k], rtol=1e-12, atol=1e-14 * np.abs(b[k]).max())
