"""Full solve on the GPU through the drop-in API against golden vectors,
the oracle and dense linear algebra."""
import numpy as np
import pytest

from oracle import mpm_oracle as O

pytestmark = pytest.mark.gpu


def drude(omega, gamma, omega_p, eps_inf):
    return eps_inf - omega_p ** 2 / (omega ** 2 + 1j * omega * gamma)


def hex_lattice(n, spacing):
    pts = []
    lim = int(np.ceil(np.sqrt(n))) * 2
    for j in range(lim):
        for i in range(lim):
            pts.append([(i + 0.5 * (j % 2)) * spacing, j * np.sqrt(3) / 2 * spacing, 0.0])
            if len(pts) == n:
                return np.array(pts)
    return np.array(pts)


def hex_box(pos, spacing, radius, tol=1e-3, xi=0.5):
    rc = np.sqrt(-np.log(tol)) / xi
    mn = 2.1 * rc * radius
    return np.array([max(pos[:, 0].max() + spacing, mn), max(pos[:, 1].max() + spacing * np.sqrt(3) / 2, mn), 1000.0])


def test_dipole_golden_bicgstab(golden):
    import cumpm_b200 as cuMPM
    g = golden("ref_dipole_monodisperse.npz")
    s = cuMPM.dipole_solver(g["box"], g["eps_p"], radius=float(g["radius"]), eps_m=float(g["eps_m"]),
                            tol=float(g["tol"]), field_type="monodisperse", solver_type="bicgstab", quiet=True,
                            precision="double")
    s.compute(g["pos"])
    np.testing.assert_allclose(s.get_eff_polarizability(physical=False), g["alpha_py"], rtol=1e-3, atol=1e-3)
    np.testing.assert_allclose(s.get_dipoles(physical=False), g["dips_py"], rtol=1e-3, atol=1e-3)


def test_quadrupole_golden(golden):
    import cumpm_b200 as cuMPM
    g = golden("ref_quadrupoles_monodisperse.npz")
    s = cuMPM.dipole_solver(g["box"], complex(g["eps_p"]), radius=1.0, eps_m=1.0, xi=float(g["xi"]),
                            tol=float(g["tol"]), field_type="monodisperse", quiet=True, quadrupoles=True,
                            precision="double")
    s.compute(g["pos"])
    d, q = s.get_dipoles(), s.get_quadrupoles()
    assert d.shape == (2, 3, 3) and q.shape == (2, 3, 5)
    for k in range(3):
        np.testing.assert_allclose(d[:, k], g["dips_py_all"][k], rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(q[:, k], g["quads_py_all"][k], rtol=1e-5, atol=1e-5)


def test_near_field_golden(golden):
    import cumpm_b200 as cuMPM
    g = golden("ref_near_field.npz")
    nf = cuMPM.Near_Field(g["box"], g["E0"], radius=1.0, dip=g["dipoles"], dip_pos=g["dip_pos"],
                          field_points=g["field_points"])
    I = nf.calculate()
    assert I.shape == (3,)
    np.testing.assert_allclose(I, g["intensity_py"], rtol=1e-4, atol=1e-4)
    # and the oracle restatement of the same evaluation (fp32 reciprocal here)
    Io = O.near_field_intensity(g["box"], g["E0"], 1.0, g["dipoles"], g["dip_pos"], g["field_points"])
    np.testing.assert_allclose(I, Io, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("solver_type", ["gmres", "bicgstab"])
def test_solution_matches_dense_solve(solver_type):
    """Converged GPU dipoles equal the dense FP64 solve of the same operator."""
    import cumpm_b200 as cuMPM
    rng = np.random.default_rng(21)
    box = np.array([22.0, 22.0, 22.0])
    pos = rng.uniform(0, 22, (9, 3))
    eps = np.array([-6.0 + 1.5j, -3.0 + 0.8j])
    s = cuMPM.dipole_solver(box, eps, radius=1.0, eps_m=1.0, tol=1e-10, quiet=True, solver_type=solver_type,
                            field_type="monodisperse", precision="double", guess_type="mean_field")
    s.compute(pos)
    d = s.get_dipoles(physical=False)  # (W, N, K, 3)
    op = O.MonoEwaldOperator(box, 1e-10, 0.5, True)
    op.set_positions(pos)
    n = 27
    for w, e in enumerate(eps):
        sc = np.full(9, -3.0 / (4 * np.pi * (1 - e)))
        A = np.stack([op.apply(np.eye(n)[:, k], sc) for k in range(n)], axis=1)
        for k in range(3):
            b = np.tile(np.eye(3)[k], 9).astype(complex)
            x = np.linalg.solve(A, b).reshape(9, 3)
            np.testing.assert_allclose(d[w, :, k], x, rtol=1e-7, atol=1e-8 * np.abs(x).max())


@pytest.mark.parametrize("solver_type", ["gmres", "bicgstab"])
def test_matches_oracle_driver_hex(solver_type):
    """Driver semantics (nondimensionalisation, derivative guesses, frequency
    loop, rescaling) against the oracle restatement on a hex monolayer."""
    import cumpm_b200 as cuMPM
    pos = hex_lattice(60, 12.0)
    box = hex_box(pos, 12.0, 5.0, tol=1e-9)
    box[2] = 200.0
    omega = np.linspace(0.4, 0.8, 4)
    eps = drude(omega, 0.1, 1.8, 4.0)
    kw = dict(radius=5.0, eps_m=1.77, tol=1e-9, solver_type=solver_type, field_type="monodisperse")
    s = cuMPM.dipole_solver(box, eps, quiet=True, precision="double", **kw)
    s.compute(pos)
    o = O.DipoleSolverOracle(box, eps, **kw)
    o.compute(pos)
    np.testing.assert_allclose(s.get_dipoles(), o.get_dipoles()[0], rtol=1e-6, atol=1e-7 * np.abs(o.get_dipoles()).max())
    a_o = o.get_eff_polarizability()
    np.testing.assert_allclose(s.get_eff_polarizability(), a_o, rtol=1e-6, atol=1e-9 * np.abs(a_o).max())


def test_refinement_reaches_true_residual():
    """Mixed precision: fp32 inner solves, fp64 true residual |b-Ax|/|b| <= tol."""
    from cumpm_b200 import capi
    import torch
    rng = np.random.default_rng(31)
    pos = hex_lattice(120, 2.4)
    box = (pos[:, 0].max() + 2.4, max(pos[:, 1].max() + 2.1, 16.0), 60.0)
    N = len(pos)
    F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    F.set_positions(pos)
    eps = drude(np.linspace(0.3, 0.9, 6), 0.1, 1.8, 4.0) / 1.77
    K = 3
    M = len(eps) * K
    sc = np.repeat((3.0 / (4 * np.pi * (eps - 1)))[None, :], K, axis=1)
    sc = np.repeat(np.repeat((3.0 / (4 * np.pi * (eps - 1))), K)[None, :], N, axis=0)
    B = np.zeros((3 * N, M), complex)
    for m in range(M):
        B[m % 3::3, m] = 1.0
    Bt = torch.tensor(B, device="cuda")
    St = torch.tensor(sc, device="cuda")
    X = torch.zeros_like(Bt)
    rep = F.batch_solve(Bt, X, St, tol=1e-6, refine=True, inner_tol=1e-4)
    assert rep["num_converged"] == M
    assert 0 <= rep["max_rel_resid"] <= 1e-6
    # independent fp64 check of the residual
    R = Bt - F.apply(X, self_coef=St)
    rr = (torch.linalg.vector_norm(R, dim=0) / torch.linalg.vector_norm(Bt, dim=0)).max().item()
    assert rr <= 1e-6
    # fp64 GMRES to the same true residual gives the same dipoles
    X64 = torch.zeros_like(Bt)
    F.batch_solve(Bt, X64, St, tol=1e-9, recip_fp32=False)
    d = (X - X64).abs().max().item() / X64.abs().max().item()
    assert d < 1e-5


@pytest.mark.parametrize("method", ["gmres", "bicgstab"])
@pytest.mark.parametrize("inner_tol", [1e-4, 1e-5])
def test_compact_batch_matches_full_batch(method, inner_tol):
    """Idle columns left out of the operator: same converged dipoles, fewer column matvecs."""
    from cumpm_b200 import capi
    import torch
    pos = hex_lattice(120, 2.4)
    box = (pos[:, 0].max() + 2.4, max(pos[:, 1].max() + 2.1, 16.0), 60.0)
    N = len(pos)
    F = capi.Field(capi.FIELD_MONO, box, 1e-6, 0.5)
    F.set_positions(pos)
    eps = drude(np.linspace(0.3, 0.9, 6), 0.1, 1.8, 4.0) / 1.77
    K = 3
    M = len(eps) * K
    sc = np.repeat(np.repeat((3.0 / (4 * np.pi * (eps - 1))), K)[None, :], N, axis=0)
    B = np.zeros((3 * N, M), complex)
    for m in range(M):
        B[m % 3::3, m] = 1.0
    Bt = torch.tensor(B, device="cuda")
    St = torch.tensor(sc, device="cuda")
    meth = capi.METHOD_BICGSTAB if method == "bicgstab" else capi.METHOD_GMRES
    out = {}
    for compact in (False, True):
        X = torch.zeros_like(Bt)
        # per-column solves (the shifted first correction's seed matvecs are
        # counted per seed, not per column)
        rep = F.batch_solve(Bt, X, St, tol=1e-6, method=meth, refine=True, inner_tol=inner_tol, compact=compact,
                            shifted=False)
        assert rep["num_converged"] == M
        R = Bt - F.apply(X, self_coef=St)
        rr = (torch.linalg.vector_norm(R, dim=0) / torch.linalg.vector_norm(Bt, dim=0)).max().item()
        assert rr <= 1e-6
        out[compact] = (X, rep)
    (Xf, rf), (Xc, rc) = out[False], out[True]
    assert rc["column_matvecs"] < rf["column_matvecs"]
    assert rf["column_matvecs"] == rf["matvecs"] * M
    d = (Xc - Xf).abs().max().item() / Xf.abs().max().item()
    assert d < 1e-5


def test_batch_all_frequencies_matches_sequential():
    import cumpm_b200 as cuMPM
    pos = hex_lattice(40, 12.0)
    box = hex_box(pos, 12.0, 5.0, tol=1e-9)
    box[2] = 200.0
    eps = drude(np.linspace(0.3, 0.9, 5), 0.1, 1.8, 4.0)
    kw = dict(radius=5.0, eps_m=1.77, tol=1e-9, quiet=True, precision="double")
    a = cuMPM.dipole_solver(box, eps, **kw)
    a.compute(pos)
    b = cuMPM.dipole_solver(box, eps, **kw)
    b.set_solver_options(batch_all=True)
    b.compute(pos)
    np.testing.assert_allclose(b.get_dipoles(), a.get_dipoles(), rtol=1e-6, atol=1e-7 * np.abs(a.get_dipoles()).max())


def test_direct_vs_ewald_large_box():
    """Reference test: open-boundary direct sum vs Ewald in a large box."""
    import cumpm_b200 as cuMPM
    box = np.array([120.0, 120.0, 120.0])
    pos = np.array([[0.0, 0, 0], [12, 0, 0], [-12, 0, 0], [0, 12, 0], [0, -12, 0]])
    kw = dict(radius=1.0, eps_m=1.0, tol=1e-5, quiet=True, quadrupoles=True, precision="double")
    sd = cuMPM.dipole_solver(box, 4.5 + 0.2j, field_type="direct", **kw)
    sd.compute(pos)
    se = cuMPM.dipole_solver(box, 4.5 + 0.2j, xi=0.4, field_type="monodisperse", **kw)
    se.compute(pos)
    np.testing.assert_allclose(sd.get_eff_polarizability(), se.get_eff_polarizability(), rtol=1e-3, atol=1e-5)
    np.testing.assert_allclose(sd.get_dipoles(), se.get_dipoles(), rtol=1e-3, atol=1e-5)
    np.testing.assert_allclose(sd.get_quadrupoles(), se.get_quadrupoles(), rtol=1e-3, atol=5e-5)


def test_multiframe_and_getters():
    import cumpm_b200 as cuMPM
    rng = np.random.default_rng(41)
    box = np.array([40.0, 40.0, 40.0])
    frames = rng.uniform(0, 40, (2, 12, 3))
    eps = np.array([-4 + 1j, -5 + 1j, -6 + 1j])
    s = cuMPM.dipole_solver(box, eps, radius=1.0, tol=1e-8, quiet=True, precision="double")
    s.compute(frames)
    d = s.get_dipoles(physical=False)
    assert d.shape == (2, 3, 12, 3, 3)
    a = s.get_eff_polarizability(physical=False)
    np.testing.assert_allclose(a, d.mean(axis=(0, 2)), rtol=1e-12)
    assert s.use_jacobi_precond
    s.use_jacobi_precond = False
    assert not s.use_jacobi_precond
    assert all(i > 0 for i in s.get_iterations())
