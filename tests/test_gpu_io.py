"""A solved dipole_solver written with cumpm_b200.io.save_solution and read
back: the stored results are the solver's own, the stored inputs rebuild
the same run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_solution_file_rebuilds_the_run(tmp_path):
    import cumpm_b200 as cuMPM

    sp = 12.0
    pos = np.array([[(i + 0.5 * (j % 2)) * sp, j * np.sqrt(3) / 2 * sp, 0.0] for j in range(4) for i in range(6)])
    box = np.array([100.0, 100.0, 200.0])
    omega = np.array([0.5, 0.7])
    eps = cuMPM.drude_dielectric(omega, 0.1, 1.8, 4.0)
    s = cuMPM.dipole_solver(box, eps, radius=5.0, eps_m=1.77, tol=1e-8, quiet=True, precision="double")
    s.compute(pos)
    p = tmp_path / "run.npz"
    cuMPM.io.save_solution(p, s, pos)
    d = cuMPM.io.load_solution(p)
    np.testing.assert_array_equal(d["dipoles"], s.get_dipoles())
    np.testing.assert_array_equal(d["eff_polarizability"], s.get_eff_polarizability())
    s2 = cuMPM.dipole_solver(d["box"], d["eps_p"], radius=float(d["radius"][0]), eps_m=float(d["eps_m"]),
                             tol=float(d["tol"]), quiet=True, precision="double")
    s2.compute(d["positions"])
    np.testing.assert_allclose(s2.get_dipoles(), d["dipoles"], rtol=1e-12, atol=1e-14 * np.abs(d["dipoles"]).max())
