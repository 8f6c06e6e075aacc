"""Regenerate the golden fixtures in this directory (run where the reference
source tree is available; the fixtures themselves are committed and are all
the tests need).

* ref_dipole_monodisperse.npz / ref_quadrupoles_monodisperse.npz /
  ref_near_field.npz: the reference's own golden vectors
  (tests/data/*.npz of the reference) together with the inputs its tests
  use (tests/test_dipole_solvers.py:8-149, tests/test_near_fields.py:31-75).
* refcpu_tables.npz: real-space tables from the reference's CPU operator
  (tests/quadrupole_field.py, Electric_Field._calc_real_space_table), every
  10th entry, at xi = 0.4 and 0.5.
* refcpu_operator.npz: field E and field gradient G from that CPU operator
  for seeded random dipoles and quadrupoles on a 6-particle periodic box.
* ref_eels_vs_python_module.npz: the reference's EELS golden vector
  (tests/data/ref_eels_vs_python_module.npz) with the inputs of the test
  that reads it (tests/test_eels_solver.py:114-173): loss spectra of two
  beam positions at five frequencies and the scaled dipoles.

Usage: python tests/golden/make_golden.py <reference source tree>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if len(sys.argv) != 2:
    sys.exit(f"usage: python {os.path.relpath(__file__)} <reference source tree>")
REF = sys.argv[1]


def drude(omega, gamma, omega_p, eps_inf):
    return eps_inf - omega_p ** 2 / (omega ** 2 + 1j * omega * gamma)


def main():
    data = os.path.join(REF, "tests", "data")
    # --- reference golden vectors with their inputs
    g = np.load(os.path.join(data, "ref_dipole_monodisperse.npz"))
    d = 12.0
    omega = np.linspace(2000, 6000, 3)
    eps = drude(omega, 700, 12000, 4.0)
    np.savez(os.path.join(HERE, "ref_dipole_monodisperse.npz"), alpha_py=g["alpha_py"], dips_py=g["dips_py"],
             pos=np.array([[0, 0, 0], [d, 0, 0], [0, d, 0], [d, d, 0]], float), box=np.full(3, 5 * d),
             eps_p=np.repeat(eps[:, None], 4, axis=1), radius=4.0, eps_m=2.13, tol=1e-4)
    g = np.load(os.path.join(data, "ref_quadrupoles_monodisperse.npz"))
    np.savez(os.path.join(HERE, "ref_quadrupoles_monodisperse.npz"), dips_py_all=g["dips_py_all"],
             quads_py_all=g["quads_py_all"], pos=np.array([[10.0, 10, 10], [20, 20, 20]]), box=np.full(3, 100.0),
             xi=0.4, eps_p=4.5 + 0.2j, tol=1e-8)
    g = np.load(os.path.join(data, "ref_near_field.npz"))
    np.savez(os.path.join(HERE, "ref_near_field.npz"), intensity_py=g["intensity_py"], box=np.full(3, 50.0),
             E0=np.array([1.0, 0, 0]),
             dip_pos=np.array([[0, 0, 0], [10, 0, 0], [0, 10, 0], [0, 0, 10.0]]),
             dipoles=np.array([[0.1 + 0.05j, 0, 0], [-0.1, 0.02j, 0], [0, 0.05, -0.01j], [0.01, 0, 0.1j]]),
             field_points=np.array([[5.0, 0, 0], [0, 5, 0], [2.5, 2.5, 2.5]]))
    g = np.load(os.path.join(data, "ref_eels_vs_python_module.npz"))
    d = 25.0 + 2.6
    omega = np.linspace(2000.0, 9000.0, 5)
    np.savez(os.path.join(HERE, "ref_eels_vs_python_module.npz"), ref_eels=g["ref_eels"],
             ref_dips_stacked=g["ref_dips_stacked"], box=np.full(3, 10.0 * d),
             points=np.array([[-0.5, 0.0, 0.0], [0.5, 0.0, 0.0]]) * d, e_pos=np.array([[0.0, 0.0], [1.0, 0.0]]) * d,
             radius=0.5 * 25.0, omega_cm=omega, eps_p=drude(omega, 845.0, 11886.0, 2.25), omega_nm=omega / 1e7,
             v=0.45, eps_m=1.0)
    # --- reference CPU operator
    sys.path.insert(0, os.path.join(REF, "tests"))
    from quadrupole_field import Electric_Field

    names = ["field_dip_1", "field_dip_2", "field_quad_1", "field_quad_2", "field_quad_3", "grad_quad_1",
             "grad_quad_2", "grad_quad_3", "grad_quad_4"]
    tabs = {}
    for xi in (0.4, 0.5):
        ef = Electric_Field(np.full(3, 40.0), xi, 1e-6, eps_p=4.0)
        for n in names:
            tabs[f"{n}@{xi}"] = np.asarray(getattr(ef, n))[::10]
        tabs[f"r@{xi}"] = np.asarray(ef.r_table)[::10]
    np.savez(os.path.join(HERE, "refcpu_tables.npz"), **tabs)

    rng = np.random.default_rng(0)
    box = np.full(3, 20.0)
    xi, tol, eps = 0.5, 1e-6, 4.5 + 0.2j
    pos = np.array([[1.0, 1, 1], [5.2, 1.3, 0.7], [3, 6, 2], [9, 9, 9], [12, 3, 15], [15, 14, 3]])
    N = len(pos)
    P = rng.standard_normal((N, 3)) + 1j * rng.standard_normal((N, 3))
    Q = rng.standard_normal((N, 5)) + 1j * rng.standard_normal((N, 5))
    ef = Electric_Field(box, xi, tol, eps_p=eps)
    ef.set_points(pos)
    ef.set_dip_pos(pos)
    out = dict(box=box, xi=xi, tol=tol, eps=eps, pos=pos, P=P, Q=Q)
    for tag, (pp, qq) in {"dip": (P, 0 * Q), "quad": (0 * P, Q)}.items():
        ef.set_dipoles(pp, qq)
        E, G = ef.calculate()
        out[f"E_{tag}"] = np.array(E)
        out[f"G_{tag}"] = np.array(G)
    np.savez(os.path.join(HERE, "refcpu_operator.npz"), **out)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
