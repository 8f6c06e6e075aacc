"""On-disk result files (cumpm_b200.io): the examples' extinction-spectrum
layout and the solution dump, round-tripped on CPU (a stand-in solver object
with the dipole_solver getters; no GPU)."""
import numpy as np
import pytest

from cumpm_b200 import io


def test_spectrum_round_trip_in_the_examples_layout(tmp_path):
    w = np.linspace(3000, 9000, 120)
    c = np.sin(w / 1000.0) ** 2
    single = np.cos(w / 1000.0) ** 2
    p = tmp_path / "extinction_data_ratio_2.npz"
    io.save_spectrum(p, w, c, single)
    z = np.load(p)
    assert sorted(z.files) == ["energy_ev", "extinction_cs", "extinction_cs_single", "wavenumber_cm"]
    np.testing.assert_array_equal(z["energy_ev"], w / 8065.54)
    d = io.load_spectrum(p)
    np.testing.assert_array_equal(d["extinction_cs"], c)
    np.testing.assert_array_equal(d["extinction_cs_single"], single)
    with pytest.raises(ValueError, match="one value per wavenumber"):
        io.save_spectrum(p, w, c[:-1])


def test_extinction_cross_section_matches_the_examples_formula():
    rng = np.random.default_rng(0)
    p = rng.standard_normal((5, 7, 3)) + 1j * rng.standard_normal((5, 7, 3))
    E0 = np.array([0.0, 1.0, 0.0])
    k = np.linspace(0.1, 0.5, 5)
    got = io.extinction_cross_section(p, E0, k[:, None][:, 0])
    ref = np.array([4 * np.pi * k[w] * np.sum(np.imag(np.sum(np.conj(E0) * p[w], axis=1))) for w in range(5)])
    np.testing.assert_allclose(got, ref, rtol=1e-14)


class _Solved:
    def __init__(self, quads):
        rng = np.random.default_rng(1)
        self._args = {"box": np.array([10.0, 11.0, 12.0]), "eps_p": np.array([2 + 1j, 3 + 0.5j]),
                      "radius": np.array([1.0]), "eps_m": 1.77, "xi": 0.5, "tol": 1e-6,
                      "E0": np.eye(3, dtype=complex)}
        self.d = rng.standard_normal((2, 4, 3, 3)) + 1j * rng.standard_normal((2, 4, 3, 3))
        self.q = rng.standard_normal((2, 2, 3, 5)) + 0j if quads else np.zeros(0)

    def get_dipoles(self):
        return self.d

    def get_eff_polarizability(self):
        return self.d.mean(axis=1)

    def get_quadrupoles(self):
        return self.q


@pytest.mark.parametrize("quads", [False, True])
def test_solution_round_trip(tmp_path, quads):
    s = _Solved(quads)
    pos = np.arange(12, dtype=float).reshape(4, 3)
    p = tmp_path / "run.npz"
    io.save_solution(p, s, pos, extra={"note": "hex"})
    d = io.load_solution(p)
    np.testing.assert_array_equal(d["dipoles"], s.d)
    np.testing.assert_array_equal(d["positions"], pos)
    np.testing.assert_array_equal(d["eps_p"], s._args["eps_p"])
    assert float(d["eps_m"]) == 1.77 and str(d["note"]) == "hex"
    assert ("quadrupoles" in d) == quads
    with pytest.raises(ValueError, match="collides"):
        io.save_solution(p, s, pos, extra={"dipoles": 1})
    np.savez(tmp_path / "other.npz", a=1)
    with pytest.raises(ValueError, match="not a solution file"):
        io.load_solution(tmp_path / "other.npz")
