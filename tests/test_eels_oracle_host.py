"""The EELS oracle (oracle/mpm_eels.py) against the reference's EELS golden
vector and the reference's own K0/K1 rules.  No GPU needed."""
import numpy as np
import pytest
from scipy import special

from oracle import mpm_eels as E


def test_reference_golden_two_beams_five_frequencies(golden):
    """tests/test_eels_solver.py:114-173 of the reference: two spheres, two
    beam positions, five frequencies, direct field; loss spectra (as
    loss / (omega R) * (4 pi)^2) and scaled dipoles to the test's 2e-2."""
    g = golden("ref_eels_vs_python_module.npz")
    o = E.EELSOracle(g["box"], g["eps_p"], g["omega_nm"], float(g["v"]), eps_m=float(g["eps_m"]),
                     radius=float(g["radius"]), xi=0.5, tol=1e-3, field_type="direct")
    for e in g["e_pos"]:
        o.compute(e, g["points"])
    eels = np.array(o.eels) / (g["omega_nm"] * float(g["radius"])) * (4.0 * np.pi) ** 2
    np.testing.assert_allclose(eels, g["ref_eels"], rtol=2e-2, atol=1e-5)
    np.testing.assert_allclose(np.array(o.dipoles), g["ref_dips_stacked"], rtol=2e-2, atol=1e-5)
    # closer than the test asks: the remaining 0.3 % is the 0.5 nm soft core
    # of the beam, absent from the golden's generator
    assert np.max(np.abs(eels - g["ref_eels"]) / np.abs(g["ref_eels"])) < 5e-3


@pytest.mark.parametrize("n", [0, 1])
def test_bessel_k_follows_the_reference_rules(n):
    x = np.linspace(0.05, 12.0, 40)
    for v in x:
        assert E.eval_k(n, v) == pytest.approx(special.kv(n, v), rel=1e-14)
        # imaginary axis: the Hankel form equals K_n(iy) and K_n(-iy)
        for y in (v, -v):
            np.testing.assert_allclose(E.eval_k(n, 1j * y), special.kv(n, 1j * y), rtol=1e-12)
    # both parts nonzero: the reference keeps the real part only
    assert E.eval_k(n, 2.0 + 0.5j) == pytest.approx(special.kv(n, 2.0), rel=1e-14)


def test_loss_is_the_reciprocity_sum():
    """The loss is sum Im(p . conj(E_inc)) / (2 pi^2) over the converged
    dipoles and the beam field at the particles (eels_solver.cu:796-838),
    positive for lossy particles."""
    box, pts = np.full(3, 200.0), np.array([[-8.0, 0, 0], [8.0, 0, 0], [0, 9.0, 3.0]])
    o = E.EELSOracle(box, [4.0 + 0.2j], [0.05, 0.08], 0.4, radius=3.0, field_type="direct")
    eels, dips = o.compute([1.5, -2.0], pts)
    ls, om = 3.0, np.array([0.05, 0.08]) * 3.0
    gamma = 1.0 / np.sqrt(1.0 - 0.4 ** 2)
    for w in range(2):
        Einc = E.beam_field(pts / ls, np.array([1.5, -2.0]) / ls, om[w], 0.4, gamma, ls)
        want = np.sum(np.imag(np.sum(dips[w] * np.conj(Einc), axis=1))) / (2 * np.pi ** 2)
        assert eels[w] == pytest.approx(want, rel=1e-12)
        assert eels[w] > 0.0   # a lossy particle absorbs


def test_zone_sum_in_a_large_box_is_the_isolated_pair():
    """The Brillouin-zone sum (beam images with Bloch phases on the Ewald
    operator with the Bloch wavevector, eels_solver.cu:491-509, 847-859) of
    a pair in a box much larger than the beam's decay length gives the loss
    of the isolated pair under one beam (direct field), closer with more
    zone points."""
    box, pts = np.full(3, 60.0), np.array([[0.0, 0, 0], [9.0, 0, 0]])
    kw = dict(radius=3.0, xi=0.5, tol=1e-6)
    iso, _ = E.EELSOracle(box, [4.0 + 0.3j], [0.05], 0.4, field_type="direct", **kw).compute([5.0, 3.0], pts)
    errs = []
    for n in (1, 2):
        z, _ = E.EELSOracle(box, [4.0 + 0.3j], [0.05], 0.4, field_type="monodisperse", asm=True, asm_n=(n, n),
                            **kw).compute([5.0, 3.0], pts)
        errs.append(abs(z[0] - iso[0]) / iso[0])
    assert errs[0] < 2e-3 and errs[1] < errs[0]
