"""Regenerate ref_eels_split.npz: the reference's EELS sub-dipole offsets
(cubic, Fibonacci and fcc lattices in the unit sphere) and its splitting of
the particles near the beam, from the reference's own Python
(src/cuMPM/eels.py: _make_*_offsets :177-249, _split_close_dipoles
:261-320).  Its compiled module is replaced by a stub that only carries the
precision enum, which the splitting code never calls into.

Usage: python tests/golden/make_eels_split_golden.py <reference source tree>
"""
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if len(sys.argv) != 2:
    sys.exit(f"usage: python {os.path.relpath(__file__)} <reference source tree>")
REF = sys.argv[1]

METHODS = ("cubic", "fibonacci", "fcc")
NSPLIT = (8, 27, 50, 100)


def load_reference_eels():
    pkg = types.ModuleType("cuMPM")
    pkg.__path__ = []
    stub = types.ModuleType("cuMPM._cuMPM")

    class PrecisionMode:
        AUTO, MIXED, DOUBLE = "AUTO", "MIXED", "DOUBLE"

    stub.PrecisionMode = PrecisionMode
    sys.modules["cuMPM"] = pkg
    sys.modules["cuMPM._cuMPM"] = stub
    pkg._cuMPM = stub
    spec = importlib.util.spec_from_file_location("cuMPM.eels", os.path.join(REF, "src", "cuMPM", "eels.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cuMPM.eels"] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    ref = load_reference_eels()
    out = {}
    for m in METHODS:
        for n in NSPLIT:
            e = ref.EELS(box=[100.0] * 3, eps_p=[4.0], omega=[0.15], v=0.3, radius=2.0, split_dist=4.0, N_split=n,
                         split_method=m)
            out[f"offsets_{m}_{n}"] = e._get_unit_offsets()
    rng = np.random.default_rng(8)
    pos = np.array([[0.0, 0.0, 0.0], [10.0, 0.0, 0.0], [1.0, 1.0, 5.0], [-2.5, 2.0, -4.0]])
    radii = np.array([2.0, 2.5, 1.5, 1.8])
    eps = rng.standard_normal((2, 4)) + 1j * rng.standard_normal((2, 4))
    epos = np.array([1.0, 0.0])
    out.update(split_pos_in=pos, split_radii_in=radii, split_eps_in=eps, split_epos=epos, split_dist=4.0)
    for m, n in (("cubic", 27), ("fibonacci", 20), ("fcc", 50)):
        e = ref.EELS(box=[100.0] * 3, eps_p=[4.0], omega=[0.15, 0.2], v=0.3, radius=2.0, split_dist=4.0, N_split=n,
                     split_method=m)
        p, r, ep = e._split_close_dipoles(pos, epos, radii, eps)
        out[f"split_{m}_{n}_pos"], out[f"split_{m}_{n}_radii"], out[f"split_{m}_{n}_eps"] = p, r, ep
    np.savez(os.path.join(HERE, "ref_eels_split.npz"), **out)
    print("written", os.path.join(HERE, "ref_eels_split.npz"))


if __name__ == "__main__":
    main()
