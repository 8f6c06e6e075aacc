"""Writes mpm_fft_consts.cuh: W_N^j = exp(-2 pi i j / N) for the composite
and prime butterflies of the in-shared-memory line transforms.

cos and sin are evaluated on the first octant only and mapped to the other
octants by exact symmetries, so that conjugate pairs and quarter turns agree
to the last bit.  Run:  python gen_fft_consts.py > mpm_fft_consts.cuh
"""
import math
from fractions import Fraction as F

RADICES = (7, 9, 10, 11, 12, 13, 14, 15, 16)


def cos_sin(fr):
    """(cos, sin) of the angle 2 pi fr, fr a Fraction of a full turn."""
    fr = fr % 1
    exact = {F(0): (1.0, 0.0), F(1, 4): (0.0, 1.0), F(1, 2): (-1.0, 0.0), F(3, 4): (0.0, -1.0),
             F(1, 12): (math.sqrt(3) / 2, 0.5), F(1, 8): (math.sqrt(0.5), math.sqrt(0.5))}
    if fr in exact:
        return exact[fr]
    if fr > F(1, 2):
        c, s = cos_sin(1 - fr)
        return c, -s
    if fr > F(1, 4):
        c, s = cos_sin(F(1, 2) - fr)
        return -c, s
    if fr > F(1, 8):
        c, s = cos_sin(F(1, 4) - fr)
        return s, c
    a = 2 * math.pi * float(fr)
    return math.cos(a), math.sin(a)


def main():
    print("// Generated by gen_fft_consts.py: W_N^j = exp(-2 pi i j / N), j < N.")
    print("#pragma once\n")
    print("namespace mpm {\n")
    for ty, suf in (("double2", "d"), ("float2", "f")):
        for n in RADICES:
            vals = []
            for j in range(n):
                c, s = cos_sin(F(j, n))
                vals.append("{%.21g, %.21g}" % (c, -s) if ty == "double2" else "{%.9ef, %.9ef}" % (c, -s))
            print(f"__constant__ {ty} kW{n}{suf}[{n}] = {{{', '.join(vals)}}};")
    print("\n}  // namespace mpm")


if __name__ == "__main__":
    main()
