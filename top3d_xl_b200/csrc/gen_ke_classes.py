#!/usr/bin/env python
"""Generate topx_ke_classes.h: the value classes of the hex8 element stiffness matrix.

The 576 entries of the isotropic unit-cube Ke (interleaved DOFs 3a+c, local nodes in the
order of kHexNode in topx_mesh.cpp) take only a few distinct magnitudes, identical for
every Poisson ratio.  The header maps each entry to sign * (class + 1), classes numbered by
first occurrence in row-major order, so the level-1 operator kernel can address ten values
instead of 576 constants.  Run from this directory:  python gen_ke_classes.py
"""
import math
import os

import numpy as np

HEX_NODE = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                     [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)


def stiffness(nu):
    """2x2x2 Gauss integration of B^T D B on the unit cube (E = 1)."""
    lam = nu / ((1 + nu) * (1 - 2 * nu))
    mu = 1.0 / (2 * (1 + nu))
    D = np.full((3, 3), lam) + 2 * mu * np.eye(3)
    D = np.block([[D, np.zeros((3, 3))], [np.zeros((3, 3)), mu * np.eye(3)]])
    g = 1 / math.sqrt(3)
    K = np.zeros((24, 24))
    for gs in (-g, g):
        for gt in (-g, g):
            for gq in (-g, g):
                s, t, p = HEX_NODE.T
                dNs = 0.125 * s * (1 + t * gt) * (1 + p * gq) * 2
                dNt = 0.125 * t * (1 + s * gs) * (1 + p * gq) * 2
                dNp = 0.125 * p * (1 + s * gs) * (1 + t * gt) * 2
                B = np.zeros((6, 24))
                B[0, 0::3], B[1, 1::3], B[2, 2::3] = dNs, dNt, dNp
                B[3, 0::3], B[3, 1::3] = dNt, dNs
                B[4, 1::3], B[4, 2::3] = dNp, dNt
                B[5, 0::3], B[5, 2::3] = dNp, dNs
                K += B.T @ D @ B * 0.125
    return K


def classes():
    """sign * (class + 1) per entry; the sign is relative to the class's first entry."""
    Ks = [stiffness(nu) for nu in (0.3, 0.27, 0.41)]
    key_of, first_sign, table = {}, {}, np.zeros(576, int)
    for idx in range(576):
        i, j = divmod(idx, 24)
        vals = [K[i, j] for K in Ks]
        key = tuple(round(abs(v), 10) for v in vals)
        sgn = 1 if vals[0] > 0 else -1
        if key not in key_of:
            key_of[key] = len(key_of)
            first_sign[key] = sgn
        table[idx] = sgn * first_sign[key] * (key_of[key] + 1)
    return table, len(key_of)


def header():
    table, n = classes()
    rows = ",\n".join("    " + ", ".join("%3d" % v for v in table[r * 24:(r + 1) * 24]) for r in range(24))
    return ("// Generated by gen_ke_classes.py; do not edit.\n"
            "// Value classes of the hex8 Ke: entry (3a+i, 3b+c) = sign * value[class], stored as\n"
            "// sign * (class + 1); the sign is relative to the first entry of the class.\n"
            "#pragma once\n\nnamespace topx {\n\n"
            "constexpr int kKeClasses = %d;\n\n"
            "__host__ __device__ constexpr int ke_class_code(int idx) {\n"
            "  constexpr signed char t[576] = {\n%s};\n"
            "  return t[idx];\n}\n\n}  // namespace topx\n" % (n, rows))


if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "topx_ke_classes.h")
    with open(out, "w") as fh:
        fh.write(header())
    print(out, classes()[1], "classes")
