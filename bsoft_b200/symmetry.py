"""Point-group symmetry operators as the reference generates them (host side).

* ``Bsymmetry::Bsymmetry`` (bsoft/src/util/symmetry.cpp:42-115) and
  ``clean_symstring`` (bsoft/include/symmetry.h:73-99): the generating
  operations (axis, order) of the cyclic, dihedral, tetrahedral, octahedral
  and icosahedral groups;
* ``symmetry_get_all_views`` (symmetry.cpp:277-319): every group element
  applied to a view, in the order the reference lists them: for each
  operation and each power j = 1 .. order-1 of it, the rotation by
  j 2 pi / order about the operation's axis times every view listed so far.

The reference rotates the view's quaternion, q * qv, so the symmetric view
has the matrix M(q) M(qv): ``operators`` returns the M(q) the C ABI's
``bsg_recon_set_symmetry`` takes (identity first).  Helical symmetry and the
rotated setting I90 are not covered.
"""
from __future__ import annotations

import math

import numpy as np

GOLDEN = 1.61803398874989484820458683436563811772   # bsoft/include/utilities.h:89-90


def clean_label(sym: str) -> str:
    """clean_symstring: empty -> C1, numeric names, upper-case first letter."""
    lbl = "".join((sym or "").split())
    if not lbl:
        return "C1"
    if lbl[0].isdigit():
        digits = ""
        for ch in lbl:
            if not ch.isdigit():
                break
            digits += ch
        j = int(digits) if digits else 0
        if "532" in lbl:
            lbl = "I90" if "90" in lbl else "I"
        elif "432" in lbl:
            lbl = "O"
        elif "23" in lbl:
            lbl = "T"
        elif j > 1 and len(lbl) > 1 and lbl[1] == "2":
            lbl = f"D{j}"
        elif j > 0:
            lbl = f"C{j}"
        else:
            lbl = "C1"
    return lbl[0].upper() + lbl[1:]


def generators(sym: str):
    """The (unit axis, order) operations of Bsymmetry for a point group."""
    out = []
    for ax, order in generator_axes(sym):
        a = np.asarray(ax, dtype=np.float64)
        out.append((a / np.linalg.norm(a), int(order)))
    return out


def generator_axes(sym: str):
    """The (axis, order) operations of Bsymmetry for a point group, with the
    axes as Bsymmetry::Bsymmetry writes them (bsoft/src/util/symmetry.cpp:
    53-99), before its normalisation: the form bsg_recon_set_symmetrize
    takes."""
    lbl = clean_label(sym)
    ops = []
    g = lbl[0]
    if g == "C":
        order = 1 if lbl == "Cs" else int(lbl[1:] or 1)
        ops.append(((0, 0, 1), order))
    elif g == "D":
        ops.append(((0, 0, 1), int(lbl[1:])))
        ops.append(((1, 0, 0), 2))
    elif g == "T":
        if "-3" not in lbl:
            ops.append(((1, 1, 1), 3))
        ops.append(((0, 0, 1), 2))
        ops.append(((1, 0, 0), 2))
    elif g == "O":
        if "-3" not in lbl:
            ops.append(((1, 1, 1), 3))
        if "-4" in lbl:
            ops.append(((1, -1, 0), 2))
        elif "-2" in lbl:
            ops.append(((0, 0, 1), 4))
        else:
            ops.append(((0, 0, 1), 4))
            ops.append(((1, 0, 0), 2))
    elif g == "I":
        if "90" in lbl:
            raise ValueError("the rotated icosahedral setting I90 is not supported")
        if "-3" not in lbl:
            ops.append(((1, 1, 1), 3))
        if "-5" in lbl:
            ops.append(((1, 0, 0), 2))
        elif "-2" in lbl:
            ops.append(((1, -1, 0), 2))
        else:
            ops.append(((1, 1.0 / GOLDEN, GOLDEN), 2))
        if "-5" not in lbl:
            ops.append(((1.0 / GOLDEN, 1, 0), 5))
        if "-2" not in lbl:
            ops.append(((0, 0, 1), 2))
    else:
        raise ValueError(f"unsupported symmetry {sym!r}")
    return [(tuple(float(v) for v in ax), int(order)) for ax, order in ops]


def _quat(axis, angle):
    s = math.sin(angle / 2)
    return np.array([math.cos(angle / 2), axis[0] * s, axis[1] * s, axis[2] * s])


def _qmul(p, q):
    return np.array([p[0] * q[0] - p[1] * q[1] - p[2] * q[2] - p[3] * q[3],
                     p[0] * q[1] + p[1] * q[0] + p[2] * q[3] - p[3] * q[2],
                     p[0] * q[2] + p[2] * q[0] + p[3] * q[1] - p[1] * q[3],
                     p[0] * q[3] + p[3] * q[0] + p[1] * q[2] - p[2] * q[1]])


def _qmat(q):
    q0, q1, q2, q3 = q
    return np.array([[q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3, 2 * q1 * q2 - 2 * q0 * q3, 2 * q1 * q3 + 2 * q0 * q2],
                     [2 * q1 * q2 + 2 * q0 * q3, q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3, 2 * q2 * q3 - 2 * q0 * q1],
                     [2 * q1 * q3 - 2 * q0 * q2, 2 * q2 * q3 + 2 * q0 * q1, q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3]])


def operators(sym: str) -> np.ndarray:
    """(order, 3, 3) rotation matrices of the group elements in the order of
    symmetry_get_all_views (identity first)."""
    quats = [np.array([1.0, 0.0, 0.0, 0.0])]
    for axis, order in generators(sym):
        n = len(quats)
        for j in range(1, order):
            q = _quat(axis, j * 2.0 * math.pi / order)
            for k in range(n):
                quats.append(_qmul(q, quats[k]))
    return np.stack([_qmat(q) for q in quats])


def random_view_indices(n: int, order: int, seed: int) -> list:
    """The group element breconstruct -mode 2 picks for each of n particles,
    in particle order (random_symmetric_view, bsoft/src/util/symmetry.cpp:
    816-832): the C library's random() after srandom(seed) (the reference
    seeds it with its process id), index floor(order random() 0.99999 /
    get_rand_max()) in long double, where get_rand_max() itself draws 100
    further numbers (bsoft/src/util/random_numbers.cpp:22-30) after the
    index's draw.  Index into symmetry_get_all_views' order (operators())."""
    import ctypes
    libc = ctypes.CDLL(None)
    libc.random.restype = ctypes.c_long
    libc.srandom.argtypes = [ctypes.c_uint]
    libc.srandom(int(seed) & 0xFFFFFFFF)
    out = []
    for _ in range(n):
        r = libc.random()
        rand_max = 32767
        for _ in range(100):
            if libc.random() > rand_max:
                rand_max = 2147483647
        i = int(np.longdouble(order * r) * np.longdouble("0.99999") / np.longdouble(rand_max))
        out.append(i)
    return out
