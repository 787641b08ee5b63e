"""Shared set-up of the projection-matching tests: the golden fixtures made
by tests/golden/make_match_golden.py from the reference's own code."""
import os

import numpy as np

from bsoft_b200.geometry import view_to_matrix

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MATCH_CASES = ["match64", "match32"]


def load(case: str):
    z = np.load(os.path.join(GOLDEN, case + ".npz"))
    d = {k: z[k] for k in z.files}
    d["name"] = case
    d["N"] = int(d["map"].shape[0])
    d["n"] = int(d["images"].shape[1])
    d["pixel"] = float(d["pixel"])
    d["hi_res"] = float(d["hi_res"])
    d["diam"] = int(d["diam"])
    d["mats"] = np.stack([view_to_matrix(v) for v in d["views"]])
    return d


def ctf_records(d):
    """CTF records (8 doubles) from the fixture's rows [volt, abw00..abw40, apply]."""
    out = np.zeros((len(d["ctf_rows"]), 8))
    out[:, :6] = d["ctf_rows"][:, :6]
    out[:, 6] = d["ctf_rows"][:, 6]          # 1 = apply
    return out


def hypotheses(d):
    rows = []
    for i, v, ox, oy in d["hyps"]:
        rows.append([i, *d["mats"][int(v)].reshape(9), ox, oy])
    return np.array(rows)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
