"""Shared set-up of the grid-refinement tests: the golden fixtures made by
tests/golden/make_refine_golden.py from the reference's img_refine_grid."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REFINE_CASES = ["refine64", "refine32", "refine64ctf"]


def load(case: str):
    z = np.load(os.path.join(GOLDEN, case + ".npz"))
    d = {k: z[k] for k in z.files}
    d["case"] = case
    d["N"] = int(d["map"].shape[0])
    d["n"] = int(d["images"].shape[1])
    for k in ("pixel", "hi_res", "alpha", "accuracy", "shift_step", "shift_accuracy", "file_avg", "file_std", "volt",
              "def_std"):
        d[k] = float(d[k])
    return d
