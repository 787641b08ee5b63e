"""Golden results of brefine with -symmetry: part_refine_orientation refines
each particle from every view of symmetry_get_all_views and keeps, in view
order, the first result that beats the best so far (starting from 0),
numbering the winning view in the particle's selection (bsoft/src/mg/
mg_refine.cpp:584-621).  The compiled brefine program runs on a STAR project
of the refine32 / refine64 particles (one micrograph per particle, as
tests/test_cli.py writes it) with -symmetry D2 and C3; refine_sym.npz keeps
per case the symmetry and rows of view x, y, z, angle, origin x, y, fom,
selection.

    python tests/golden/make_refine_sym_golden.py
"""
from __future__ import annotations

import math
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from make_refine_ccurve_golden import _star_column  # noqa: E402
from bsoft_b200.project import read_project  # noqa: E402
from tests.refine_helpers import load  # noqa: E402
from tests.test_cli import _write_refine_project  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))
CASES = [("refine32", "D2"), ("refine64", "C3")]


def program(name: str, sym: str) -> np.ndarray:
    d = load(name)
    with tempfile.TemporaryDirectory() as td:
        star = _write_refine_project(d, td)
        out = os.path.join(td, "out.star")
        args = [os.path.join(REF, "brefine"), "-reference", os.path.join(td, "ref.mrc"),
                "-grid", f"{round(d['alpha'] * 180 / math.pi, 6)},{round(d['accuracy'] * 180 / math.pi, 6)}",
                "-step", f"{d['shift_step']},{d['shift_accuracy']}", "-resolution", repr(d["hi_res"]),
                "-symmetry", sym, "-output", out, star]
        subprocess.run(args, capture_output=True, text=True, check=True, timeout=3600, cwd=td,
                       env=dict(os.environ, OMP_NUM_THREADS="4"))
        proj = read_project(out)
        fom = _star_column(out, "particle.fom")
        sel = _star_column(out, "particle.select")
    rows = [[*mg.view[0], *mg.origin[0, :2]] for mg in proj.micrographs]
    return np.column_stack([np.array(rows), fom, sel])


if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF, "brefine")):
        sys.exit("build the reference first: make -C oracle ref")
    res = {}
    for name, sym in CASES:
        res[f"{name}_{sym}"] = program(name, sym)
    path = os.path.join(OUT, "refine_sym.npz")
    np.savez_compressed(path, **res)
    print(path)
