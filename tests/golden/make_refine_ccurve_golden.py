"""Golden results of brefine's grid refinement as the program runs it: the
shells of the figure of merit weighted with the reference's C_curve
(project_refine_orientations, bsoft/src/mg/mg_refine.cpp:366-367; the probe
fixtures use img_recip_space_fom's unit weights), from the reference's own
code, on the inputs of the grid-refinement fixtures (refine32, refine64,
refine64ctf):

* ``<case>_frc`` / ``<case>_dpr``: ``oracle/_ref/refine_probe`` (img_refine_grid
  after brefine's preparation) with the C_curve weights, FRC and DPR;
* ``<case>_brefine_<fom>``: the compiled ``brefine`` program itself on a STAR
  project of the same particles (one micrograph per particle, as
  tests/test_cli.py writes it), its refined views, origins, defoci and
  figures of merit read back from its output project.

    python tests/golden/make_refine_ccurve_golden.py
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

from bsoft_b200.io import mrc  # noqa: E402
from bsoft_b200.project import read_project  # noqa: E402
from make_refine_golden import CASES  # noqa: E402
from tests.refine_helpers import load  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))


def probe(name: str, case: dict, fom_type: int) -> np.ndarray:
    z = np.load(os.path.join(OUT, f"{name}.npz"))
    vol, imgs = z["map"], z["images"]
    N = vol.shape[0]
    pixel = float(z["pixel"])
    with tempfile.TemporaryDirectory() as td:
        mapf = os.path.join(td, "ref.mrc")
        stackf = os.path.join(td, "parts.mrcs")
        mrc.write_stack(mapf, vol, pixel, origin_pixels=(N // 2, N // 2, N // 2), volume=True)
        mrc.write_stack(stackf, imgs, pixel)
        np.savetxt(os.path.join(td, "start.txt"), z["start"], fmt="%.17g")
        np.savetxt(os.path.join(td, "ctf.txt"), z["ctf_rows"], fmt="%.17g")
        args = [os.path.join(REF, "refine_probe"), mapf, stackf, repr(pixel), repr(case["hi_res"]),
                os.path.join(td, "start.txt"), os.path.join(td, "ctf.txt"), repr(case["alpha"]),
                repr(case["accuracy"]), repr(case["shift_step"]), repr(case["shift_accuracy"]), "0",
                repr(float(z["def_std"])), str(fom_type), "0", "1"]
        r = subprocess.run(args, capture_output=True, text=True, check=True, timeout=3600)
    out = np.array([[float(t) for t in line.split()] for line in r.stdout.splitlines() if line.strip()])
    assert out.shape == (len(imgs), 10), out.shape
    return out


def program(name: str, fomtype: str) -> np.ndarray:
    """The compiled brefine on the project test_cli writes; rows: view x, y,
    z, angle (radians), origin x, y, defocus, fom, cv."""
    from tests.test_cli import _write_refine_project
    d = load(name)
    with tempfile.TemporaryDirectory() as td:
        star = _write_refine_project(d, td)
        out = os.path.join(td, "out.star")
        args = [os.path.join(REF, "brefine"), "-reference", os.path.join(td, "ref.mrc"),
                "-grid", f"{round(d['alpha'] * 180 / math.pi, 6)},{round(d['accuracy'] * 180 / math.pi, 6)}",
                "-step", f"{d['shift_step']},{d['shift_accuracy']}", "-resolution", repr(d["hi_res"]),
                "-fomtype", fomtype, "-output", out, star]
        if d["def_std"] > 0:
            args[1:1] = ["-defocus", repr(d["def_std"])]
        subprocess.run(args, capture_output=True, text=True, check=True, timeout=3600, cwd=td,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
        proj = read_project(out)
        foms = _star_column(out, "particle.fom"), _star_column(out, "particle.fom_crossvalidation")
    rows = []
    for mg in proj.micrographs:
        rows.append([*mg.view[0], *mg.origin[0, :2], mg.defocus[0]])
    return np.column_stack([np.array(rows), foms[0], foms[1]])


def _star_column(path: str, tag: str) -> np.ndarray:
    """Values of a loop column over all blocks, in order."""
    from bsoft_b200.io.star import read_star
    vals = []
    for b in read_star(path):
        for lp in b.loops:
            if lp.index(tag) >= 0:
                vals.extend(float(v) for v in lp.column(tag))
    return np.array(vals)


if __name__ == "__main__":
    for exe in ("refine_probe", "brefine"):
        if not os.path.exists(os.path.join(REF, exe)):
            sys.exit("build the reference first: make -C oracle ref")
    res = {}
    for name, case in CASES.items():
        res[name + "_frc"] = probe(name, case, 0)
        res[name + "_dpr"] = probe(name, case, 1)
        for fomtype in ("frc", "dpr"):
            res[f"{name}_brefine_{fomtype}"] = program(name, fomtype)
    path = os.path.join(OUT, "refine_ccurve.npz")
    np.savez_compressed(path, **res)
    print(path)
