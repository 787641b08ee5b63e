"""Golden results of brefine's grid refinement with the magnification search
(brefine -magnification: img_refine_grid's second stage over a 21 x 21 grid of
per-axis pixel-size factors 1 - m .. 1 + m in steps of m / 10, each fitted by
img_fit_in_recip_space_grid with shift steps 0.4 -> 0.1; bsoft/src/mg/
mg_refine.cpp:1151-1187), from the reference's own library code.

``refine_probe`` (oracle/ref_harness/refine_probe.cpp, built by
``make -C oracle ref``) runs ``img_refine_grid`` with max_mag > 0 on the
inputs of the grid-refinement fixtures (refine32, refine64, refine64ctf) and
prints, besides view, origin, figure of merit, cross-validation figure,
hypothesis count and defocus, the refined sampling of the cut transform.
refine_mag.npz keeps, per fixture, the max_mag, the probe's (particles, 12)
array with img_recip_space_fom's unit shell weights (``<case>``) and with
brefine's C_curve weights (``<case>_ccurve``), and the compiled ``brefine``
program's own results on a STAR project of the same particles
(``<case>_brefine``: view x, y, z, angle, origin x, y, defocus, fom, cv,
pixel size x, y, read back from its output project).

    python tests/golden/make_refine_mag_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from bsoft_b200.io import mrc  # noqa: E402
from make_refine_golden import CASES  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))
MAX_MAG = {"refine32": 0.05, "refine64": 0.03, "refine64ctf": 0.02}


def run(name: str, case: dict, max_mag: float, c_curve: int = 0) -> np.ndarray:
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
                repr(float(z["def_std"])), "0", repr(max_mag), str(c_curve)]
        r = subprocess.run(args, capture_output=True, text=True, check=True, timeout=3600)
    out = np.array([[float(t) for t in line.split()] for line in r.stdout.splitlines() if line.strip()])
    assert out.shape == (len(imgs), 12), out.shape
    return out


if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF, "refine_probe")):
        sys.exit("build the reference first: make -C oracle ref")
    from make_refine_ccurve_golden import _star_column
    from bsoft_b200.project import read_project
    from tests.refine_helpers import load
    from tests.test_cli import _write_refine_project
    import math

    def program(name: str, max_mag: float) -> np.ndarray:
        d = load(name)
        with tempfile.TemporaryDirectory() as td:
            star = _write_refine_project(d, td)
            out = os.path.join(td, "out.star")
            args = [os.path.join(REF, "brefine"), "-reference", os.path.join(td, "ref.mrc"),
                    "-grid", f"{round(d['alpha'] * 180 / math.pi, 6)},{round(d['accuracy'] * 180 / math.pi, 6)}",
                    "-step", f"{d['shift_step']},{d['shift_accuracy']}", "-resolution", repr(d["hi_res"]),
                    "-magnification", repr(max_mag), "-output", out, star]
            if d["def_std"] > 0:
                args[1:1] = ["-defocus", repr(d["def_std"])]
            subprocess.run(args, capture_output=True, text=True, check=True, timeout=7200, cwd=td,
                           env=dict(os.environ, OMP_NUM_THREADS="4"))
            proj = read_project(out)
            cols = [_star_column(out, t) for t in ("particle.fom", "particle.fom_crossvalidation",
                                                  "particle.pixel_size_x", "particle.pixel_size_y")]
        rows = [[*mg.view[0], *mg.origin[0, :2], mg.defocus[0]] for mg in proj.micrographs]
        return np.column_stack([np.array(rows), *cols])

    res = {}
    for name, case in CASES.items():
        res[name] = run(name, case, MAX_MAG[name])
        res[name + "_ccurve"] = run(name, case, MAX_MAG[name], 1)
        res[name + "_brefine"] = program(name, MAX_MAG[name])
        res[name + "_max_mag"] = np.array(MAX_MAG[name])
    path = os.path.join(OUT, "refine_mag.npz")
    np.savez_compressed(path, **res)
    print(path)
