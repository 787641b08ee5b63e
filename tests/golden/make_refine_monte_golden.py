"""Golden results of brefine's Monte Carlo refinement (brefine -monte:
img_refine_monte with img_fit_in_recip_space_monte, bsoft/src/mg/
mg_refine.cpp:783-860, 979-1050), from the reference's own library code.

``refine_probe`` (oracle/ref_harness/refine_probe.cpp) runs img_refine_monte
with brefine's C_curve shell weights on the inputs of the grid-refinement
fixtures, with random() seeded once before the first particle (the
reference seeds it with its process id).  refine_monte.npz keeps, per
fixture, the parameters (max_iter, shift_std, view_std, max_angle in
degrees, max_mag, seed), the probe's per-particle results, and
(``<case>_brefine``) the compiled brefine program's own results on a STAR
project of the same particles with its process id pinned to the seed
(``oracle/_ref/brefine_pid``, one OpenMP thread so that the particles draw
one after another): view x, y, z, angle, origin x, y, defocus, fom, cv,
pixel size x, y.

    python tests/golden/make_refine_monte_golden.py
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
# max_iter, shift_std (cut pixels), view_std, max_angle (degrees), max_mag, seed
PARAMS = {"refine32": (12, 0.5, 0.02, 3.0, 0.0, 11),
          "refine64": (10, 0.3, 0.03, 2.0, 0.02, 12),
          "refine64ctf": (8, 0.4, 0.02, 2.0, 0.0, 13)}


def run(name: str, case: dict) -> np.ndarray:
    z = np.load(os.path.join(OUT, f"{name}.npz"))
    vol, imgs = z["map"], z["images"]
    N = vol.shape[0]
    pixel = float(z["pixel"])
    it, sh, vw, ang, mag, seed = PARAMS[name]
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
                repr(float(z["def_std"])), "0", repr(mag), "1", str(it), repr(sh), repr(vw), repr(ang), str(seed)]
        r = subprocess.run(args, capture_output=True, text=True, check=True, timeout=3600)
    out = np.array([[float(t) for t in line.split()] for line in r.stdout.splitlines() if line.strip()])
    assert out.shape[0] == len(imgs), out.shape
    return out


if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF, "refine_probe")):
        sys.exit("build the reference first: make -C oracle ref")
    import math
    from make_refine_ccurve_golden import _star_column
    from bsoft_b200.project import read_project
    from tests.refine_helpers import load
    from tests.test_cli import _write_refine_project

    def program(name: str) -> np.ndarray:
        d = load(name)
        it, sh, vw, ang, mag, seed = PARAMS[name]
        with tempfile.TemporaryDirectory() as td:
            star = _write_refine_project(d, td)
            out = os.path.join(td, "out.star")
            args = [os.path.join(REF, "brefine_pid"), "-reference", os.path.join(td, "ref.mrc"),
                    "-monte", str(it), "-shift", repr(sh), "-view", repr(vw), "-angle", repr(ang),
                    "-resolution", repr(d["hi_res"]), "-output", out, star]
            if mag > 0:
                args[1:1] = ["-magnification", repr(mag)]
            if d["def_std"] > 0:
                args[1:1] = ["-defocus", repr(d["def_std"])]
            subprocess.run(args, capture_output=True, text=True, check=True, timeout=3600, cwd=td,
                           env=dict(os.environ, OMP_NUM_THREADS="1", BSG_REF_PID=str(seed)))
            proj = read_project(out)
            cols = [_star_column(out, t) for t in ("particle.fom", "particle.fom_crossvalidation",
                                                  "particle.pixel_size_x", "particle.pixel_size_y")]
        rows = [[*mg.view[0], *mg.origin[0, :2], mg.defocus[0]] for mg in proj.micrographs]
        return np.column_stack([np.array(rows), *cols])

    res = {}
    for name, case in CASES.items():
        res[name] = run(name, case)
        res[name + "_params"] = np.array(PARAMS[name], dtype=np.float64)
        res[name + "_brefine"] = program(name)
    path = os.path.join(OUT, "refine_monte.npz")
    np.savez_compressed(path, **res)
    print(path)
