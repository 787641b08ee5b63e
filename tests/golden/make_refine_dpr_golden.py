"""Golden results of brefine's grid refinement with the DPR figure of merit
(brefine -fomtype dpr), from the reference's own library code.

``refine_probe`` (oracle/ref_harness/refine_probe.cpp, built by
``make -C oracle ref``) runs ``img_refine_grid``
(bsoft/src/mg/mg_refine.cpp:1086-1195) with fom_type 1 on the inputs of the
grid-refinement fixtures (refine64, refine32, refine64ctf: map, particle
stack, start records, CTF rows, steps).  The refined view, origin, figure of
merit, cross-validation figure, hypothesis count and defocus of each
particle go to refine_dpr.npz, one array per fixture.

    python tests/golden/make_refine_dpr_golden.py
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


def run(name: str, case: dict) -> np.ndarray:
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
                repr(float(z["def_std"])), "1"]
        r = subprocess.run(args, capture_output=True, text=True, check=True, timeout=3600)
    out = np.array([[float(t) for t in line.split()] for line in r.stdout.splitlines() if line.strip()])
    assert out.shape == (len(imgs), 10), out.shape
    return out


if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF, "refine_probe")):
        sys.exit("build the reference first: make -C oracle ref")
    res = {name: run(name, case) for name, case in CASES.items()}
    path = os.path.join(OUT, "refine_dpr.npz")
    np.savez_compressed(path, **res)
    print(path)
