"""Generate the golden fixture of brefine's grid refinement from the
reference's own library code.

``refine_probe`` (oracle/ref_harness/refine_probe.cpp, built by
``make -C oracle ref``) prepares the map and each particle as
project_refine_orientations / part_refine_orientation do and runs
``img_refine_grid`` (bsoft/src/mg/mg_refine.cpp:1086-1195) from a start
view and origin: without CTF, or with the CTF and the defocus search that
brefine -defocus turns on (the only way its grid refinement applies a CTF).
Defocus starts are the true defoci perturbed by a few hundred angstrom.

    python tests/golden/make_refine_golden.py

Start poses are the true poses of the synthetic particles perturbed by a
few degrees and a fraction of a pixel.  The fixture keeps the inputs (map,
images, the stack header's average and standard deviation, start records,
steps in radians as the probe computes them) and the reference's refined
view, origin, figure of merit, cross-validation figure and hypothesis count.
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

from bsoft_b200.ctf import electron_wavelength  # noqa: E402
from bsoft_b200.io import mrc  # noqa: E402
from bsoft_b200.synth import DatasetSpec, generate, phantom_volume  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # 64^2 particles, 64^3 map cut to 42^3; steps 2 deg -> 0.5 deg, 0.4 -> 0.1 px
    "refine64": dict(spec=DatasetSpec(box=64, n_particles=6, n_blobs=16, pixel=1.5, snr=1.0, ctf=False, seed=51,
                                      shift_range=1.5),
                     hi_res=5.0, alpha=2.0, accuracy=0.5, shift_step=0.4, shift_accuracy=0.1,
                     view_noise=0.04, angle_noise=0.04, origin_noise=0.4),
    # 32^2 particles cut to 20; coarser steps whose origin loops are ragged
    "refine32": dict(spec=DatasetSpec(box=32, n_particles=4, n_blobs=8, pixel=2.0, snr=2.0, ctf=False, seed=52,
                                      shift_range=1.0),
                     hi_res=7.0, alpha=3.0, accuracy=0.7, shift_step=0.3, shift_accuracy=0.07,
                     view_noise=0.05, angle_noise=0.05, origin_noise=0.3),
    # CTF-modulated particles, defocus search of +-5 x 300 angstrom
    "refine64ctf": dict(spec=DatasetSpec(box=64, n_particles=5, n_blobs=16, pixel=1.5, snr=1.0, ctf=True, seed=53,
                                         defocus_range=(9000.0, 20000.0), astig_range=(0.0, 300.0),
                                         shift_range=1.5),
                        hi_res=5.0, alpha=2.0, accuracy=0.5, shift_step=0.4, shift_accuracy=0.1,
                        view_noise=0.04, angle_noise=0.04, origin_noise=0.4, def_std=300.0, def_noise=700.0),
}


def make(name: str, case: dict) -> str:
    spec = case["spec"]
    ph, imgs, meta = generate(spec)
    vol = phantom_volume(ph).astype(np.float32)
    N = spec.box
    rng = np.random.default_rng(spec.seed + 2000)
    nimg = spec.n_particles
    start = np.zeros((nimg, 6))
    for i in range(nimg):
        v = np.asarray(meta["views"][i], dtype=np.float64)
        start[i, :3] = v[:3] + rng.normal(0, case["view_noise"], 3)
        start[i, 3] = v[3] + rng.normal(0, case["angle_noise"])
        start[i, 4:6] = np.asarray(meta["origins"][i][:2]) + rng.uniform(-1, 1, 2) * case["origin_noise"]
    def_std = case.get("def_std", 0.0)
    if def_std > 0:
        t2 = -math.pi * electron_wavelength(spec.volt)
        ctf_rows = np.array([[spec.volt, *meta["coefs"][i][:5], 1] for i in range(nimg)], dtype=np.float64)
        ctf_rows[:, 2] += t2 * rng.uniform(-1, 1, nimg) * case["def_noise"]
    else:
        ctf_rows = np.array([[spec.volt, 0, 0, 0, 0, 0, 0]] * nimg, dtype=np.float64)
    with tempfile.TemporaryDirectory() as td:
        mapf = os.path.join(td, "ref.mrc")
        stackf = os.path.join(td, "parts.mrcs")
        mrc.write_stack(mapf, vol, spec.pixel, origin_pixels=(N // 2, N // 2, N // 2), volume=True)
        mrc.write_stack(stackf, imgs, spec.pixel)
        np.savetxt(os.path.join(td, "start.txt"), start, fmt="%.17g")
        np.savetxt(os.path.join(td, "ctf.txt"), ctf_rows, fmt="%.17g")
        args = [os.path.join(REF, "refine_probe"), mapf, stackf, repr(spec.pixel), repr(case["hi_res"]),
                os.path.join(td, "start.txt"), os.path.join(td, "ctf.txt"), repr(case["alpha"]),
                repr(case["accuracy"]), repr(case["shift_step"]), repr(case["shift_accuracy"]), "0", repr(def_std)]
        r = subprocess.run(args, capture_output=True, text=True, check=True, timeout=1800)
    out = np.array([[float(t) for t in line.split()] for line in r.stdout.splitlines() if line.strip()])
    assert out.shape == (nimg, 10), out.shape
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(path, map=vol, images=imgs, pixel=spec.pixel, hi_res=case["hi_res"],
                        file_avg=float(imgs.mean()), file_std=float(imgs.std()),
                        start=start, true_views=meta["views"], true_origins=meta["origins"],
                        # the probe's conversion: atof(deg) * M_PI / 180.0
                        alpha=case["alpha"] * math.pi / 180.0, accuracy=case["accuracy"] * math.pi / 180.0,
                        shift_step=case["shift_step"], shift_accuracy=case["shift_accuracy"],
                        ctf_rows=ctf_rows, volt=spec.volt, def_std=def_std,
                        true_coefs=meta["coefs"] if spec.ctf else np.zeros((nimg, 7)), result=out)
    return path


if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF, "refine_probe")):
        sys.exit("build the reference first: make -C oracle ref")
    for name, case in CASES.items():
        print(make(name, case))
