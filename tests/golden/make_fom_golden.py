"""Golden outputs of breconstruct's figure-of-merit map (-fom) and its
reconstruction statistics, from the reference compiled from its sources.

For each case the golden datasets (ds_ctf16.npz, ds_plain24.npz) are written
out and ``oracle/_ref/breconstruct -verbose 1 ... -fom fom.mrc`` is run.
Stored per case in fom_stats.npz: the map, the FOM map
(fspace_reconstruction_snr, bsoft/src/img/Bimage_reconstruct.cpp:610-634,
written in reciprocal-space order), and the text the reference prints for
the reconstruction: Friedel residual and coverage
(bsoft/src/mg/mg_reconstruct.cpp:328-349) and the shell table of
fspace_reconstruction_stats (Bimage_reconstruct.cpp:526-599).

    python tests/golden/make_fom_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from bsoft_b200.io import mrc  # noqa: E402
from tests.helpers import materialize_dataset  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))

# (case, dataset, breconstruct options, map suffixes)
CASES = [
    ("fom_ctf16_tri_flip", "ctf16", "-interp trilinear -CTF flip", ("",)),
    ("fom_plain24_tri", "plain24", "-interp trilinear", ("",)),
    ("fom_ctf16_near_apply", "ctf16", "-interp nearest -CTF apply", ("",)),
    ("fom_ctf16_tri_flip_half", "ctf16", "-interp trilinear -CTF flip -halfmaps", ("_01", "_02")),
]


def run_case(name, ds, opts, suffixes):
    with tempfile.TemporaryDirectory() as d:
        materialize_dataset(ds, d)
        cmd = f"{REF}/breconstruct -verbose 1 {opts} -threads 2 -fom fom.mrc -recon ref.mrc particles.star"
        r = subprocess.run(cmd, cwd=d, shell=True, check=True, capture_output=True, text=True,
                           env=dict(os.environ, OMP_NUM_THREADS="2"))
        out = {"options": np.array(opts), "dataset": np.array(ds), "stdout": np.array(r.stdout)}
        for suf in suffixes:
            out["map" + suf] = mrc.read_volume(os.path.join(d, f"ref{suf}.mrc"))[0]
            out["fom" + suf] = mrc.read_volume(os.path.join(d, f"fom{suf}.mrc"))[0]
        return out


if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF, "breconstruct")):
        sys.exit("build the reference first: make -C oracle ref")
    res = {}
    for name, ds, opts, suffixes in CASES:
        for k, v in run_case(name, ds, opts, suffixes).items():
            res[f"{name}__{k}"] = v
    path = os.path.join(OUT, "fom_stats.npz")
    np.savez_compressed(path, **res)
    print(path)
