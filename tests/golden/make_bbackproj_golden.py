"""Golden maps of the reference's bbackproj (real-space weighted
back-projection of a STAR project: project_back_projection over
Bimage::back_project, img_backprojection_accumulate, then -symmetry and
-rescale; bsoft/src/bbackproj.cpp:170-207), from the reference compiled from
its sources (oracle/_ref/bbackproj), on the golden datasets.  bbackproj.npz
keeps, per case, the dataset name, the options and the map(s).

    python tests/golden/make_bbackproj_golden.py
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

CASES = [
    ("ctf16_bp", "ctf16", "-resolution 5"),
    ("plain24_bp", "plain24", "-resolution 4"),
    ("plain24_bp_half", "plain24", "-resolution 6 -halfmaps -threads 2"),
    ("plain24_bp_full_half", "plain24", "-resolution 6 -fullmap -halfmaps -threads 4"),
    ("plain24_bp_d2", "plain24", "-resolution 6 -symmetry D2"),
    ("ctf16_bp_rs", "ctf16", "-resolution 5 -rescale 0.5,2"),
]


def main():
    if not os.path.exists(os.path.join(REF, "bbackproj")):
        sys.exit("build the reference first: make -C oracle ref")
    res = {}
    for name, ds, opts in CASES:
        with tempfile.TemporaryDirectory() as d:
            materialize_dataset(ds, d)
            subprocess.run(f"{REF}/bbackproj {opts} -recon ref.mrc particles.star", cwd=d, shell=True,
                           check=True, capture_output=True, env=dict(os.environ, OMP_NUM_THREADS="2"))
            for f in sorted(os.listdir(d)):
                if f.startswith("ref") and f.endswith(".mrc"):
                    tag = "map" if f == "ref.mrc" else "map" + f[3:-4]
                    res[f"{name}__{tag}"] = mrc.read_volume(os.path.join(d, f))[0]
            res[name + "__dataset"] = np.array(ds)
            res[name + "__options"] = np.array(opts)
    path = os.path.join(OUT, "bbackproj.npz")
    np.savez_compressed(path, **res)
    print(path, sorted(k for k in res if "__map" in k))


if __name__ == "__main__":
    main()
