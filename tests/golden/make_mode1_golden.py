"""Golden maps of breconstruct with symmetry after reconstruction
(-symmetry X -mode 1: particles inserted once, the finished real-space map
symmetrized by Bimage::symmetrize, bsoft/src/breconstruct.cpp:335), with
-rescale and with -ewald, from the reference compiled from its sources, on the golden
datasets.  mode1.npz
keeps, per case, the dataset name, the options and the map.

    python tests/golden/make_mode1_golden.py
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
    ("plain24_tri_d2_m1", "plain24", "-interp trilinear -symmetry D2 -mode 1"),
    ("ctf16_tri_flip_c3_m1", "ctf16", "-interp trilinear -CTF flip -symmetry C3 -mode 1"),
    ("plain24_near_t_m1", "plain24", "-interp nearest -symmetry T -mode 1"),
    ("plain24_tri_i_m1", "plain24", "-interp trilinear -symmetry I -mode 1"),
    # -rescale avg,std of the finished map (Bimage::rescale_to_avg_std, breconstruct.cpp:336)
    ("ctf16_tri_flip_rs", "ctf16", "-interp trilinear -CTF flip -rescale 0.5,2.0"),
    ("plain24_tri_d2_m1_rs", "plain24", "-interp trilinear -symmetry D2 -mode 1 -rescale -0.1,5.2"),
    # Ewald-sphere insertion (-ewald: both surfaces s_z = +-(lambda/2) s^2,
    # Bimage_reconstruct.cpp:157-168, mg_reconstruct.cpp:209-210)
    ("ctf16_tri_flip_ew", "ctf16", "-interp trilinear -CTF flip -ewald"),
    ("ctf16_near_apply_ew", "ctf16", "-interp nearest -CTF apply -ewald"),
    ("ctf16_tri_flip_d3_ew", "ctf16", "-interp trilinear -CTF flip -symmetry D3 -ewald"),
]

if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF, "breconstruct")):
        sys.exit("build the reference first: make -C oracle ref")
    res = {}
    for name, ds, opts in CASES:
        with tempfile.TemporaryDirectory() as d:
            materialize_dataset(ds, d)
            subprocess.run(f"{REF}/breconstruct {opts} -threads 2 -recon ref.mrc particles.star", cwd=d, shell=True,
                           check=True, capture_output=True, env=dict(os.environ, OMP_NUM_THREADS="2"))
            res[name + "__map"] = mrc.read_volume(os.path.join(d, "ref.mrc"))[0]
            res[name + "__dataset"] = np.array(ds)
            res[name + "__options"] = np.array(opts)
    path = os.path.join(OUT, "mode1.npz")
    np.savez_compressed(path, **res)
    print(path)
