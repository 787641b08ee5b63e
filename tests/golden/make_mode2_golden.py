"""Golden data of breconstruct -mode 2 (each particle inserted once, with a
random one of its symmetry-related views: random_symmetric_view,
bsoft/src/util/symmetry.cpp:816-832, mg_reconstruct.cpp:175).

* views: for 40 seeded views and several point groups, the view the
  reference's random_symmetric_view returns after srandom(seed)
  (oracle/_ref/symview_probe);
* maps: the reference's breconstruct maps with its process id pinned to the
  seed (oracle/_ref/breconstruct_pid, getpid() wrapped) and its OpenMP loop on
  one thread, so that the partial maps draw one after another.

mode2.npz keeps, per case, the dataset, options, seed and map, and per point
group the input views, the seed and the picked views.

    python tests/golden/make_mode2_golden.py
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

VIEW_CASES = [("D3", 12345), ("C5", 7), ("T", 99), ("O", 2024), ("I", 31337)]
MAP_CASES = [
    ("ctf16_tri_flip_d3_m2", "ctf16", "-interp trilinear -CTF flip -symmetry D3 -mode 2 -threads 2", 4242),
    ("plain24_tri_i_m2", "plain24", "-interp trilinear -symmetry I -mode 2 -threads 3", 17),
    ("plain24_near_t_m2_half", "plain24", "-interp nearest -symmetry T -mode 2 -threads 3 -halfmaps", 5),
]


def main():
    for exe in ("symview_probe", "breconstruct_pid"):
        if not os.path.exists(os.path.join(REF, exe)):
            sys.exit("build the reference first: make -C oracle ref")
    rng = np.random.default_rng(2718)
    res = {}
    v = rng.normal(size=(40, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    views = np.concatenate([v, rng.uniform(-np.pi, np.pi, size=(40, 1))], axis=1)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "views.txt")
        np.savetxt(path, views, fmt="%.17g")
        for sym, seed in VIEW_CASES:
            out = subprocess.run([os.path.join(REF, "symview_probe"), sym, str(seed), path], check=True,
                                 capture_output=True, text=True).stdout
            res[f"views_{sym}__in"] = views
            res[f"views_{sym}__seed"] = np.array(seed)
            res[f"views_{sym}__out"] = np.array([[float(x) for x in ln.split()] for ln in out.splitlines()])
    for name, ds, opts, seed in MAP_CASES:
        with tempfile.TemporaryDirectory() as d:
            materialize_dataset(ds, d)
            subprocess.run(f"{REF}/breconstruct_pid {opts} -recon ref.mrc particles.star", cwd=d, shell=True,
                           check=True, capture_output=True,
                           env=dict(os.environ, OMP_NUM_THREADS="1", BSG_REF_PID=str(seed)))
            maps = {}
            for f in sorted(os.listdir(d)):
                if f.startswith("ref") and f.endswith(".mrc"):
                    maps[f] = mrc.read_volume(os.path.join(d, f))[0]
            for f, m in maps.items():
                tag = "map" if f == "ref.mrc" else "map" + f[3:-4]
                res[f"{name}__{tag}"] = m
            res[name + "__dataset"] = np.array(ds)
            res[name + "__options"] = np.array(opts)
            res[name + "__seed"] = np.array(seed)
    path = os.path.join(OUT, "mode2.npz")
    np.savez_compressed(path, **res)
    print(path, sorted(res))


if __name__ == "__main__":
    main()
