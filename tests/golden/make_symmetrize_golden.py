"""Generate the golden fixture of the reference's real-space point-group
symmetrization (Bimage::symmetrize(sym, 1), bsoft/src/img/
Bimage_symmetry.cpp:31-100; breconstruct -symmetry with sym_mode 1).

``symmetrize_probe`` (oracle/ref_harness/symmetrize_probe.cpp, built by
``make -C oracle ref``) applies the reference's own function to a raw float
map about a given origin.  Inputs: two seeded maps of blobs and noise, one
of even edge 16 about its centre and one of odd edge 15 about an off-centre
origin.  The fixture keeps each input map, its origin and the reference's
output for every group listed.

    python tests/golden/make_symmetrize_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
GROUPS = ["C3", "C4", "D2", "D5", "T", "O", "I"]
CASES = {"a": (16, (8.0, 8.0, 8.0), 11), "b": (15, (7.0, 7.5, 6.25), 12)}


def make_map(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    z, y, x = np.mgrid[:n, :n, :n].astype(np.float64)
    m = 0.2 * rng.standard_normal((n, n, n))
    for _ in range(5):
        c = rng.uniform(0.25 * n, 0.75 * n, 3)
        s = rng.uniform(1.0, 2.0)
        m += rng.uniform(0.5, 1.0) * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * s * s))
    return m.astype(np.float32)


def main() -> None:
    exe = os.path.join(ROOT, "oracle", "_ref", "symmetrize_probe")
    if not os.path.exists(exe):
        sys.exit("build the reference harness first: make -C oracle ref")
    out = {"groups": np.array(GROUPS)}
    with tempfile.TemporaryDirectory() as d:
        for key, (n, origin, seed) in CASES.items():
            m = make_map(n, seed)
            src = os.path.join(d, "in.raw")
            m.tofile(src)
            out[f"{key}_map"] = m
            out[f"{key}_origin"] = np.array(origin)
            for g in GROUPS:
                dst = os.path.join(d, "out.raw")
                subprocess.run([exe, src, str(n), *(repr(float(o)) for o in origin), g, dst], check=True,
                               capture_output=True)
                out[f"{key}_{g}"] = np.fromfile(dst, dtype=np.float32).reshape(n, n, n)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "symmetrize.npz"), **out)


if __name__ == "__main__":
    main()
