"""Generate the golden fixture of the reference's real-space weighted
back-projection (bbackproj: project_back_projection over
Bimage::back_project, bsoft/src/img/Bimage_project.cpp:466-509).

``backproject_probe`` (oracle/ref_harness/backproject_probe.cpp, built by
``make -C oracle ref``) back-projects seeded images (noise plus a block) at
seeded views and origins into a map about its default origin.  Two cases:
even images into an equal map, and odd images into a larger map; the first
view of each is the untilted one.  The fixture keeps the images, their
records (ox, oy, vx, vy, vz, angle in radians), the pixel size, the
resolution and the reference's map.

    python tests/golden/make_backproject_golden.py
"""
from __future__ import annotations

import math
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
CASES = {"a": dict(n=16, N=16, K=5, pixel=1.5, res=4.0, seed=21),
         "b": dict(n=15, N=20, K=6, pixel=2.0, res=5.0, seed=22)}


def inputs(n, K, seed):
    rng = np.random.default_rng(seed)
    imgs = (0.3 * rng.standard_normal((K, n, n))).astype(np.float32)
    imgs[:, n // 3:n // 2 + 2, n // 3:n // 2 + 3] += 1.0
    params = [(n / 2, n / 2, 0.0, 0.0, 1.0, 0.0)]
    for _ in range(K - 1):
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        params.append((n // 2 + rng.uniform(-1, 1), n // 2 + rng.uniform(-1, 1), v[0], v[1], v[2],
                       rng.uniform(-math.pi, math.pi)))
    return imgs, np.array(params)


def main() -> None:
    exe = os.path.join(ROOT, "oracle", "_ref", "backproject_probe")
    if not os.path.exists(exe):
        sys.exit("build the reference harness first: make -C oracle ref")
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for key, c in CASES.items():
            imgs, params = inputs(c["n"], c["K"], c["seed"])
            src, ptxt, dst = (os.path.join(d, f) for f in ("in.raw", "params.txt", "out.raw"))
            imgs.tofile(src)
            with open(ptxt, "w") as f:
                for p in params:
                    f.write(" ".join(repr(float(x)) for x in p) + "\n")
            subprocess.run([exe, src, ptxt, str(c["K"]), str(c["n"]), repr(c["pixel"]), repr(c["res"]),
                            str(c["N"]), dst], check=True, capture_output=True)
            out[f"{key}_images"] = imgs
            out[f"{key}_params"] = params
            out[f"{key}_scalars"] = np.array([c["pixel"], c["res"], c["N"]], dtype=np.float64)
            out[f"{key}_map"] = np.fromfile(dst, dtype=np.float32).reshape(c["N"], c["N"], c["N"])
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "backproject.npz"), **out)


if __name__ == "__main__":
    main()
