"""Generate the golden fixture of the Fourier shell correlation from the
reference's own code.

``fsc_probe`` (oracle/ref_harness/fsc_probe.cpp, built by
``make -C oracle ref``) transforms two maps with Bimage::fft and calls
Bimage::fsc(Bimage*), as bresolve does for complex input, on two seeded
noisy copies of a blob phantom (32^3, 2 angstrom/voxel) at two resolution
limits:

    python tests/golden/make_fsc_golden.py
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
from bsoft_b200.synth import phantom_volume, random_phantom  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))


def main() -> str:
    rng = np.random.default_rng(41)
    N, u = 32, 2.0
    vol = phantom_volume(random_phantom(rng, N, 10))
    s = vol.std()
    m1 = (vol + 0.5 * s * rng.normal(size=vol.shape)).astype(np.float32)
    m2 = (vol + 0.5 * s * rng.normal(size=vol.shape)).astype(np.float32)
    out = {"map1": m1, "map2": m2, "sampling": u}
    with tempfile.TemporaryDirectory() as td:
        mrc.write_stack(os.path.join(td, "a.mrc"), m1, u, volume=True)
        mrc.write_stack(os.path.join(td, "b.mrc"), m2, u, volume=True)
        for key, res in (("res5", 5.0), ("res3", 3.0)):
            r = subprocess.run([os.path.join(REF, "fsc_probe"), os.path.join(td, "a.mrc"), os.path.join(td, "b.mrc"),
                                repr(res)], capture_output=True, text=True, check=True)
            out[key] = np.array([[float(x) for x in line.split()] for line in r.stdout.splitlines()])
    path = os.path.join(OUT, "fsc32.npz")
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF, "fsc_probe")):
        sys.exit("build the reference first: make -C oracle ref")
    print(main())
