"""Generate the golden fixture of img_recip_space_fom's DPR form (brefine
-fomtype dpr; bsoft/src/mg/mg_refine.cpp:660-781, the phase-residual branch)
from the reference's own code.

The inputs are those of the matching fixtures (tests/golden/match32.npz,
match64.npz, made by make_match_golden.py): the map, the particle stack and
the view, CTF and hypothesis lists are written back out and
``match_probe`` (oracle/ref_harness/match_probe.cpp, built by
``make -C oracle ref``) scores every hypothesis again with
MATCH_PROBE_FOM_TYPE=1.  The fixture keeps (fom, cv) per hypothesis for
each case.

    python tests/golden/make_match_dpr_golden.py
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

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))


def main() -> None:
    exe = os.path.join(REF, "match_probe")
    if not os.path.exists(exe):
        sys.exit("build the reference harness first: make -C oracle ref")
    out = {}
    for name in ("match32", "match64"):
        z = np.load(os.path.join(OUT, name + ".npz"))
        vol, imgs, pixel = z["map"], z["images"], float(z["pixel"])
        N = vol.shape[0]
        with tempfile.TemporaryDirectory() as td:
            mapf, stackf = os.path.join(td, "ref.mrc"), os.path.join(td, "parts.mrcs")
            mrc.write_stack(mapf, vol, pixel, origin_pixels=(N // 2, N // 2, N // 2), volume=True)
            mrc.write_stack(stackf, imgs, pixel)
            for key in ("views", "ctf_rows", "hyps"):
                np.savetxt(os.path.join(td, key + ".txt"), z[key], fmt="%.17g")
            probe = os.path.join(td, "probe")
            subprocess.run([exe, mapf, stackf, repr(pixel), repr(float(z["hi_res"])),
                            os.path.join(td, "views.txt"), os.path.join(td, "ctf_rows.txt"),
                            os.path.join(td, "hyps.txt"), probe],
                           env=dict(os.environ, MATCH_PROBE_FOM_TYPE="1"), capture_output=True, text=True,
                           check=True)
            out[name] = np.loadtxt(probe + ".fom").reshape(-1, 2)
            # the FRC scores of the same run reproduce the stored ones
            subprocess.run([exe, mapf, stackf, repr(pixel), repr(float(z["hi_res"])),
                            os.path.join(td, "views.txt"), os.path.join(td, "ctf_rows.txt"),
                            os.path.join(td, "hyps.txt"), probe], capture_output=True, text=True, check=True)
            frc = np.loadtxt(probe + ".fom").reshape(-1, 2)
            if not np.array_equal(frc, z["fom"]):
                sys.exit(f"{name}: the rewritten inputs do not reproduce the stored FRC scores")
    np.savez_compressed(os.path.join(OUT, "match_dpr.npz"), **out)


if __name__ == "__main__":
    main()
