"""Per-stage CPU time of the reference's reconstruction loop on the insertion
benchmark's particles (256^2 -> 256^3, pad 2, trilinear, CTF flip), so the
reference's FFT share is reported apart from its insertion (gridding) share.

Measurement infrastructure only: it writes the first `count` particles of
the benchmark workload as MRC + STAR (bench.reference_project) and runs
oracle/_ref/stage_probe, the reference's own per-particle calls of
particle_reconstruct (bsoft/src/mg/mg_reconstruct.cpp:143-229) timed one by
one on one thread.  The FFT is the reference's fft() over the project's
FFTW3-API stand-in (oracle/fftw3_standin), not FFTW.

    python -m oracle.ref_stage_times [count]      (prints one JSON line)
"""
from __future__ import annotations

import json
import os
import subprocess
import sys


def main(count: int = 16) -> dict:
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    import bench
    exe = os.path.join(here, "_ref", "stage_probe")
    if not os.path.exists(exe):
        raise SystemExit("oracle/_ref/stage_probe is not built (make -C oracle ref)")
    w = bench.make_workload(max(count, 2))
    d = bench.reference_project(w, count)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run([exe, os.path.join(d, "p.star"), str(count)], cwd=d, env=env, capture_output=True,
                       text=True, check=True)
    vals = {}
    for line in r.stdout.splitlines():
        k, v = line.split()
        vals[k] = float(v)
    n = int(vals.pop("particles"))
    ft = int(vals.pop("ft"))
    total = sum(vals.values())
    out = {"particles": n, "ft": ft, "threads": 1,
           "ms_per_particle": {k: round(1e3 * v / n, 3) for k, v in vals.items()},
           "share": {k: round(v / total, 4) for k, v in vals.items()},
           "total_ms_per_particle": round(1e3 * total / n, 3)}
    return out


if __name__ == "__main__":
    print(json.dumps(main(int(sys.argv[1]) if len(sys.argv) > 1 else 16)))
