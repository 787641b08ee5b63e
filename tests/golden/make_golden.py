"""Generate the golden fixtures of the reconstruction path from the
reference's own programs.

The fixtures pin the CPU oracle (oracle/) and the CUDA path to Bsoft's
``breconstruct`` compiled from its sources (``make -C oracle ref``), run on
small seeded synthetic datasets:

    python tests/golden/make_golden.py

Each fixture stores the particle images, the STAR project text, the exact
command-line options and the reference's output map(s).  ``recon_probe``
(oracle/ref_harness) adds per-stage dumps of single particles: padded FFT,
origin shift, CTF, and that particle's inserted volume.
"""
from __future__ import annotations

import os
import shlex
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from bsoft_b200.io import mrc  # noqa: E402
from bsoft_b200.synth import DatasetSpec, generate, write_dataset  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))

DATASETS = {
    # 4 micrographs, per-micrograph astigmatism, CTF, noise
    "ctf16": DatasetSpec(box=16, n_particles=64, n_blobs=8, pixel=2.0, snr=0.5, ctf=True, seed=11,
                         defocus_range=(8000.0, 20000.0), astig_range=(0.0, 400.0), shift_range=1.5,
                         mean_per_micrograph=16),
    # no CTF, larger box
    "plain24": DatasetSpec(box=24, n_particles=48, n_blobs=10, pixel=1.5, snr=1.0, ctf=False, seed=12,
                           shift_range=2.0),
}

# (fixture name, dataset, breconstruct options, outputs)
CASES = [
    ("ctf16_tri_none", "ctf16", "-interp trilinear", None),
    ("ctf16_tri_flip", "ctf16", "-interp trilinear -CTF flip", None),
    ("ctf16_near_apply", "ctf16", "-interp nearest -CTF apply", None),
    ("ctf16_wtd_correct", "ctf16", "-interp weighted -CTF correct", None),
    ("ctf16_tri_flip_res", "ctf16", "-interp trilinear -CTF flip -resolution 5", None),
    ("ctf16_tri_flip_half", "ctf16", "-interp trilinear -CTF flip -halfmaps", ("_01", "_02")),
    ("plain24_tri", "plain24", "-interp trilinear", None),
    ("plain24_near", "plain24", "-interp nearest", None),
    # point-group symmetry inserted during reconstruction (-symmetry, mode 0)
    ("ctf16_tri_flip_d3", "ctf16", "-interp trilinear -CTF flip -symmetry D3", None),
    ("plain24_tri_t", "plain24", "-interp trilinear -symmetry T", None),
    ("plain24_near_c4", "plain24", "-interp nearest -symmetry C4", None),
]

PROBES = [("ctf16", 0, 2, 1), ("ctf16", 37, 2, 1)]


def run(cmd, cwd):
    env = dict(os.environ, OMP_NUM_THREADS="2")
    subprocess.run(cmd, cwd=cwd, shell=True, check=True, env=env,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)


def main():
    """All fixtures, or only the cases named on the command line (then the
    dataset fixtures and the probes are left as they are)."""
    if not os.path.exists(os.path.join(REF, "breconstruct")):
        sys.exit("build the reference first: make -C oracle ref")
    only = set(sys.argv[1:])
    tmp = tempfile.mkdtemp(prefix="golden_")
    data = {}
    for name, spec in DATASETS.items():
        d = os.path.join(tmp, name)
        ph, imgs, meta = generate(spec)
        star = write_dataset(d, spec, ph, imgs, meta)
        with open(star) as f:
            star_text = f.read()
        stacks = {fn: mrc.read_stack(os.path.join(d, fn))[0] for fn in sorted(os.listdir(d)) if fn.endswith(".mrcs")}
        data[name] = (d, star_text, stacks)
        if only:
            continue
        np.savez_compressed(os.path.join(OUT, f"ds_{name}.npz"), star=np.array(star_text),
                            stack_names=np.array(list(stacks)), **{"stack_" + k: v for k, v in stacks.items()})
    for fname, ds, opts, suffixes in CASES:
        if only and fname not in only:
            continue
        d, star_text, stacks = data[ds]
        run(f"{REF}/breconstruct {opts} -threads 2 -recon ref.mrc particles.star", d)
        outs = {}
        for suf in (suffixes or ("",)):
            vol, _ = mrc.read_volume(os.path.join(d, f"ref{suf}.mrc"))
            outs["map" + suf] = vol
            os.remove(os.path.join(d, f"ref{suf}.mrc"))
        np.savez_compressed(os.path.join(OUT, fname + ".npz"), dataset=np.array(ds), options=np.array(opts),
                            **outs)
        print("wrote", fname, list(outs))
    for ds, idx, interp, ctf in ([] if only else PROBES):
        d, star_text, stacks = data[ds]
        run(f"{REF}/recon_probe particles.star {idx} {interp} {ctf} probe", d)
        ft = int(np.sqrt(os.path.getsize(os.path.join(d, "probe.fft")) // 8))
        rd = lambda ext, dt=np.float32: np.fromfile(os.path.join(d, "probe" + ext), dtype=dt)
        np.savez_compressed(os.path.join(OUT, f"probe_{ds}_{idx}.npz"), dataset=np.array(ds), index=idx, interp=interp, ctf_action=ctf, bkg=rd(".bkg", np.float64),
                            fft=rd(".fft").reshape(ft, ft, 2), shift=rd(".shift").reshape(ft, ft, 2),
                            ctf=rd(".ctf").reshape(ft, ft, 2), vol=rd(".vol"), w=rd(".w"))
        print("wrote probe", ds, idx)
    print("command lines:", " | ".join(shlex.quote(c[2]) for c in CASES))


if __name__ == "__main__":
    main()
