"""Generate the golden fixture of the projection-matching path from the
reference's own library code.

``match_probe`` (oracle/ref_harness/match_probe.cpp, built by
``make -C oracle ref``) runs Bsoft's brefine steps on a seeded synthetic
case: the reference-map preparation, central sections through
``Bimage::central_section`` with the default FSI kernel (8, 2), the particle
preparation, and ``img_recip_space_fom`` for a list of (image, view, origin)
hypotheses with and without the CTF.

    python tests/golden/make_match_golden.py

``project_probe`` adds Bimage::project of the map for the same views.
``views_probe`` lists the views of ``asymmetric_unit_views`` for a few point
groups and steps (views.npz).

The fixture keeps the inputs (map, images, views, CTF rows, hypotheses, and
the stack header's average and standard deviation, which the reference's
particle normalisation uses) and
the reference's outputs, so the oracle and the CUDA path are checked
against them without the reference present.
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
from bsoft_b200.synth import DatasetSpec, generate, phantom_volume  # noqa: E402
from bsoft_b200.geometry import random_views  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # 64^3 map cut to 42^3 (5 angstrom at 1.5 angstrom/pixel), astigmatic CTFs
    "match64": dict(spec=DatasetSpec(box=64, n_particles=6, n_blobs=16, pixel=1.5, snr=0.5, ctf=True, seed=31,
                                     defocus_range=(9000.0, 20000.0), astig_range=(0.0, 500.0),
                                     shift_range=1.5),
                    hi_res=5.0, n_random_views=6, ctf_apply=[1, 1, 1, 1, 0, 0]),
    # 32^3 at a coarser limit: a deeper cut (32 -> 20)
    "match32": dict(spec=DatasetSpec(box=32, n_particles=4, n_blobs=8, pixel=2.0, snr=1.0, ctf=True, seed=32,
                                     defocus_range=(8000.0, 15000.0), astig_range=(0.0, 0.0), shift_range=1.0),
                    hi_res=7.0, n_random_views=4, ctf_apply=[1, 0, 1, 0]),
}


def make(name: str, case: dict) -> str:
    spec = case["spec"]
    ph, imgs, meta = generate(spec)
    vol = phantom_volume(ph).astype(np.float32)
    N = spec.box
    rng = np.random.default_rng(spec.seed + 1000)
    views = np.concatenate([meta["views"], random_views(rng, case["n_random_views"])], axis=0)
    nimg = spec.n_particles
    ctf_rows = np.array([[spec.volt, *meta["coefs"][i][:5], case["ctf_apply"][i]] for i in range(nimg)])
    hyps = []
    for i in range(nimg):
        ox, oy = meta["origins"][i][:2]
        hyps.append([i, i, ox, oy])
        hyps.append([i, i, ox + 0.5, oy - 0.3])
        hyps.append([i, i, N / 2, N / 2])
        for r in range(2):
            hyps.append([i, nimg + (i + r) % case["n_random_views"], ox, oy])
    hyps = np.array(hyps, dtype=np.float64)
    with tempfile.TemporaryDirectory() as td:
        mapf = os.path.join(td, "ref.mrc")
        stackf = os.path.join(td, "parts.mrcs")
        mrc.write_stack(mapf, vol, spec.pixel, origin_pixels=(N // 2, N // 2, N // 2), volume=True)
        mrc.write_stack(stackf, imgs, spec.pixel)
        np.savetxt(os.path.join(td, "views.txt"), views, fmt="%.17g")
        np.savetxt(os.path.join(td, "ctf.txt"), ctf_rows, fmt="%.17g")
        np.savetxt(os.path.join(td, "hyps.txt"), hyps, fmt="%.17g")
        out = os.path.join(td, "probe")
        r = subprocess.run([os.path.join(REF, "match_probe"), mapf, stackf, repr(spec.pixel), repr(case["hi_res"]),
                            os.path.join(td, "views.txt"), os.path.join(td, "ctf.txt"),
                            os.path.join(td, "hyps.txt"), out],
                           capture_output=True, text=True, check=True)
        info = r.stdout.split()
        kv = {info[i]: info[i + 1:i + 4] for i in range(len(info)) if not _isnum(info[i])}
        diam = int(kv["diam"][0])
        map_origin = np.array([float(x) for x in kv["map_origin"][:3]])
        map_spec = np.fromfile(out + ".map", dtype=np.complex64).reshape(diam, diam, diam)
        secs = np.fromfile(out + ".sec", dtype=np.complex64).reshape(len(views), diam, diam)
        prep = np.fromfile(out + ".img", dtype=np.complex64).reshape(nimg, diam, diam)
        fom = np.loadtxt(out + ".fom").reshape(-1, 2)
        # Bimage::project of the same map for the same views (project_probe)
        pres = spec.pixel * 2.0
        rp = subprocess.run([os.path.join(REF, "project_probe"), mapf, repr(pres), os.path.join(td, "views.txt"),
                             out + ".proj"], capture_output=True, text=True, check=True)
        proj = np.fromfile(out + ".proj", dtype=np.float32).reshape(len(views), N, N)
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(path, map=vol, images=imgs, pixel=spec.pixel, hi_res=case["hi_res"], views=views,
                        ctf_rows=ctf_rows, hyps=hyps, diam=diam, map_origin=map_origin,
                        true_views=meta["views"], true_origins=meta["origins"],
                        map_spec=map_spec, sections=secs, prepared=prep, fom=fom,
                        file_avg=float(imgs.mean()), file_std=float(imgs.std()),
                        proj=proj, proj_res=pres,
                        probe_stdout=r.stdout)
    return path


def _isnum(t: str) -> bool:
    try:
        float(t)
        return True
    except ValueError:
        return False


# asymmetric_unit_views (views_probe): point group, theta and phi steps in
# degrees, flag (1 full sphere, 2 no in-plane angle)
VIEW_CASES = [("C1", 3.0, 3.0, 1), ("C1", 7.5, 7.5, 1), ("C1", 10.0, 5.0, 0), ("C3", 6.0, 6.0, 1),
              ("C1", 3.0, 3.0, 3), ("D2", 5.0, 5.0, 1), ("D3", 4.0, 4.0, 0), ("D7", 6.0, 3.0, 1),
              ("T", 3.0, 4.0, 0), ("T", 2.0, 2.0, 1), ("O", 4.0, 4.0, 1), ("O", 3.0, 3.0, 0),
              ("I", 3.0, 3.0, 1), ("I", 2.0, 2.0, 0), ("I90", 3.0, 3.0, 1), ("I90", 2.5, 2.5, 0)]


def make_views() -> str:
    out = {}
    for sym, t, p, f in VIEW_CASES:
        r = subprocess.run([os.path.join(REF, "views_probe"), sym, repr(t), repr(p), str(f)],
                           capture_output=True, text=True, check=True)
        out[f"{sym}_{t}_{p}_{f}"] = np.loadtxt(r.stdout.splitlines()).reshape(-1, 4)
    path = os.path.join(OUT, "views.npz")
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF, "match_probe")):
        sys.exit("build the reference first: make -C oracle ref")
    if sys.argv[1:] != ["views"]:          # "views": only the view lists
        for name, case in CASES.items():
            print(make(name, case))
    print(make_views())
