"""Shared test helpers: golden-fixture loading and error metrics."""
from __future__ import annotations

import os
import shlex

import numpy as np

from bsoft_b200.io import mrc
from bsoft_b200.plan import INTERP, ReconOptions, load_images, plan_reconstruction
from bsoft_b200.project import read_project

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CASES = ["ctf16_tri_none", "ctf16_tri_flip", "ctf16_near_apply", "ctf16_wtd_correct",
         "ctf16_tri_flip_res", "ctf16_tri_flip_half", "plain24_tri", "plain24_near",
         "ctf16_tri_flip_d3", "plain24_tri_t", "plain24_near_c4"]


def ref_tol(case: str) -> float:
    """Agreement bar with the reference's map: 1e-5, or 3e-5 for the 12-fold
    tetrahedral case, where the reference's own FP32 accumulation of ~12x
    more contributions per voxel reaches ~1.3e-5 against the FP64 oracle
    (the error is largest at low resolution, where contributions pile up)."""
    return 3e-5 if case == "plain24_tri_t" else 1e-5


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    a = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
    b = b.astype(np.complex128 if np.iscomplexobj(b) else np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def materialize_dataset(name: str, directory: str) -> str:
    """Write a golden dataset's stacks and STAR file into `directory`."""
    z = np.load(os.path.join(GOLDEN, f"ds_{name}.npz"))
    for fn in z["stack_names"]:
        mrc.write_stack(os.path.join(directory, str(fn)), z["stack_" + str(fn)], pixel_size=1.0)
    # the pixel size that matters is the STAR one; rewrite headers with it
    path = os.path.join(directory, "particles.star")
    with open(path, "w") as f:
        f.write(str(z["star"]))
    proj = read_project(path)
    for mg in proj.micrographs:
        stack = z["stack_" + mg.particle_file]
        mrc.write_stack(os.path.join(directory, mg.particle_file), stack, pixel_size=float(mg.pixel[0]))
    return path


def options_from_args(args: str) -> ReconOptions:
    """Map a breconstruct option string onto ReconOptions (the subset the
    fixtures use; prefix matching as bsoft/src/util/options.cpp does)."""
    opt = ReconOptions()
    toks = shlex.split(args)
    i = 0
    while i < len(toks):
        t = toks[i].lstrip("-")
        val = toks[i + 1] if i + 1 < len(toks) and not toks[i + 1].startswith("-") else None
        if t == "rescale" and i + 1 < len(toks):        # its average may be negative
            val = toks[i + 1]
        if "interpolation".startswith(t):
            opt.interp = INTERP[{"n": "nearest", "w": "weighted", "t": "trilinear"}[val[0]]]
        elif t == "CTF":
            v = val.lower()
            opt.ctf_action = 1 if "fli" in v else 2 if "app" in v else 3 if "cor" in v else 4 if "wie" in v else 0
        elif "resolution".startswith(t):
            opt.resolution = float(val)
        elif t == "halfmaps":
            opt.nmaps = 2
        elif t == "pad":
            opt.pad = int(val)
        elif "symmetry".startswith(t) and len(t) >= 3:
            opt.symmetry = val
        elif t == "mode":
            opt.sym_mode = int(val)
        elif t == "threads":
            opt.threads = int(val)
        elif t == "seed":
            opt.seed = int(val)
        elif t == "ewald":
            opt.ewald = True
        elif t == "rescale":
            a, b = (float(x) for x in val.split(","))
            opt.rescale = (a, b)
        i += 2 if val is not None else 1
    return opt


def load_case(name: str, directory: str):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    star = materialize_dataset(str(z["dataset"]), directory)
    opt = options_from_args(str(z["options"]))
    plan = plan_reconstruction(read_project(star), opt)
    images = load_images(plan)
    refs = {k: z[k] for k in z.files if k.startswith("map")}
    return plan, images, refs


def backproj_options_from_args(args: str):
    """bbackproj's command-line options (the subset the golden cases use) as
    BackprojOptions: -resolution, -fullmap / -halfmaps, -threads, -symmetry,
    -rescale, -size, -scale."""
    from bsoft_b200.backproj import BackprojOptions
    opt = BackprojOptions()
    toks = shlex.split(args)
    full = half = False
    i = 0
    while i < len(toks):
        t = toks[i].lstrip("-")
        val = toks[i + 1] if i + 1 < len(toks) else None
        if "resolution".startswith(t):
            opt.resolution = float(val); i += 2
        elif t == "fullmap":
            full = True; i += 1
        elif t == "halfmaps":
            half = True; i += 1
        elif t == "threads":
            opt.threads = int(val); i += 2
        elif "symmetry".startswith(t) and len(t) >= 3:
            opt.symmetry = val; i += 2
        elif t == "rescale":
            opt.rescale = tuple(float(x) for x in val.split(",")); i += 2
        elif t == "size":
            opt.size = int(val.split(",")[0]); i += 2
        elif t == "scale":
            opt.scale = float(val); i += 2
        else:
            raise ValueError(f"option {toks[i]}")
    opt.nmaps = (1 if full or not half else 0) + (2 if half else 0)
    return opt
