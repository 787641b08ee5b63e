"""Host-side planning of a reconstruction: everything ``breconstruct`` decides
before the per-particle loop, restated so the GPU path and the checker get
identical per-particle parameters.

Sources (all under bsoft/src):
* option defaults and clamps            breconstruct.cpp:71-160, 190-245
* map size / sampling                    mg/mg_reconstruct.cpp:596-651
* transform size                         mg/mg_reconstruct.cpp:38-64 (part_ft_size)
* resolution limit                       img/Bimage.cpp:633-648 (check_resolution)
* partial-map assignment / half maps     mg/mg_reconstruct.cpp:669-780, 266-300
* per-particle CTF, origin, view, scale  mg/mg_reconstruct.cpp:143-212
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from .ctf import CTFParams, electron_wavelength
from .geometry import view_to_matrix
from .io import mrc, stacks  # noqa: F401
from .project import Project

# interpolation / CTF action codes (breconstruct.cpp:131-135; options.h:418-442)
INTERP = {"nearest": 0, "weighted": 1, "trilinear": 2}
CTF_ACTIONS = {"none": 0, "flip": 1, "apply": 2, "correct": 3, "wiener": 4}

# per-particle record layout shared with the C-ABI (include/bsgpu.h,
# bsg_particle): 32 doubles per particle
PARTICLE_DOUBLES = 32
P_ORIGIN, P_BKG, P_MAT, P_PIXEL, P_SCALE, P_WEIGHT, P_CTF, P_MAP = 0, 2, 4, 13, 14, 15, 16, 23
P_NORM = 24       # image normalisation scale, shift (breconstruct -rescale); scale 0 = none
P_EWALD = 26      # electron wavelength (angstrom) for Ewald-sphere insertion (-ewald); 0 = plane


def find_next_power_of(n: int, base: int = 2) -> int:
    """utilities.cpp:447-461: smallest power of `base` >= n."""
    p = 1
    while p < n:
        p *= base
    return p


def part_ft_size(xsize: int, scale: float, pad_factor: int) -> int:
    """mg_reconstruct.cpp:38-64."""
    if xsize <= 0:
        raise ValueError("part_ft_size: size not set")
    ft = xsize
    if scale > 1:
        ft = int(xsize * scale)
    if pad_factor < 1:
        return ft
    pad_factor = min(pad_factor, 8)
    ft = find_next_power_of(int(pad_factor * xsize * scale), 2)
    if ft < xsize:
        ft = find_next_power_of(xsize, 2)
    return ft


def check_resolution(resolution: float, size: int, sampling: float, dims: int = 3) -> float:
    """Bimage::check_resolution (Bimage.cpp:633-648) for a cubic map."""
    if resolution > size * sampling:
        return size * sampling
    rm = 2.0 / math.sqrt(dims / (sampling * sampling))
    return max(resolution, rm)


@dataclass
class ReconOptions:
    interp: int = 0               # reference default: nearest
    pad: int = 2
    ctf_action: int = 0
    wiener: float = 0.0
    resolution: float = 0.0       # angstrom; 0 = default
    size: int = 0                 # map edge; 0 = from images
    sampling: float = 0.0         # angstrom/voxel; 0 = from particles
    scale: float = 1.0
    nmaps: int = 1                # 1 full, 2 half maps, 3 full + halves
    bootstrap: bool = False
    fom: bool = False             # keep power / weight^2 channels
    threads: int = 2              # reference partial maps (only sets half-map parity)
    symmetry: str = ""            # point group (-symmetry; "" = C1)
    sym_mode: int = 0             # -mode: 0 during reconstruction, 1 after it (real space)
    rescale: tuple = ()           # -rescale (average, standard deviation) of the finished map
    ewald: bool = False           # -ewald: insert on the Ewald sphere (both surfaces)
    seed: int = -1                # -mode 2's random() seed (< 0: the process id, as the reference)


@dataclass
class ReconPlan:
    n: int
    ft: int
    map: int
    map_sampling: float
    hi_res: float
    interp: int
    ctf_action: int
    wiener: float
    params: np.ndarray            # (P, 32) float64 per-particle records
    stack_index: list = field(default_factory=list)   # (stack file, image index) per particle
    nmaps: int = 1
    symmetry: str = "C1"          # point group inserted during reconstruction (mode 0)
    resolution: float = 0.0       # breconstruct's limit before any check (the statistics' limit)
    sym_mode: int = 0             # 0: symmetry inserted; 1: the finished map symmetrized
    rescale: tuple = ()           # (average, standard deviation) of the finished map, or ()


def partial_maps(npart: int, opt: ReconOptions) -> int:
    """Number of partial maps breconstruct splits the selection into
    (thread_limit: at least 2, at most npart/2, even with half maps;
    breconstruct.cpp:204-205, mg_reconstruct.cpp:676)."""
    t = max(2, opt.threads)
    t = max(1, min(t, npart // 2))
    if opt.nmaps & 2 and t % 2:
        t += 1
    return t


def mode2_draw_order(npart: int, opt: ReconOptions) -> list:
    """Selected-particle indices in the order breconstruct -mode 2 draws their
    random views: particle k belongs to partial map k mod T (the round-robin of
    project_configure_for_reconstruction, mg_reconstruct.cpp:757-763), and the
    partial maps run one after another when its OpenMP loop has one thread
    (breconstruct.cpp:281-289).  With more threads the reference's draws
    interleave unpredictably; this order is the reproducible one."""
    t = partial_maps(npart, opt)
    return [k for m in range(t) for k in range(m, npart, t)]


def plan_reconstruction(project: Project, opt: ReconOptions) -> ReconPlan:
    mgs = [m for m in project.micrographs if m.n > 0]
    if not mgs:
        raise ValueError("no particles")
    first = mgs[0]
    first_file = project.resolve(first.particle_file)
    hdr = stacks.read_header(first_file)

    # project_set_reconstruction_size
    sam = opt.sampling
    if sam < 0.1:
        sam = float(first.pixel[0]) if first.pixel[0] > 0 else 0.0
    if sam < 0.1:
        sam = first.pixel_size
    if sam < 0.1:
        sam = hdr.sampling[0]
    size = opt.size or int(hdr.nx * opt.scale)
    resolution = opt.resolution if opt.resolution >= 0.1 else sam
    ft = first.box_size or hdr.nx
    if size > ft:
        ft = size
    ft = part_ft_size(ft, 1, opt.pad)
    # particle_reconstruct: pixel size of the map, check_resolution
    map_sampling = sam / opt.scale
    hi_res = check_resolution(resolution, size, map_sampling)
    wiener = opt.wiener
    if opt.ctf_action > 2 and wiener < 0.01:
        wiener = 0.2

    rows = []
    index = []
    k = 0
    em = CTFParams()       # CTFparam defaults when a micrograph has no CTF block
    for mg in mgs:
        path = project.resolve(mg.particle_file)
        h = stacks.read_header(path)
        if mg.ctf is not None:
            em = CTFParams(**vars(mg.ctf))
        for i in range(mg.n):
            if mg.select[i] <= 0:
                continue
            r = np.zeros(PARTICLE_DOUBLES)
            file_origin = h.image_origin_of(int(mg.part_id[i]) - 1)
            ori = mg.origin[i].copy()
            if ori[0] <= 0:
                ori = np.array(file_origin) if file_origin[0] > 0 else np.zeros(3)
            r[P_ORIGIN:P_ORIGIN + 2] = ori[:2]
            r[P_BKG:P_BKG + 2] = file_origin[:2]
            r[P_MAT:P_MAT + 9] = view_to_matrix(mg.view[i]).reshape(-1)
            r[P_PIXEL] = mg.pixel[i] if mg.pixel[i] > 0 else h.sampling[0]
            r[P_SCALE] = 1.0 / mg.magnification[i] if mg.magnification[i] > 0 else 1.0
            r[P_WEIGHT] = float(mg.select[i]) if opt.bootstrap else 1.0
            c = CTFParams(**vars(em))
            if mg.defocus[i] > 0:
                c.defocus = float(mg.defocus[i])
            r[P_CTF:P_CTF + 7] = c.coefficients()
            # round-robin partial maps; even maps form half 1 (mg_reconstruct.cpp:757-763, 283-290)
            r[P_MAP] = k % 2
            if opt.ewald:
                # particle_reconstruct: ew_wl = em_ctf.lambda() (mg_reconstruct.cpp:209-210)
                r[P_EWALD] = electron_wavelength(c.volt)
            if opt.rescale:
                # particle_reconstruct: rescale_to_avg_std(0, 1) with the
                # statistics read_img attaches (mg_reconstruct.cpp:155)
                avg, sd = h.file_stats
                if sd < 1e-30:
                    img = stacks.read_stack(path, int(mg.part_id[i]) - 1, 1)[0][0].astype(np.float64)
                    avg = img.sum() / img.size
                    sd = (img * img).sum() / img.size - avg * avg
                    sd = math.sqrt(sd) if sd > 0 else 0.0
                scale = 1.0 / sd if sd > 1e-30 else 1.0
                r[P_NORM] = scale
                r[P_NORM + 1] = 0.0 - avg * scale
            rows.append(r)
            index.append((path, int(mg.part_id[i]) - 1))
            k += 1
    params = np.array(rows, dtype=np.float64).reshape(-1, PARTICLE_DOUBLES)
    if opt.sym_mode == 2 and (opt.symmetry or "C1") != "C1":
        # particle_reconstruct with sym_mode 2: each particle inserted once,
        # with a random one of its symmetry-related views
        # (random_symmetric_view, mg_reconstruct.cpp:175)
        from .symmetry import operators, random_view_indices
        S = operators(opt.symmetry)
        for j, i in zip(mode2_draw_order(len(params), opt), random_view_indices(len(params), len(S), opt.seed if opt.seed >= 0 else os.getpid())):
            params[j, P_MAT:P_MAT + 9] = (S[i] @ params[j, P_MAT:P_MAT + 9].reshape(3, 3)).reshape(-1)
    return ReconPlan(n=hdr.nx, ft=ft, map=size, map_sampling=map_sampling, hi_res=hi_res,
                     interp=opt.interp, ctf_action=opt.ctf_action, wiener=wiener,
                     params=params,
                     stack_index=index, nmaps=opt.nmaps, symmetry=opt.symmetry or "C1", resolution=resolution,
                     sym_mode=opt.sym_mode, rescale=tuple(opt.rescale))


def load_images(plan: ReconPlan, sel=None) -> np.ndarray:
    """Read the plan's particle images (host float32, (P, n, n))."""
    idx = plan.stack_index if sel is None else [plan.stack_index[i] for i in sel]
    out = np.empty((len(idx), plan.n, plan.n), dtype=np.float32)
    cache = {}
    for j, (path, num) in enumerate(idx):
        if path not in cache:
            cache[path] = stacks.read_stack(path)[0]
        out[j] = cache[path][num]
    return out
