"""Real-space weighted back-projection on the GPU (bbackproj).

``BackProjector`` is the object form of bbackproj's
``project_back_projection`` -> ``img_backprojection_accumulate`` sequence
(bsoft/src/bbackproj.cpp:170-207, bsoft/src/mg/mg_reconstruct.cpp:1524-1684)
over ``Bimage::back_project`` (bsoft/src/img/Bimage_project.cpp:466-509),
driven through libbsgpu's C ABI (bsg_backproj_*):

    plan = plan_backprojection(read_project("in.star"), BackprojOptions(resolution=8))
    with BackProjector(plan) as bp:
        bp.add(load_images(plan), plan.records)
        volume = bp.finish()               # (N, N, N) float32, z, y, x

``plan_backprojection`` resolves what project_back_projection takes from the
project: the map size and sampling (project_set_reconstruction_size,
mg_reconstruct.cpp:596-651), each selected particle's origin (a coordinate
<= 0 falls back to the image file's origin, then to the map's, per axis:
:1585-1596), view, magnification over the scale, and pixel size, and the
half-map index of the round-robin partial maps (project_configure_for_
reconstruction, :669-780; even partial maps form the first half).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .geometry import view_to_matrix
from .io import stacks
from .project import Project

B_ORIGIN, B_MAT, B_MAG, B_MAP, B_PIXEL = 0, 2, 11, 12, 13


@dataclass
class BackprojOptions:
    resolution: float = 0.0       # -resolution (angstrom); 0: the finest the check allows
    size: int = 0                 # -size (0: from the particle images and the scale)
    sampling: float = 0.0         # -sampling (0: from the particles)
    scale: float = 1.0            # -scale
    nmaps: int = 1                # 1 full, 2 half maps, 3 full + halves
    threads: int = 1              # the reference's partial maps per class (half-map parity)
    symmetry: str = "C1"          # -symmetry: the finished map symmetrized
    rescale: tuple = ()           # -rescale avg,std of the finished map


@dataclass
class BackprojPlan:
    n: int
    map: int
    map_sampling: float
    pixel: float
    resolution: float
    records: np.ndarray           # (P, BACKPROJ_DOUBLES)
    stack_index: list = field(default_factory=list)
    nmaps: int = 1
    symmetry: str = "C1"
    rescale: tuple = ()


def plan_backprojection(project: Project, opt: BackprojOptions) -> BackprojPlan:
    mgs = [m for m in project.micrographs if m.n > 0]
    if not mgs:
        raise ValueError("no particles")
    first = mgs[0]
    hdr = stacks.read_header(project.resolve(first.particle_file))
    sam = opt.sampling
    if sam < 0.1:
        sam = float(first.pixel[0]) if first.pixel[0] > 0 else 0.0
    if sam < 0.1:
        sam = first.pixel_size
    if sam < 0.1:
        sam = hdr.sampling[0]
    size = opt.size or max(1, int(hdr.nx * opt.scale))
    o = size // 2                 # the map's default origin
    nmaps = max(1, min(3, opt.nmaps))
    t = max(1, opt.threads)
    if nmaps & 2 and t % 2:
        t += 1
    rows, index = [], []
    k = 0
    for mg in mgs:
        path = project.resolve(mg.particle_file)
        h = stacks.read_header(path)
        for i in range(mg.n):
            if mg.select[i] <= 0:
                continue
            r = np.zeros(_lib.BACKPROJ_DOUBLES)
            fo = h.image_origin_of(int(mg.part_id[i]) - 1)
            ori = mg.origin[i]
            r[B_ORIGIN] = ori[0] if ori[0] > 0 else (fo[0] if fo[0] > 0 else o)
            r[B_ORIGIN + 1] = ori[1] if ori[1] > 0 else (fo[1] if fo[1] > 0 else o)
            r[B_MAT:B_MAT + 9] = view_to_matrix(mg.view[i]).reshape(-1)
            mag = mg.magnification[i] if mg.magnification[i] > 0 else 1.0     # Bparticle's default
            r[B_MAG] = mag / opt.scale
            # partial map k mod t; with half maps the even ones form half 1
            r[B_MAP] = (k % t) % 2 if nmaps & 2 else 0
            r[B_PIXEL] = mg.pixel[i] if mg.pixel[i] > 0 else h.sampling[0]
            rows.append(r)
            index.append((path, int(mg.part_id[i]) - 1))
            k += 1
    records = np.array(rows, dtype=np.float64).reshape(-1, _lib.BACKPROJ_DOUBLES)
    return BackprojPlan(n=hdr.nx, map=size, map_sampling=sam / opt.scale, pixel=float(records[0, B_PIXEL]),
                        resolution=opt.resolution, records=records, stack_index=index, nmaps=nmaps,
                        symmetry=opt.symmetry or "C1", rescale=tuple(opt.rescale))


def load_images(plan: BackprojPlan, sel=None) -> np.ndarray:
    """The selected particle images (P, n, n) float32, in record order."""
    idx = range(len(plan.stack_index)) if sel is None else sel
    out = np.empty((len(idx), plan.n, plan.n), dtype=np.float32)
    cache = {}
    for j, i in enumerate(idx):
        path, k = plan.stack_index[i]
        if path not in cache:
            cache[path] = stacks.read_stack(path)[0]
        out[j] = cache[path][k]
    return out


class BackProjector:
    def __init__(self, plan: BackprojPlan, batch: int = 0, device: int = 0):
        L = _lib.load()
        self.plan = plan
        self.N = plan.map
        cfg = _lib.BackprojConfig(plan.n, plan.map, plan.pixel, plan.resolution, plan.nmaps, batch, device)
        h = C.c_void_p()
        _lib.check(L.bsg_backproj_create(C.byref(cfg), C.byref(h)), "bsg_backproj_create")
        self._h = h
        if plan.symmetry and plan.symmetry != "C1":
            self.set_symmetrize(plan.symmetry)
        if plan.rescale:
            self.set_rescale(*plan.rescale)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().bsg_backproj_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, images, records: np.ndarray) -> None:
        records = np.ascontiguousarray(records, dtype=np.float64).reshape(-1, _lib.BACKPROJ_DOUBLES)
        if hasattr(images, "data_ptr") and getattr(images, "is_cuda", False):
            ptr, flags = C.c_void_p(images.data_ptr()), _lib.BSG_DEVICE_PTR
        else:
            images = np.ascontiguousarray(images, dtype=np.float32)
            ptr, flags = C.c_void_p(images.ctypes.data), 0
        _lib.check(_lib.load().bsg_backproj_add(self._h, ptr, records.ctypes.data_as(C.POINTER(C.c_double)),
                                                len(records), flags), "bsg_backproj_add")

    def finish(self, imap: int = 0) -> np.ndarray:
        out = np.empty((self.N, self.N, self.N), dtype=np.float32)
        _lib.check(_lib.load().bsg_backproj_finish(self._h, imap, C.c_void_p(out.ctypes.data), 0),
                   "bsg_backproj_finish")
        return out

    def set_symmetrize(self, sym):
        from .symmetry import generator_axes
        ops = [] if not sym or sym == "C1" else generator_axes(sym)
        axes = np.ascontiguousarray([a for a, _ in ops] or [[0.0, 0.0, 1.0]], dtype=np.float64)
        orders = np.ascontiguousarray([k for _, k in ops] or [1], dtype=np.int32)
        _lib.check(_lib.load().bsg_backproj_set_symmetrize(self._h, axes.ctypes.data_as(C.POINTER(C.c_double)),
                                                           orders.ctypes.data_as(C.POINTER(C.c_int)), len(ops)),
                   "bsg_backproj_set_symmetrize")

    def set_rescale(self, avg: float = 0.0, std: float = 0.0):
        _lib.check(_lib.load().bsg_backproj_set_rescale(self._h, float(avg), float(std)), "bsg_backproj_set_rescale")

    def reset(self):
        _lib.check(_lib.load().bsg_backproj_reset(self._h), "bsg_backproj_reset")


def records_from_views(origins, views, mag: float = 1.0, pixel: float = 0.0, half=None) -> np.ndarray:
    """Records for images given as origins (K, 2) and views (K, 4: x, y, z,
    angle in radians)."""
    K = len(views)
    r = np.zeros((K, _lib.BACKPROJ_DOUBLES))
    for k in range(K):
        r[k, B_ORIGIN:B_ORIGIN + 2] = origins[k][:2]
        r[k, B_MAT:B_MAT + 9] = view_to_matrix(views[k]).reshape(-1)
        r[k, B_MAG] = mag
        r[k, B_PIXEL] = pixel
        r[k, B_MAP] = 0 if half is None else half[k]
    return r
