"""Reconstruction project: micrographs, their CTF blocks and particles.

Host-side mirror of the parts of ``Bproject``/``Bmicrograph``/``Bparticle``
(bsoft/include/mg_processing.h:101-137, 279-374, 505-536) and of the STAR
project reader (bsoft/src/rwparam/rwmgSTAR.cpp:195-262 particle loop,
:458-519 CTF block, :521-655 micrograph block, :769-907 block walk) that the
reconstruction path reads.

Conventions carried over:
* particle view: ``particle.view_{x,y,z}`` + ``particle.view_angle`` (deg),
  or Euler ``particle.psi|omega, theta, phi`` (deg) -> view (Euler.h:62-66);
* ``particle.origin_{x,y,z}`` in pixels; ``particle.defocus`` (angstrom)
  replaces the micrograph's average defocus when > 0
  (bsoft/src/mg/mg_reconstruct.cpp:187);
* ``particle.magnification`` > 0 scales the frequency by 1/mag (:183-185);
* ``particle.select`` drives class selection and bootstrap weights;
* particle stacks are shared per micrograph (``particle.file_name`` item),
  ``particle.id`` being the 1-based image number in the stack (:150-154).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from .ctf import CTFParams
from .io.star import StarBlock, StarLoop, read_star, write_star


@dataclass
class Micrograph:
    id: str
    particle_file: str
    box_size: int
    pixel_size: float
    ctf: CTFParams | None
    part_id: np.ndarray            # (n,) int, 1-based image number in the stack
    origin: np.ndarray             # (n, 3) pixels
    view: np.ndarray               # (n, 4) x, y, z, angle (radians)
    defocus: np.ndarray            # (n,) angstrom, 0 = use micrograph value
    magnification: np.ndarray      # (n,)
    select: np.ndarray             # (n,) int
    pixel: np.ndarray              # (n,) particle pixel size (angstrom)
    pixel_y: np.ndarray | None = None   # (n,) along y, where it differs from x (brefine -magnification)

    @property
    def n(self) -> int:
        return int(self.part_id.shape[0])


@dataclass
class Project:
    micrographs: list = field(default_factory=list)
    base_dir: str = "."

    @property
    def n_particles(self) -> int:
        return sum(m.n for m in self.micrographs)

    def resolve(self, path: str) -> str:
        return path if os.path.isabs(path) else os.path.join(self.base_dir, path)


def _euler_to_view(psi, theta, phi):
    from .geometry import angle_set_negpi_to_pi
    return (math.cos(phi) * math.sin(theta), math.sin(phi) * math.sin(theta),
            math.cos(theta), angle_set_negpi_to_pi(psi + phi))


def _ctf_from_block(b: StarBlock) -> CTFParams | None:
    if not b.has("ctf.voltage"):
        return None
    if b.has("ctf.amplitude_phase_shift"):
        amp_shift = b.real("ctf.amplitude_phase_shift")
    else:
        amp_shift = math.asin(b.real("ctf.amp_contrast"))
    if b.has("ctf.defocus_average"):
        dav = b.real("ctf.defocus_average")
        dev = b.real("ctf.defocus_deviation")
    else:
        dmin, dmax = b.real("ctf.defocus_min"), b.real("ctf.defocus_max")
        dav, dev = (dmax + dmin) / 2, abs(dmax - dmin) / 2
    volt = b.real("ctf.voltage")
    if volt < 1e3:
        volt *= 1e3      # kV given (rwmg.cpp:641)
    return CTFParams(volt=volt, cs=b.real("ctf.Cs"), amp_shift=amp_shift,
                     defocus=dav, def_dev=dev,
                     ast_angle=b.real("ctf.astigmatism_angle") * math.pi / 180.0,
                     beam_tilt_x=b.real("ctf.beam_tilt_x"), beam_tilt_y=b.real("ctf.beam_tilt_y"))


def read_project(path: str) -> Project:
    blocks = read_star(path)
    proj = Project(base_dir=os.path.dirname(os.path.abspath(path)))
    for b in blocks:
        if not (b.has("micrograph.id") or b.has("micrograph.file_name")):
            continue
        mgid = b.items.get("micrograph.id") or os.path.splitext(os.path.basename(b.items["micrograph.file_name"]))[0]
        pfile = b.items.get("particle.file_name", "")
        # box size vector as micrograph_from_starblock fills it (rwmgSTAR.cpp:590-605)
        bs = [0, 0, 0]
        if b.has("particle.box_radius"):
            bs = [2 * b.integer("particle.box_radius")] * 3
        if b.has("particle.box_radius_x"):
            bs = [2 * b.integer("particle.box_radius_" + a) for a in "xyz"]
        if b.has("particle.box_size"):
            bs = [b.integer("particle.box_size")] * 3
        if b.has("particle.box_size_x"):
            bs = [b.integer("particle.box_size_" + a) for a in "xyz"]
        box = bs[0]
        mg_pixel = b.real("micrograph.pixel_size") or b.real("micrograph.pixel_size_x")
        lp = b.loop_with("particle.id")
        n = len(lp.rows) if lp else 0

        def col(tag, default=0.0, conv=float):
            c = lp.column(tag) if lp else None
            if c is None:
                return np.full(n, default, dtype=np.float64 if conv is float else np.int64)
            return np.array([conv(float(v)) for v in c])

        ids = col("particle.id", 0, int).astype(np.int64)
        origin = np.stack([col("particle.origin_x"), col("particle.origin_y"), col("particle.origin_z")], 1) \
            if n else np.zeros((0, 3))
        if lp is not None and lp.index("particle.view_angle") >= 0:
            view = np.stack([col("particle.view_x"), col("particle.view_y"), col("particle.view_z"),
                             col("particle.view_angle") * math.pi / 180.0], 1)
        elif lp is not None and (lp.index("particle.psi") >= 0 or lp.index("particle.omega") >= 0):
            if lp.index("particle.psi") >= 0:
                psi = col("particle.psi") * math.pi / 180.0
            else:
                psi = -col("particle.omega") * math.pi / 180.0
            th = col("particle.theta") * math.pi / 180.0
            ph = col("particle.phi") * math.pi / 180.0
            view = np.array([_euler_to_view(a, b_, c) for a, b_, c in zip(psi, th, ph)]).reshape(n, 4)
        else:
            view = np.tile(np.array([0.0, 0.0, 1.0, 0.0]), (n, 1))
        pix = col("particle.pixel_size_x", 0.0)
        if lp is not None and lp.index("particle.pixel_size_x") < 0:
            pix = col("particle.pixel_size", 0.0)
        pix = np.where(pix > 0, pix, mg_pixel)
        pix_y = None
        if lp is not None and lp.index("particle.pixel_size_y") >= 0:
            pix_y = col("particle.pixel_size_y", 0.0)
            pix_y = np.where(pix_y > 0, pix_y, pix)
        # read_project post-processing (rwmg.cpp:650-659): an origin further
        # than box_x/4 (integer division) from box/2 (integer halves, z
        # included) is reset to box/2; then origin z = 0.
        half = np.array([bs[0] // 2, bs[1] // 2, bs[2] // 2], dtype=np.float64)
        for i in range(n):
            if np.linalg.norm(origin[i] - half) > bs[0] // 4:
                origin[i] = half
            origin[i, 2] = 0.0
        mg = Micrograph(id=str(mgid), particle_file=pfile, box_size=box, pixel_size=mg_pixel,
                        ctf=_ctf_from_block(b), part_id=ids, origin=origin, view=view,
                        defocus=col("particle.defocus"), magnification=col("particle.magnification"),
                        select=col("particle.select", 1, int).astype(np.int64), pixel=pix, pixel_y=pix_y)
        proj.micrographs.append(mg)
    if not proj.micrographs:
        raise ValueError(f"{path}: no micrograph blocks found")
    return proj


def write_project(path: str, proj: Project) -> None:
    blocks = []
    for mg in proj.micrographs:
        b = StarBlock(mg.id)
        b.items["micrograph.id"] = mg.id
        b.items["micrograph.pixel_size"] = float(mg.pixel_size)
        b.items["particle.file_name"] = mg.particle_file
        # per-axis box size with z = 1: a cubic box_size would make the
        # reference reset every particle origin to the box centre on read
        b.items["particle.box_size_x"] = int(mg.box_size)
        b.items["particle.box_size_y"] = int(mg.box_size)
        b.items["particle.box_size_z"] = 1
        if mg.ctf is not None:
            c = mg.ctf
            b.items["ctf.voltage"] = float(c.volt)
            b.items["ctf.Cs"] = float(c.cs)
            b.items["ctf.amplitude_phase_shift"] = float(c.amp_shift)
            b.items["ctf.defocus_average"] = float(c.defocus)
            b.items["ctf.defocus_deviation"] = float(c.def_dev)
            b.items["ctf.astigmatism_angle"] = float(c.ast_angle * 180.0 / math.pi)
        lp = StarLoop(tags=["particle.id", "particle.defocus", "particle.magnification",
                            "particle.pixel_size_x", "particle.pixel_size_y", "particle.pixel_size_z",
                            "particle.origin_x", "particle.origin_y", "particle.origin_z",
                            "particle.view_x", "particle.view_y", "particle.view_z",
                            "particle.view_angle", "particle.select"])
        for i in range(mg.n):
            lp.rows.append([int(mg.part_id[i]), float(mg.defocus[i]), float(mg.magnification[i]),
                            float(mg.pixel[i]), float(mg.pixel[i] if mg.pixel_y is None else mg.pixel_y[i]),
                            float(mg.pixel[i]),
                            float(mg.origin[i, 0]), float(mg.origin[i, 1]), float(mg.origin[i, 2]),
                            float(mg.view[i, 0]), float(mg.view[i, 1]), float(mg.view[i, 2]),
                            float(mg.view[i, 3] * 180.0 / math.pi), int(mg.select[i])])
        b.loops.append(lp)
        blocks.append(b)
    write_star(path, blocks)
