"""Seeded synthetic single-particle data (host side, FP64 arithmetic).

Phantoms are sums of isotropic 3-D Gaussian blobs; a projection of a blob is
a 2-D Gaussian (its line integral), so particle images are analytic:

    p(x, y) = sum_b a_b sqrt(2 pi) s_b exp(-((x - ox - b.c0)^2 + (y - oy - b.c1)^2) / (2 s_b^2))

with (c0, c1) the first two columns of the particle's rotation matrix
(geometry.view_to_matrix), b the blob centre relative to the map centre
(N/2) and (ox, oy) the particle origin.  The CTF is applied in Fourier space
as sin(chi) (ctf.py) and white Gaussian noise is added at a stated SNR
(signal variance inside the particle circle / noise variance).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

from .ctf import CTFParams, ctf_chi
from .geometry import random_views, views_to_matrices
from .io import mrc
from .project import Micrograph, Project, write_project


@dataclass
class Phantom:
    size: int
    centers: np.ndarray   # (K, 3) voxel offsets from the map centre (x, y, z)
    sigma: np.ndarray     # (K,) voxels
    amp: np.ndarray       # (K,)


def random_phantom(rng: np.random.Generator, size: int, n_blobs: int,
                   sigma_range=(2.0, 4.0), amp_range=(0.5, 1.0), radius_frac=0.35) -> Phantom:
    r = radius_frac * size
    d = rng.normal(size=(n_blobs, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rad = r * rng.uniform(0, 1, size=n_blobs) ** (1.0 / 3.0)
    return Phantom(size, d * rad[:, None], rng.uniform(*sigma_range, size=n_blobs),
                   rng.uniform(*amp_range, size=n_blobs))


def phantom_volume(ph: Phantom) -> np.ndarray:
    """Point-sampled phantom on the N^3 grid, array order [z, y, x]."""
    n = ph.size
    g = np.arange(n, dtype=np.float64) - n // 2
    vol = np.zeros((n, n, n), dtype=np.float64)
    for c, s, a in zip(ph.centers, ph.sigma, ph.amp):
        gx = np.exp(-(g - c[0]) ** 2 / (2 * s * s))
        gy = np.exp(-(g - c[1]) ** 2 / (2 * s * s))
        gz = np.exp(-(g - c[2]) ** 2 / (2 * s * s))
        vol += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return vol


def project_blobs(ph: Phantom, mats: np.ndarray, origins: np.ndarray, n: int) -> np.ndarray:
    """Analytic projections (B, n, n) [y, x] for rotation matrices (B, 3, 3)
    and particle origins (B, >=2) in pixels."""
    B = mats.shape[0]
    out = np.empty((B, n, n), dtype=np.float64)
    xs = np.arange(n, dtype=np.float64)
    w = ph.amp * math.sqrt(2 * math.pi) * ph.sigma
    for i in range(B):
        px = ph.centers @ mats[i, :, 0] + origins[i, 0]
        py = ph.centers @ mats[i, :, 1] + origins[i, 1]
        inv = 1.0 / (2 * ph.sigma * ph.sigma)
        gx = np.exp(-((xs[:, None] - px[None, :]) ** 2) * inv[None, :])     # (n, K)
        gy = np.exp(-((xs[:, None] - py[None, :]) ** 2) * inv[None, :])
        out[i] = (gy * w[None, :]) @ gx.T
    return out


def apply_ctf(images: np.ndarray, coefs: np.ndarray, pixel: float) -> np.ndarray:
    """Multiply each image's transform by sin(chi) of its own coefficients."""
    B, n, _ = images.shape
    f = np.arange(n, dtype=np.float64)
    f[f > (n - 1) // 2] -= n
    f /= n * pixel
    sy, sx = np.meshgrid(f, f, indexing="ij")
    s2 = sx * sx + sy * sy
    ang = np.arctan2(sy, sx)
    ft = np.fft.fft2(images)
    for i in range(B):
        ft[i] *= np.sin(ctf_chi(coefs[i], s2, ang))
    return np.real(np.fft.ifft2(ft))


def add_noise(rng: np.random.Generator, images: np.ndarray, snr: float) -> np.ndarray:
    if snr is None or snr <= 0:
        return images
    B, n, _ = images.shape
    yy, xx = np.mgrid[0:n, 0:n]
    r2 = (xx - n / 2) ** 2 + (yy - n / 2) ** 2
    inside = r2 <= (n / 2) ** 2
    out = np.empty_like(images)
    for i in range(B):
        var = images[i][inside].var()
        out[i] = images[i] + rng.normal(scale=math.sqrt(var / snr) if var > 0 else 0.0, size=(n, n))
    return out


@dataclass
class DatasetSpec:
    box: int = 64
    n_particles: int = 2000
    n_blobs: int = 50
    pixel: float = 1.5
    volt: float = 200000.0
    cs: float = 2.7e7
    amp_contrast: float = 0.07
    defocus_range: tuple = (1.0e4, 3.0e4)
    astig_range: tuple = (0.0, 0.0)
    shift_range: float = 2.0
    snr: float | None = 0.1
    mean_per_micrograph: float = 0.0     # 0 = one micrograph; else Poisson mean
    ctf: bool = True
    seed: int = 1


def generate(spec: DatasetSpec, rng: np.random.Generator | None = None):
    """Return (phantom, images (n, box, box) float32, per-particle dict)."""
    rng = rng or np.random.default_rng(spec.seed)
    ph = random_phantom(rng, spec.box, spec.n_blobs)
    n = spec.n_particles
    views = random_views(rng, n)
    mats = views_to_matrices(views)
    shifts = rng.uniform(-spec.shift_range, spec.shift_range, size=(n, 2))
    origins = np.concatenate([spec.box // 2 + shifts, np.zeros((n, 1))], axis=1)
    defocus = rng.uniform(*spec.defocus_range, size=n)
    dev = rng.uniform(*spec.astig_range, size=n)
    ast = rng.uniform(-math.pi, math.pi, size=n)
    coefs = np.stack([CTFParams.from_amp_contrast(spec.volt, spec.cs, spec.amp_contrast,
                                                  defocus[i], dev[i], ast[i]).coefficients()
                      for i in range(n)])
    imgs = np.empty((n, spec.box, spec.box), dtype=np.float32)
    chunk = 256
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        p = project_blobs(ph, mats[s:e], origins[s:e], spec.box)
        if spec.ctf:
            p = apply_ctf(p, coefs[s:e], spec.pixel)
        p = add_noise(rng, p, spec.snr)
        imgs[s:e] = p.astype(np.float32)
    if spec.mean_per_micrograph > 0:
        counts = []
        left = n
        while left > 0:
            c = int(max(1, min(left, rng.poisson(spec.mean_per_micrograph))))
            counts.append(c)
            left -= c
    else:
        counts = [n]
    return ph, imgs, dict(views=views, mats=mats, origins=origins, defocus=defocus,
                          def_dev=dev, ast_angle=ast, coefs=coefs, counts=counts)


def write_dataset(outdir: str, spec: DatasetSpec, ph: Phantom, imgs: np.ndarray, meta: dict,
                  star_name: str = "particles.star") -> str:
    """Write one particle stack + one STAR block per micrograph.  Each
    micrograph's CTF block carries its particles' astigmatism only when the
    micrograph holds one particle; per-particle defocus goes into
    ``particle.defocus``."""
    os.makedirs(outdir, exist_ok=True)
    proj = Project(base_dir=outdir)
    start = 0
    for mi, c in enumerate(meta["counts"]):
        sl = slice(start, start + c)
        fname = f"mg{mi + 1:05d}.mrcs"
        mrc.write_stack(os.path.join(outdir, fname), imgs[sl], spec.pixel)
        ctf = None
        if spec.ctf:
            ctf = CTFParams.from_amp_contrast(spec.volt, spec.cs, spec.amp_contrast,
                                              float(meta["defocus"][start]),
                                              float(meta["def_dev"][start]), float(meta["ast_angle"][start]))
        proj.micrographs.append(Micrograph(
            id=f"mg{mi + 1:05d}", particle_file=fname, box_size=spec.box, pixel_size=spec.pixel, ctf=ctf,
            part_id=np.arange(1, c + 1), origin=meta["origins"][sl], view=meta["views"][sl],
            defocus=meta["defocus"][sl] if spec.ctf else np.zeros(c), magnification=np.ones(c),
            select=np.ones(c, dtype=np.int64), pixel=np.full(c, spec.pixel)))
        start += c
    path = os.path.join(outdir, star_name)
    write_project(path, proj)
    return path


def batched_insertion_workload(n_particles: int = 50000, box: int = 256, n_blobs: int = 400, pool: int = 512,
                               pixel: float = 1.5, snr: float = 0.05, mean_per_micrograph: float = 200.0,
                               defocus_range=(8000.0, 35000.0), astig_range=(0.0, 1000.0),
                               volt: float = 200000.0, cs: float = 2.7e7, amp_contrast: float = 0.07,
                               seed: int = 2):
    """Synthetic stand-in for a large insertion job: per-particle parameter
    records (C-ABI layout, see plan.py) for `n_particles` particles grouped
    into micrographs of Poisson(mean) particles with per-particle defocus and
    astigmatism, and a pool of `pool` distinct CTF-modulated noisy
    projections of one blob phantom.  Particle i uses pool image i % pool;
    the images carry the value distribution of the workload, the records its
    geometry."""
    from .plan import (P_BKG, P_CTF, P_MAP, P_MAT, P_ORIGIN, P_PIXEL, P_SCALE, P_WEIGHT, PARTICLE_DOUBLES,
                       check_resolution)
    rng = np.random.default_rng(seed)
    ph = random_phantom(rng, box, n_blobs)
    views = random_views(rng, n_particles)
    mats = views_to_matrices(views)
    origins = box // 2 + rng.uniform(-2.0, 2.0, size=(n_particles, 2))
    defocus = rng.uniform(*defocus_range, size=n_particles)
    dev = rng.uniform(*astig_range, size=n_particles)
    ast = rng.uniform(-math.pi, math.pi, size=n_particles)
    counts = []
    left = n_particles
    while left > 0:
        c = int(max(1, min(left, rng.poisson(mean_per_micrograph))))
        counts.append(c)
        left -= c
    P = np.zeros((n_particles, PARTICLE_DOUBLES))
    P[:, P_ORIGIN:P_ORIGIN + 2] = origins
    P[:, P_BKG:P_BKG + 2] = 0.0
    P[:, P_MAT:P_MAT + 9] = mats.reshape(n_particles, 9)
    P[:, P_PIXEL] = pixel
    P[:, P_SCALE] = 1.0
    P[:, P_WEIGHT] = 1.0
    for i in range(n_particles):
        P[i, P_CTF:P_CTF + 7] = CTFParams.from_amp_contrast(volt, cs, amp_contrast, defocus[i], dev[i],
                                                            ast[i]).coefficients()
    P[:, P_MAP] = np.arange(n_particles) % 2
    pool = min(pool, n_particles)
    imgs = np.empty((pool, box, box), dtype=np.float32)
    chunk = 64
    for s in range(0, pool, chunk):
        e = min(pool, s + chunk)
        p = project_blobs(ph, mats[s:e], np.concatenate([origins[s:e], np.zeros((e - s, 1))], 1), box)
        p = apply_ctf(p, P[s:e, P_CTF:P_CTF + 7], pixel)
        imgs[s:e] = add_noise(rng, p, snr).astype(np.float32)
    hi_res = check_resolution(pixel, box, pixel)
    return dict(params=P, pool=imgs, counts=counts, phantom=ph, hi_res=hi_res, pixel=pixel, box=box)
