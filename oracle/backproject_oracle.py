"""CPU restatement of the reference's real-space weighted back-projection
(bbackproj: project_back_projection, bsoft/src/mg/mg_reconstruct.cpp:
1524-1624, over Bimage::back_project, bsoft/src/img/Bimage_project.cpp:
466-509).  Test infrastructure only: nothing here is shipped or timed as the
product.

Per image, following the reference:
* check_resolution (bsoft/src/img/Bimage.cpp:633-648): the limit is at most
  the image's real size and at least 2 / sqrt(sum 1/u^2) over its axes;
* fspace_weigh_ramp (bsoft/src/img/Bimage_fspace.cpp:1220-1268): forward
  transform, each coefficient times |s| (s = |k| / real size per axis, with
  k folded at the half size) or 0 beyond the limit, inverse transform, real
  part (the reference's normalised transform pair is the identity round
  trip);
* rescale to mean 0 and standard deviation 1 (Bimage_rescale.cpp:163-182
  over Bimage_stats.cpp: population statistics), stored as float;
* the fill is the image background about the image origin
  (calculate_background, Bimage_background.cpp:27-80);
* every map voxel c (relative to the map's default origin, the integer half
  size) adds the image sampled at M^T c + origin (z dropped), M the view's
  matrix, with Bimage::interpolate (symmetrize_oracle.interpolate), the sum
  stored as float.

Magnification 1 only.  Arrays are (y, x) images and (z, y, x) maps.
"""
from __future__ import annotations

import numpy as np

from .refine_oracle import view_matrix
from .symmetrize_oracle import background, interpolate


def check_resolution(resolution: float, n: int, pixel: float) -> float:
    real = n * pixel
    if resolution > real:
        return real
    rm = 2.0 / np.sqrt(1.0 / (pixel * pixel) + 1.0 / (pixel * pixel))
    return max(resolution, rm)


def weigh_ramp(img: np.ndarray, resolution: float, pixel: float) -> np.ndarray:
    """fspace_weigh_ramp of a square image (float32 result)."""
    n = img.shape[0]
    res = check_resolution(resolution, n, pixel)
    s2max = 1.0 / (res * res)
    idx = np.arange(n)
    h = n // 2
    k = np.where(idx > h, n - idx, idx).astype(np.float64)
    real = n * pixel
    s = k / real
    s2 = s[None, :] ** 2 + s[:, None] ** 2
    w = np.where(s2 > s2max, 0.0, np.sqrt(s2))
    f = np.fft.fft2(img.astype(np.float64))
    return np.real(np.fft.ifft2(f * w)).astype(np.float32)


def back_project(vol: np.ndarray, img: np.ndarray, origin, view, resolution: float, pixel: float) -> np.ndarray:
    """Bimage::back_project of one image into `vol` (float32, in place and
    returned).  origin: (ox, oy) of the image; view: (vx, vy, vz, angle)."""
    p = weigh_ramp(img, resolution, pixel).astype(np.float64)
    avg = p.mean()
    std = np.sqrt(max(0.0, (p * p).mean() - avg * avg))
    scale = 1.0 / std if std > 1e-30 else 1.0
    p = (p * scale + (0.0 - avg * scale)).astype(np.float32)
    fill = background(p[None], (origin[0], origin[1], 0.0))
    mat = view_matrix(view).T
    N = vol.shape[0]
    o = N // 2
    zz, yy, xx = np.meshgrid(np.arange(N, dtype=np.float64), np.arange(N, dtype=np.float64),
                             np.arange(N, dtype=np.float64), indexing="ij")
    c0, c1, c2 = xx - o, yy - o, zz - o
    X = c0 * mat[0][0] + c1 * mat[0][1] + c2 * mat[0][2] + origin[0]
    Y = c0 * mat[1][0] + c1 * mat[1][1] + c2 * mat[1][2] + origin[1]
    v = interpolate(p[None], X, Y, np.zeros_like(X), fill)
    vol[...] = (vol.astype(np.float64) + v).astype(np.float32)
    return vol


def back_projection(images: np.ndarray, params, N: int, resolution: float, pixel: float) -> np.ndarray:
    """project_back_projection over images (K, n, n) with params rows
    (ox, oy, vx, vy, vz, angle): the (N, N, N) float32 map."""
    vol = np.zeros((N, N, N), dtype=np.float32)
    for img, (ox, oy, vx, vy, vz, va) in zip(images, params):
        back_project(vol, img, (ox, oy), (vx, vy, vz, va), resolution, pixel)
    return vol
