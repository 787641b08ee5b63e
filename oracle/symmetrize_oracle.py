"""CPU restatement of the reference's real-space point-group symmetrization,
Bimage::symmetrize(sym, flag 1) (bsoft/src/img/Bimage_symmetry.cpp:31-100),
which breconstruct applies to each finished map with -symmetry and
sym_mode 1 (bsoft/src/breconstruct.cpp:335).  Test infrastructure only:
nothing here is shipped or timed as the product.

Steps, each following the reference:
* the fill value is the map's background (calculate_background, flag 0:
  the mean outside the ellipsoid of half-axes (x/2, y/2, z/2) about the
  origin; bsoft/src/img/Bimage_background.cpp:27-80);
* for each generating operation (axis, order m) of the group, in Bsymmetry's
  order and with its axis normalized as Bsymmetry stores it, the map
  becomes the float sum of itself and its m - 1 rotations by j 2 pi / m
  about the axis (Bimage::sum, Bimage_combine.cpp:23-40); the sum's
  background is the sum of the copies' (the rotated copies carry 0), so the
  fill of later operations stays the first background;
* a rotation is Bimage::transform (Bimage_transform.cpp:138-240): the new
  voxel at nu (relative to the origin) takes the old map at M^T nu + origin,
  by Bimage::interpolate (bsoft/src/img/Bimage.cpp:1436-1484, trilinear over
  the in-range neighbours, the fill outside [0, size)), stored as float;
  M = Matrix3(axis, angle) through Quaternion::from_axis_angle
  (bsoft/include/Quaternion.h:34-41) and Matrix3::from_quaternion
  (bsoft/include/Matrix3.h:21-42, entries below 1e-12 set to 0);
* finally every value is multiplied by 1 / (group order).

Arrays are (z, y, x) float32 maps; the origin is (x, y, z).
"""
from __future__ import annotations

import math

import numpy as np

from . import symmetry_ops


def normalize(v):
    """Vector3::normalize (bsoft/include/Vector3.h:264-273): v * (1 / |v|)."""
    v = [float(a) for a in v]
    ln = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    if ln < 1e-30:
        return [v[0], v[1], 1.0]
    div = 1.0 / ln
    return [v[0] * div, v[1] * div, v[2] * div]


def axis_angle_matrix(axis, angle: float) -> np.ndarray:
    """Matrix3(axis, angle) of the reference, as its arithmetic forms it."""
    u = normalize(axis)
    a = angle / 2.0
    sa = math.sin(a)
    q = [math.cos(a), u[0] * sa, u[1] * sa, u[2] * sa]
    q = [0.0 if abs(v) < 1e-30 else v for v in q]
    q0, q1, q2, q3 = q
    d = [[q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3, 2 * q1 * q2 - 2 * q0 * q3, 2 * q1 * q3 + 2 * q0 * q2],
         [2 * q1 * q2 + 2 * q0 * q3, q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3, 2 * q2 * q3 - 2 * q0 * q1],
         [2 * q1 * q3 - 2 * q0 * q2, 2 * q2 * q3 + 2 * q0 * q1, q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3]]
    for i in range(3):
        for j in range(3):
            v = d[i][j]
            if abs(v) < 1e-12:
                v = 0.0
            d[i][j] = min(1.0, max(-1.0, v))
    return np.array(d)


def background(m: np.ndarray, origin) -> float:
    """calculate_background, flag 0 (voxels with r = sum((c - o)/h)^2 - 1 > 0)."""
    nz, ny, nx = m.shape
    hx, hy, hz = nx // 2, ny // 2, nz // 2
    zz, yy, xx = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                             np.arange(nx, dtype=np.float64), indexing="ij")
    x2 = ((xx - origin[0]) / hx) ** 2 if nx > 1 else 0.0
    y2 = ((yy - origin[1]) / hy) ** 2 if ny > 1 else 0.0
    z2 = ((zz - origin[2]) / hz) ** 2 if nz > 1 else 0.0
    sel = (x2 + y2 + z2 - 1) > 0
    if not sel.any():
        return 0.0
    return float(m[sel].astype(np.float64).sum() / sel.sum())


def interpolate(m: np.ndarray, X, Y, Z, fill: float) -> np.ndarray:
    """Bimage::interpolate at (X, Y, Z) (float64 arrays), replaying its loop:
    the fractional weights are flipped (f = 1 - f) once per visited sample
    and not reset between rows, so at the upper edge (one neighbour) the
    weights come out as the reference's do; the sum is divided by the sum of
    the weights."""
    nz, ny, nx = m.shape
    out = np.full(X.shape, fill, dtype=np.float64)
    ok = (X >= 0) & (X < nx) & (Y >= 0) & (Y < ny) & (Z >= 0) & (Z < nz)
    x, y, z = X[ok], Y[ok], Z[ok]
    ix, iy, iz = x.astype(np.int64), y.astype(np.int64), z.astype(np.int64)
    cx = np.where(nx < ix + 2, 1, 2)
    cy = np.where(ny < iy + 2, 1, 2)
    cz = np.where(nz < iz + 2, 1, 2)
    fx, fy, fz = x - ix, y - iy, z - iz
    flat = m.reshape(-1).astype(np.float64)
    value = np.zeros(x.shape)
    ws = np.zeros(x.shape)
    for zk in range(2):
        az = zk < cz
        fz = np.where(az, 1.0 - fz, fz)
        for yk in range(2):
            ay = az & (yk < cy)
            fy = np.where(ay, 1.0 - fy, fy)
            wyz = fy * fz
            for xk in range(2):
                ax = ay & (xk < cx)
                fx = np.where(ax, 1.0 - fx, fx)
                w = fx * wyz
                idx = (np.minimum(iz + zk, nz - 1) * ny + np.minimum(iy + yk, ny - 1)) * nx + \
                    np.minimum(ix + xk, nx - 1)
                ws = ws + np.where(ax, w, 0.0)
                value = value + np.where(ax, flat[idx] * w, 0.0)
    out[ok] = np.where(ws != 0, value / np.where(ws != 0, ws, 1.0), fill)
    return out


def rotate(m: np.ndarray, mat: np.ndarray, origin, fill: float) -> np.ndarray:
    """Bimage::transform with scale 1 and no translation: new(nu) = old(M^T nu + o)."""
    nz, ny, nx = m.shape
    zz, yy, xx = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                             np.arange(nx, dtype=np.float64), indexing="ij")
    n0, n1, n2 = xx - origin[0], yy - origin[1], zz - origin[2]
    old = [n0 * mat[0][i] + n1 * mat[1][i] + n2 * mat[2][i] + origin[i] for i in range(3)]
    return interpolate(m, old[0], old[1], old[2], fill).astype(np.float32)


def symmetrize(m: np.ndarray, origin, sym: str) -> np.ndarray:
    """Bimage::symmetrize(sym, 1) of a (z, y, x) float32 map about `origin`
    (x, y, z).  Groups C, D, T, O, I (the reference's standard settings)."""
    img = np.asarray(m, dtype=np.float32).copy()
    ops = symmetry_ops(sym)
    order = 1
    for _, k in ops:
        order *= k
    if order < 2:
        return img
    fill = background(img, origin)
    # Bsymmetry stores each operation's axis normalized (symmetry.cpp:113-114);
    # Matrix3(axis, angle) normalizes it again
    ops = [(normalize(axis), k) for axis, k in ops]
    for axis, k in ops:
        acc = img.copy()
        for j in range(1, k):
            acc = acc + rotate(img, axis_angle_matrix(axis, j * math.pi * 2.0 / k), origin, fill)
        img = acc
    return (img.astype(np.float64) * (1.0 / order)).astype(np.float32)
