"""Orientation conventions of the reference, restated in numpy (host side).

A particle orientation is a *view*: a unit view vector v (the projection
direction) and an in-plane rotation angle a.  The reference turns it into a
rotation matrix through a quaternion:

* ``View::quaternion``  bsoft/include/View.h:131-152
* ``Matrix3(Quaternion)`` bsoft/include/Matrix3.h:30-42 (with ``check``,
  Matrix3.h:21-29: |d| < 1e-12 -> 0, clamp to [-1, 1])
* ``View::normalize`` / ``check``  View.h:30-35, 110-116
* ``angle_set_negPI_to_PI``  bsoft/src/util/utilities.cpp:606-615

The matrix maps the 2-D Fourier pixel (h, k, 0) of a particle image onto the
3-D frequency R (h, k, 0) of the map (Bimage_reconstruct.cpp:150-158), so its
third column is the view vector.
"""
from __future__ import annotations

import math

import numpy as np

SMALLFLOAT = 1e-30
TRIGPRECISION = 1e-30


def angle_set_negpi_to_pi(angle: float) -> float:
    if not math.isfinite(angle):
        return 0.0
    n = int(angle / math.pi)                       # C++ truncation toward zero
    rem = int(math.fmod(n, 2))                     # C++ % keeps the sign
    return angle - (n + rem) * math.pi


def normalize_view(view):
    x, y, z, a = (float(t) for t in view)
    size = math.sqrt(x * x + y * y + z * z)
    if size < SMALLFLOAT:
        x, y, z = 0.0, 0.0, 1.0
    else:
        x, y, z = x / size, y / size, z / size
    x = 0.0 if abs(x) < TRIGPRECISION else x
    y = 0.0 if abs(y) < TRIGPRECISION else y
    z = 0.0 if abs(z) < TRIGPRECISION else z
    a = angle_set_negpi_to_pi(a)
    if abs(a) < TRIGPRECISION:
        a = 0.0
    return x, y, z, a


def view_to_quaternion(view):
    x, y, z, a = normalize_view(view)
    ang = a / 2.0
    ca, sa = math.cos(ang), math.sin(ang)
    z1 = z + 1.0
    q = [ca, 0.0, 0.0, sa]
    if z < 1.0 - SMALLFLOAT:
        if z <= SMALLFLOAT - 1.0:
            q = [0.0, sa, ca, 0.0]
        else:
            f1 = math.sqrt(z1 / 2.0)
            f2 = math.sqrt(1.0 / (2 * z1))
            q = [f1 * ca, f2 * (x * sa - y * ca), f2 * (x * ca + y * sa), f1 * sa]
    return [0.0 if abs(t) < TRIGPRECISION else t for t in q]


def quaternion_to_matrix(q) -> np.ndarray:
    q0, q1, q2, q3 = q
    d = np.array([
        [q0*q0 + q1*q1 - q2*q2 - q3*q3, 2*q1*q2 - 2*q0*q3, 2*q1*q3 + 2*q0*q2],
        [2*q1*q2 + 2*q0*q3, q0*q0 - q1*q1 + q2*q2 - q3*q3, 2*q2*q3 - 2*q0*q1],
        [2*q1*q3 - 2*q0*q2, 2*q2*q3 + 2*q0*q1, q0*q0 - q1*q1 - q2*q2 + q3*q3],
    ], dtype=np.float64)
    d[np.abs(d) < 1e-12] = 0.0
    return np.clip(d, -1.0, 1.0)


def view_to_matrix(view) -> np.ndarray:
    return quaternion_to_matrix(view_to_quaternion(view))


def views_to_matrices(views: np.ndarray) -> np.ndarray:
    return np.stack([view_to_matrix(v) for v in np.asarray(views, dtype=np.float64)])


def random_views(rng: np.random.Generator, n: int) -> np.ndarray:
    """Views uniform on SO(3): view vector uniform on the sphere and angle
    uniform on [-pi, pi) (the stabiliser of the view vector is the in-plane
    rotation, so this is the Haar measure).  Returns (n, 4): x, y, z, angle."""
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    a = rng.uniform(-math.pi, math.pi, size=n)
    return np.concatenate([v, a[:, None]], axis=1)


def matrix_to_view(m: np.ndarray):
    """Inverse of view_to_matrix for proper rotations: (x, y, z, angle)."""
    m = np.asarray(m, dtype=np.float64)
    x, y, z = (float(t) for t in m[:, 2])
    v = (0.0, 0.0, -1.0) if z <= -1 + 1e-12 else (x, y, z)
    return (*v, angle_set_negpi_to_pi(_solve_angle(m, v)))


def _solve_angle(m, v):
    r0 = view_to_matrix((*v, 0.0))
    rz = r0.T @ m
    return math.atan2(rz[1, 0], rz[0, 0])


def angular_distance_deg(ra: np.ndarray, rb: np.ndarray) -> np.ndarray:
    """Geodesic angle (degrees) between rotation matrices (..., 3, 3)."""
    t = np.einsum("...ij,...ij->...", ra, rb)
    c = np.clip((t - 1.0) / 2.0, -1.0, 1.0)
    return np.degrees(np.arccos(c))


def asymmetric_unit_views_c(order: int, theta_step: float, phi_step: float, full: bool = True,
                            inplane: bool = True) -> np.ndarray:
    """Views (x, y, z, angle) tiling the asymmetric unit of the cyclic point
    group C<order> (asymmetric_unit_views below with label "C<order>").
    C1 at 3 degrees gives 4,586 views."""
    return asymmetric_unit_views(f"C{int(order)}", theta_step, phi_step, full=full, inplane=inplane)


GOLDEN_RATIO = 1.61803398874989484820458683436563811772


def _angle_neg_pi_to_pi(a: float) -> float:
    """angle_set_negPI_to_PI (bsoft/src/util/utilities.cpp:606-615): subtract
    (n + n % 2) pi with n = trunc(a / pi) (C remainder), so pi -> -pi."""
    if not math.isfinite(a):
        return 0.0
    n = int(a / math.pi)
    r = int(math.fmod(n, 2))
    return a - (n + r) * math.pi


def _view_normalize(x: float, y: float, z: float, a: float):
    """View::normalize + View::check (bsoft/include/View.h:32-36, 110-116)."""
    size = math.sqrt(x * x + y * y + z * z)
    if size < 1e-30:
        x, y, z = 0.0, 0.0, 1.0
    else:
        x, y, z = x / size, y / size, z / size
    x = 0.0 if abs(x) < 1e-30 else x
    y = 0.0 if abs(y) < 1e-30 else y
    z = 0.0 if abs(z) < 1e-30 else z
    a = _angle_neg_pi_to_pi(a)
    if abs(a) < 1e-30:
        a = 0.0
    return x, y, z, a


def symmetry_point(label: str):
    """Point-group code and order of the first operation of Bsymmetry
    (bsoft/src/util/symmetry.cpp:53-99): Cn -> (100 + n, n), Dn -> (200 + n,
    n), T -> (320, 3), O -> (432, 3), I -> (532, 3) (order 2 or 5 for the
    "-3" settings, which drop the 3-fold operation)."""
    g = (label or "C1").strip()
    c = g[0].upper()
    if c == "C":
        n = 1 if g == "Cs" else int(g[1:])
        return 100 + n, n
    if c == "D":
        n = int(g[1:])
        return 200 + n, n
    if c == "T":
        return 320, 2 if "-3" in g else 3
    if c == "O":
        return 432, (4 if "-4" not in g else 2) if "-3" in g else 3
    if c == "I":
        if "-3" not in g:
            return 532, 3
        return 532, 5 if "-5" in g else 2
    raise ValueError(f"unsupported point group {label!r}")


def asymmetric_unit_views(label: str, theta_step: float, phi_step: float, full: bool = True,
                          inplane: bool = True) -> np.ndarray:
    """Views (x, y, z, angle) tiling the asymmetric unit of a point group:
    asymmetric_unit_views (bsoft/src/util/symmetry.cpp:383-549) for cyclic,
    dihedral, tetrahedral, octahedral and icosahedral groups (the "I90"
    setting included).  Steps in radians; `full` (flag bit 1) covers both
    halves, `inplane` (no flag bit 2) gives cyclic and dihedral views their
    azimuth as in-plane angle.  The floating loops, the View constructor's
    normalisation and the final View::normalize of every view are the
    reference's, so the list matches it bit for bit."""
    if theta_step < math.pi / 1800:
        theta_step = math.pi / 180
    if phi_step < math.pi / 1800:
        phi_step = math.pi / 180
    point, order0 = symmetry_point(label)
    max_theta = math.pi / 2 + 1e-6
    ntheta = int(max_theta / theta_step + 0.5)
    nphi = int(math.pi * 2.0 / (order0 * phi_step) + 0.5)
    if point < 200:
        if full:
            max_theta = math.pi + 1e-6
            ntheta += ntheta
    elif point == 432:
        max_theta = math.pi / 4 + 1e-6
        ntheta = int(max_theta / theta_step + 0.5)
    elif point == 532:
        max_theta = math.atan(1 / (GOLDEN_RATIO + 1)) + 1e-6
        ntheta = int(max_theta / theta_step + 2.5)
        nphi = int(math.atan(1 / GOLDEN_RATIO) / phi_step + 1.5)
    if ntheta < 1:
        ntheta = 1
    if nphi < 1:
        nphi = 1
    raw = []                       # (x, y, z, angle) as constructed, before the final normalize

    def make(x, y, z, a=0.0):
        v = _view_normalize(x, y, z, 0.0)      # the constructor's normalize (angle 0 checked)
        return [v[0], v[1], v[2], a]

    if point < 500:
        raw.append([0.0, 0.0, 1.0, 0.0])
    if 100 < point < 200:
        theta = theta_step
        while theta <= max_theta:
            nrphi = int(nphi * math.sin(theta) / 2 + 0.5)
            phi = 0.0
            istart = 0
            if nrphi:
                phi = math.pi * 1.0 / (order0 * nrphi)
                istart = -nrphi
                if point < 102:
                    nrphi -= 1
            for j in range(istart, nrphi + 1):
                v = make(math.sin(theta) * math.cos(j * phi), math.sin(theta) * math.sin(j * phi), math.cos(theta))
                if inplane:
                    v[3] = j * phi
                raw.append(v)
            theta += theta_step
        if full and raw[-1][2] > -0.999999:
            raw.append([0.0, 0.0, -1.0, 0.0])
    elif 200 < point < 300:
        theta = theta_step
        while theta <= max_theta:
            nrphi = int(nphi * math.sin(theta) / 2 + 0.5)
            phi = math.pi * 1.0 / (order0 * nrphi) if nrphi else 0.0
            istart = -nrphi if full else 0
            for j in range(istart, nrphi + 1):
                v = make(math.sin(theta) * math.cos(j * phi), math.sin(theta) * math.sin(j * phi), math.cos(theta))
                if inplane:
                    v[3] = j * phi
                raw.append(v)
            theta += theta_step
    elif point == 320:
        theta = theta_step
        while theta <= max_theta:
            phi_start, phi_end = 0.0, theta
            if theta > math.pi / 4:
                phi_end = math.pi / 2 - theta
            if full:
                phi_start = -theta
            if full and theta > math.pi / 4:
                phi_start = theta - math.pi / 2
            phi = phi_start
            while phi <= phi_end:
                raw.append(make(math.sin(theta), math.sin(phi), math.cos(theta)))
                phi += phi_step
            theta += theta_step
    elif point == 432:
        theta = theta_step
        while theta <= max_theta:
            phi = -theta if full else 0.0
            while phi <= theta:
                raw.append(make(math.sin(theta), math.sin(phi), math.cos(theta)))
                phi += phi_step
            theta += theta_step
    elif point == 532:
        if "I90" in label:
            theta = -ntheta * theta_step if full else 0.0
            while theta <= max_theta:
                phi = 0.0
                while phi <= GOLDEN_RATIO * (max_theta - abs(theta)):
                    raw.append(make(math.tan(phi), math.tan(theta), math.cos(theta)))
                    phi += phi_step
                theta += theta_step
        else:
            theta = 0.0
            while theta <= max_theta:
                nrphi = int(GOLDEN_RATIO * (max_theta - theta) / phi_step)
                phi = -nrphi * phi_step if full else 0.0
                while phi <= GOLDEN_RATIO * (max_theta - theta):
                    raw.append(make(math.tan(theta), math.tan(phi), math.cos(theta)))
                    phi += phi_step
                theta += theta_step
    else:
        raise ValueError(f"point group {label!r} (code {point}) is not supported")
    return np.array([_view_normalize(*v) for v in raw], dtype=np.float64).reshape(-1, 4)


def search_views(directions: np.ndarray, n_inplane: int) -> np.ndarray:
    """Every direction at n_inplane in-plane angles 2 pi i / n_inplane added
    to its own angle: (ndir * n_inplane, 4), direction-major."""
    d = np.asarray(directions, dtype=np.float64)
    psi = 2 * math.pi * np.arange(n_inplane) / n_inplane
    out = np.repeat(d, n_inplane, axis=0)
    out[:, 3] = np.array([angle_set_negpi_to_pi(a) for a in (out[:, 3] + np.tile(psi, len(d)))])
    return out
