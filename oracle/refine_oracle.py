"""CPU restatement of brefine's grid refinement (img_refine_grid).

TEST INFRASTRUCTURE ONLY: the checker for bsg_match_refine
(bsoft_b200/csrc/refine.cu); nothing in the product imports it.  Pinned to
the reference's own img_refine_grid through the golden fixtures of
tests/golden/make_refine_golden.py (tests/test_refine_oracle.py).

Follows, one particle at a time:
  * img_refine_grid              bsoft/src/mg/mg_refine.cpp:1086-1195
  * img_fit_in_recip_space_grid  bsoft/src/mg/mg_refine.cpp:862-950
  * views_for_refinement         bsoft/src/util/View.cpp:371-424
  * Quaternion (axis-angle, product, rotate)  bsoft/include/Quaternion.h:28-177
  * View normalisation, View::quaternion      bsoft/include/View.h:30-157
with every hypothesis scored by the FP64 oracle's central section and
img_recip_space_fom (match_oracle.c).  Floating-point loops are written as
the reference writes them, so ragged origin grids come out the same.

The defocus search (brefine -defocus: img_fit_in_recip_space_grid
:866-911, img_refine_grid :1105-1106, 1118, 1133, 1186-1191) goes through
CTFparam's defocus accessors (bsoft/include/ctf.h:133-134, 76-79, 309-317),
whose wavelength term t2 is a long double: np.longdouble (x87 extended on
x86-64, as the reference's build) reproduces their rounding.
"""
from __future__ import annotations

import math

import numpy as np

from . import central_section, fsi_kernel, phase_shift_2d, recip_space_fom

TRIG = 1e-30

# bsoft/include/utilities.h:55-58
PLANCK, EMASS, ECHARGE, LIGHTSPEED = 6.626070E-34, 9.109384E-31, 1.602177E-19, 299792458


class Defocus:
    """CTFparam's defocus_average set/get for one accelerating voltage."""

    def __init__(self, volt: float):
        LD = np.longdouble
        root = math.sqrt(2.0 * EMASS * ECHARGE * volt * (1.0 + ECHARGE * volt / (2.0 * EMASS * LIGHTSPEED * LIGHTSPEED)))
        wl = float(LD(PLANCK) * LD(1e10) / LD(root))        # ctf.h:311, stored as double
        self.t2 = LD(-math.pi * wl)                         # ctf.h:78, double product held as long double

    def abw20(self, defocus: float) -> float:
        return float(self.t2 * np.longdouble(defocus))

    def defocus(self, abw20: float) -> float:
        return float(np.longdouble(abw20) / self.t2)


def _angle_neg_pi_to_pi(a: float) -> float:
    if not math.isfinite(a):
        return 0.0
    n = int(a / math.pi)
    rem = int(math.fmod(n, 2))
    return a - (n + rem) * math.pi


def _norm_view(w, times: int = 1):
    x, y, z, a = w
    for _ in range(times):
        size = math.sqrt(x * x + y * y + z * z)
        if size < TRIG:
            x, y, z = 0.0, 0.0, 1.0
        else:
            x, y, z = x / size, y / size, z / size
        x, y, z = (0.0 if abs(t) < TRIG else t for t in (x, y, z))
        a = _angle_neg_pi_to_pi(a)
        if abs(a) < TRIG:
            a = 0.0
    return (x, y, z, a)


def _vnorm(v):
    ln = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    if ln < 1e-30:
        return [v[0], v[1], 1.0]
    d = 1.0 / ln
    return [v[0] * d, v[1] * d, v[2] * d]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _qcheck(q):
    return [0.0 if abs(t) < TRIG else t for t in q]


def _qaxis(axis, angle):
    a = angle / 2.0
    u = _vnorm(axis)
    s = math.sin(a)
    return _qcheck([math.cos(a), u[0] * s, u[1] * s, u[2] * s])


def _qmul(p, q):
    s, v0, v1, v2 = p
    return [s * q[0] - (v0 * q[1] + v1 * q[2] + v2 * q[3]),
            s * q[1] + v0 * q[0] + v1 * q[3] - v2 * q[2],
            s * q[2] + v1 * q[0] + v2 * q[1] - v0 * q[3],
            s * q[3] + v2 * q[0] + v0 * q[2] - v1 * q[1]]


def _qrotate(q, p):
    inv = _qcheck(q)
    size2 = inv[0] * inv[0] + (inv[1] * inv[1] + inv[2] * inv[2] + inv[3] * inv[3])
    div = 1 / size2
    inv = [inv[0] * div, inv[1] * -div, inv[2] * -div, inv[3] * -div]
    return _qmul(_qmul(q, p), inv)


def view_matrix(w) -> np.ndarray:
    """View::matrix of a view as the reference holds it (one more normalisation)."""
    x, y, z, a = _norm_view(w)
    ang = a / 2.0
    ca, sa = math.cos(ang), math.sin(ang)
    z1 = z + 1
    q = [ca, 0.0, 0.0, sa]
    if z < 1.0 - TRIG:
        if z <= TRIG - 1.0:
            q = [0.0, sa, ca, 0.0]
        else:
            f1, f2 = math.sqrt(z1 / 2.0), math.sqrt(1.0 / (2 * z1))
            q = [f1 * ca, f2 * (x * sa - y * ca), f2 * (x * ca + y * sa), f1 * sa]
    q = _qcheck(q)
    m = [q[0] * q[0] + q[1] * q[1] - q[2] * q[2] - q[3] * q[3],
         2 * q[1] * q[2] - 2 * q[0] * q[3],
         2 * q[1] * q[3] + 2 * q[0] * q[2],
         2 * q[1] * q[2] + 2 * q[0] * q[3],
         q[0] * q[0] - q[1] * q[1] + q[2] * q[2] - q[3] * q[3],
         2 * q[2] * q[3] - 2 * q[0] * q[1],
         2 * q[1] * q[3] - 2 * q[0] * q[2],
         2 * q[2] * q[3] + 2 * q[0] * q[1],
         q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3]]
    m = [0.0 if abs(t) < 1e-12 else min(1.0, max(-1.0, t)) for t in m]
    return np.array(m).reshape(3, 3)


def views_for_refinement(theview, alpha_step: float):
    """The 27 views around theview (the by-value copy; normalised once more here)."""
    if alpha_step <= 0:
        return [theview]
    w = _norm_view(theview)
    vv = [w[0], w[1], w[2]]
    axis1 = _cross(vv, [0.0, 0.0, 1.0])
    if math.sqrt(sum(t * t for t in axis1)) < 0.001:
        axis1[0] = 1.0
    axis1 = _vnorm(axis1)
    axis2 = _cross(vv, axis1)
    if math.sqrt(sum(t * t for t in axis2)) < 0.001:
        axis2[1] = 1.0
    axis2 = _vnorm(axis2)
    qv = _qcheck([0.0, *vv])
    out = []
    a1 = -alpha_step
    while a1 <= alpha_step:
        q1 = _qaxis(axis1, a1)
        a2 = -alpha_step
        while a2 <= alpha_step:
            q = _qmul(_qaxis(axis2, a2), q1)
            q = _qrotate(q, qv)
            a3 = -alpha_step
            while a3 <= alpha_step:
                out.append(_norm_view((q[1], q[2], q[3], w[3] + a3)))
                a3 += alpha_step
            a2 += alpha_step
        a1 += alpha_step
    return out


def origin_grid(ox: float, oy: float, step: float):
    """img_fit_in_recip_space_grid's floating loops: y outer, x inner."""
    pts = []
    y = oy - step
    while y <= oy + step:
        x = ox - step
        while x <= ox + step:
            pts.append((x, y))
            x += step
        y += step
    return pts


class Scorer:
    """Exact figure of merit of (view, origin in cut pixels) for one particle."""

    def __init__(self, spec, prep, n: int, pixel: float, N: int, hi_res: float):
        self.spec, self.prep = spec, prep
        self.D = spec.shape[0]
        self.samp = pixel * N / self.D
        self.real_img = n * pixel
        self.hi_res = hi_res
        self.kernel = fsi_kernel(8, 2)
        self._sec = {}
        self._img = {}

    def __call__(self, view, origin, ctf=None):
        """ctf: [abw00, abw20, abw22, abw2m2, abw40] applied to the section, or None."""
        mat = view_matrix(view)
        key = mat.tobytes()
        sec = self._sec.get(key)
        if sec is None:
            sec = central_section(self.spec, mat, self.D * self.samp, self.hi_res / 1.11, self.kernel)
            self._sec[key] = sec
        x = self._img.get(origin)
        if x is None:
            x = phase_shift_2d(self.prep, origin)
            self._img[origin] = x
        return recip_space_fom(x, sec, self.real_img, self.D * self.samp, self.samp, self.hi_res, ctf=ctf)


class CtfSearch:
    """The particle's CTF (aberration weights) and defocus step of brefine -defocus."""

    def __init__(self, volt: float, coefs, def_std: float):
        self.dz = Defocus(volt)
        self.coefs = [float(c) for c in coefs[:5]]
        self.def_std = def_std
        self.abw20 = self.coefs[1]        # the CTFparam's current abw[2,0]

    def current(self):
        c = list(self.coefs)
        c[1] = self.abw20
        # img_recip_space_fom applies the CTF only for a defocus >= 1 (mg_refine.cpp:685-686)
        return c if self.dz.defocus(self.abw20) >= 1 else None


def fit_origin(score, view, ox, oy, step, accuracy, counter, ctf=None):
    """img_fit_in_recip_space_grid: (fom, (x, y), cv); with a CtfSearch the
    defocus loop comes first and leaves the best defocus in ctf.abw20."""
    bestfom, bestcv, best = -1.0, 0.0, (ox, oy)
    if ctf is not None:
        bestdef = ctf.dz.defocus(ctf.abw20)
        def_start, def_end = bestdef - 5 * ctf.def_std, bestdef + 5 * ctf.def_std
        d = def_start
        while d <= def_end:
            ctf.abw20 = ctf.dz.abw20(d)
            f, cv = score(view, (ox, oy), ctf.current())
            counter[0] += 1
            if bestfom < f:
                bestfom, bestdef, bestcv = f, d, cv
            d += ctf.def_std
        ctf.abw20 = ctf.dz.abw20(bestdef)
    cc = ctf.current() if ctf is not None else None
    while step >= accuracy:
        prevfom, bestfom = bestfom, -1.0
        pts = origin_grid(ox, oy, step)
        ibest = 0
        for i, o in enumerate(pts):
            f, cv = score(view, o, cc)
            counter[0] += 1
            if bestfom < f:
                bestfom, ibest, best, bestcv = f, i, o, cv
        if ibest == len(pts) // 2 or abs(prevfom - bestfom) < 1e-6:
            step /= 2
    return bestfom, best, bestcv


def refine_grid(score, view, origin_cut, alpha_step, accuracy, shift_step, shift_accuracy, ctf=None):
    """img_refine_grid without magnification search for one particle.

    view: (x, y, z, angle) as given; origin_cut: origin in cut pixels; ctf:
    a CtfSearch (brefine -defocus) or None (no CTF).
    Returns (view, origin_cut, fom, cv, number, defocus)."""
    counter = [0]
    bestview = _norm_view(view, 4)          # constructed, stored, read back, copied
    bestfom, bestcv, bestorigin = -1.0, 0.0, tuple(origin_cut)
    defocus = bestdef = 0.0
    if ctf is not None and ctf.def_std and ctf.dz.defocus(ctf.abw20):
        defocus = bestdef = ctf.dz.defocus(ctf.abw20)
    elif ctf is not None:
        ctf = None
    while alpha_step >= accuracy:
        prefom, bestfom = bestfom, -1.0
        views = views_for_refinement(_norm_view(bestview), alpha_step)
        ibest = 0
        for i, v in enumerate(views):
            if defocus:
                ctf.abw20 = ctf.dz.abw20(defocus)          # resets defocus to the original
            f, o, cv = fit_origin(score, _norm_view(v, 3), origin_cut[0], origin_cut[1], shift_step,
                                  shift_accuracy, counter, ctf)
            if bestfom < f:
                bestfom, ibest, bestview, bestorigin, bestcv = f, i, v, o, cv
                if defocus:
                    bestdef = ctf.dz.defocus(ctf.abw20)
        if ibest == len(views) // 2 or abs(prefom - bestfom) < 1e-6:
            alpha_step /= 2
    out_def = 0.0
    if defocus:
        out_def = bestdef if defocus - 5 * ctf.def_std < bestdef < defocus + 5 * ctf.def_std else defocus
        out_def = ctf.dz.defocus(ctf.dz.abw20(out_def))
    return _norm_view(bestview, 3), bestorigin, bestfom, bestcv, counter[0], out_def
