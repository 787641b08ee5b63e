"""ctypes front end of the FP64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke``
and by the CPU-baseline leg of bench.py, and only as the checker.  The
product path (bsoft_b200) never imports this package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


class ReconCfg(C.Structure):
    _fields_ = [("n", C.c_int), ("ft", C.c_int), ("map", C.c_int), ("map_sampling", C.c_double),
                ("hi_res", C.c_double), ("interp", C.c_int), ("ctf_action", C.c_int),
                ("wiener", C.c_double)]


class Particle(C.Structure):
    _fields_ = [("origin", C.c_double * 2), ("bkg_center", C.c_double * 2), ("mat", C.c_double * 9),
                ("pixel", C.c_double), ("scale", C.c_double), ("weight", C.c_double),
                ("ctf", C.c_double * 7), ("ewald", C.c_double)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.orc_insert.argtypes = [C.POINTER(ReconCfg), C.POINTER(C.c_float), C.POINTER(Particle), C.c_long,
                                 dp, dp, dp, dp]
        L.orc_insert.restype = C.c_int
        L.orc_particle_transform.argtypes = [C.POINTER(ReconCfg), C.POINTER(C.c_float), C.POINTER(Particle), dp]
        L.orc_particle_transform.restype = C.c_int
        L.orc_finish.argtypes = [C.POINTER(ReconCfg), dp, dp, dp, dp, dp, C.c_int]
        L.orc_finish.restype = C.c_long
        L.orc_fsc.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, C.c_int, dp]
        L.orc_fsc.restype = C.c_int
        L.orc_fsi_kernel.argtypes = [C.c_int, C.c_int, dp]
        L.orc_fsi_kernel.restype = C.c_int
        L.orc_match_diam.argtypes = [C.c_int, C.c_double, C.c_double]
        L.orc_match_diam.restype = C.c_int
        L.orc_match_map.argtypes = [C.c_int, C.POINTER(C.c_float), dp, C.c_double, C.c_double, dp,
                                    C.POINTER(C.c_int)]
        L.orc_match_map.restype = C.c_int
        L.orc_central_section.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, dp, C.c_int, dp]
        L.orc_central_section.restype = C.c_int
        L.orc_match_particle.argtypes = [C.c_int, C.POINTER(C.c_float), C.c_int, C.c_double, C.c_double, dp]
        L.orc_match_particle.restype = C.c_int
        L.orc_phase_shift_2d.argtypes = [C.c_int, dp, dp]
        L.orc_phase_shift_2d.restype = None
        L.orc_recip_space_fom.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_int, dp, C.c_int, dp]
        L.orc_recip_space_fom.restype = C.c_double
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def cfg_from_plan(plan) -> ReconCfg:
    return ReconCfg(plan.n, plan.ft, plan.map, plan.map_sampling, plan.hi_res, plan.interp,
                    plan.ctf_action, plan.wiener)


def particles_from_params(params: np.ndarray):
    from bsoft_b200.plan import P_ORIGIN, P_BKG, P_MAT, P_PIXEL, P_SCALE, P_WEIGHT, P_CTF, P_EWALD
    arr = (Particle * len(params))()
    for i, r in enumerate(params):
        p = arr[i]
        p.origin[:] = list(r[P_ORIGIN:P_ORIGIN + 2])
        p.bkg_center[:] = list(r[P_BKG:P_BKG + 2])
        p.mat[:] = list(r[P_MAT:P_MAT + 9])
        p.pixel, p.scale, p.weight = r[P_PIXEL], r[P_SCALE], r[P_WEIGHT]
        p.ctf[:] = list(r[P_CTF:P_CTF + 7])
        p.ewald = r[P_EWALD]
    return arr


def insert(plan, images: np.ndarray, params: np.ndarray, vol=None, weight=None, power=None, weight2=None,
           aux=False):
    N3 = plan.map ** 3
    if vol is None:
        vol = np.zeros(2 * N3)
        weight = np.zeros(N3)
        if aux:
            power = np.zeros(N3)
            weight2 = np.zeros(N3)
    imgs = np.ascontiguousarray(images, dtype=np.float32)
    cfg = cfg_from_plan(plan)
    parts = particles_from_params(params)
    rc = lib().orc_insert(C.byref(cfg), imgs.ctypes.data_as(C.POINTER(C.c_float)), parts, len(params),
                          _dp(vol), _dp(weight), _dp(power), _dp(weight2))
    if rc:
        raise RuntimeError(f"orc_insert failed: {rc}")
    return vol, weight, power, weight2


def finish(plan, vol, weight, power=None, weight2=None, sinc=None):
    if sinc is None:
        sinc = plan.interp == 2
    out = np.zeros(plan.map ** 3)
    cfg = cfg_from_plan(plan)
    cov = lib().orc_finish(C.byref(cfg), _dp(vol), _dp(weight), _dp(power), _dp(weight2), _dp(out), int(sinc))
    return out.reshape(plan.map, plan.map, plan.map), cov


def symmetry_ops(sym: str):
    """The generating operations (axis, order) of Bsymmetry::Bsymmetry
    (bsoft/src/util/symmetry.cpp:53-99) for Cn, Dn, T, O, I, in its order."""
    g = (sym or "C1").strip().upper()
    phi = (1 + 5 ** 0.5) / 2
    if g[0] == "C":
        return [((0, 0, 1), int(g[1:] or 1))]
    if g[0] == "D":
        return [((0, 0, 1), int(g[1:])), ((1, 0, 0), 2)]
    if g == "T":
        return [((1, 1, 1), 3), ((0, 0, 1), 2), ((1, 0, 0), 2)]
    if g == "O":
        return [((1, 1, 1), 3), ((0, 0, 1), 4), ((1, 0, 0), 2)]
    if g == "I":
        return [((1, 1, 1), 3), ((1, 1 / phi, phi), 2), ((1 / phi, 1, 0), 5), ((0, 0, 1), 2)]
    raise ValueError(sym)


def symmetry_matrices(sym: str) -> np.ndarray:
    """Group elements of a point group as rotation matrices, in the order of
    symmetry_get_all_views (bsoft/src/util/symmetry.cpp:277-319) with the
    generating operations of Bsymmetry::Bsymmetry (symmetry.cpp:53-99):
    Cn, Dn, T, O, I."""
    ops = symmetry_ops(sym)

    def rot(axis, ang):
        a = np.asarray(axis, float) / np.linalg.norm(axis)
        K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        return np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K     # Rodrigues

    mats = [np.eye(3)]
    for axis, order in ops:
        n = len(mats)
        for j in range(1, order):
            r = rot(axis, j * 2 * np.pi / order)
            mats += [r @ mats[k] for k in range(n)]
    return np.stack(mats)


def expand_symmetry(plan, images: np.ndarray, params: np.ndarray):
    """Every particle once per symmetry-related view (fspace_pack_2D over
    symmetry_get_all_views, Bimage_reconstruct.cpp:248-266): matrix S R."""
    sym = getattr(plan, "symmetry", "C1") or "C1"
    if sym == "C1":
        return images, params
    S = symmetry_matrices(sym)
    P = np.repeat(params, len(S), axis=0).copy()
    R = params[:, 4:13].reshape(-1, 3, 3)
    P[:, 4:13] = np.einsum("sab,pbc->psac", S, R).reshape(-1, 9)
    return np.repeat(images, len(S), axis=0), P


def reconstruct(plan, images: np.ndarray, sel=None):
    """Full-map FP64 reconstruction of the selected particles (all by default)."""
    params = plan.params if sel is None else plan.params[sel]
    imgs = images if sel is None else images[sel]
    imgs, params = expand_symmetry(plan, imgs, params)
    vol, w, _, _ = insert(plan, imgs, params)
    m, _ = finish(plan, vol, w)
    return m


def particle_transform(plan, image: np.ndarray, params_row: np.ndarray) -> np.ndarray:
    out = np.zeros(2 * plan.ft * plan.ft)
    cfg = cfg_from_plan(plan)
    parts = particles_from_params(params_row[None])
    img = np.ascontiguousarray(image, dtype=np.float32)
    rc = lib().orc_particle_transform(C.byref(cfg), img.ctypes.data_as(C.POINTER(C.c_float)), parts, _dp(out))
    if rc:
        raise RuntimeError(f"orc_particle_transform failed: {rc}")
    return out.view(np.complex128).reshape(plan.ft, plan.ft)


def ref_binary(name: str) -> str:
    return os.path.join(REF_DIR, name)


# ---- projection matching -------------------------------------------------

def fsi_kernel(width: int = 8, power: int = 2) -> np.ndarray:
    """FSI_Kernel table, shape (513, width)."""
    w = 1 if power < 0 else width
    t = np.zeros(513 * w)
    lib().orc_fsi_kernel(width, power, _dp(t))
    return t.reshape(513, w)


def match_diam(N: int, sampling: float, hi_res: float) -> int:
    return int(lib().orc_match_diam(N, sampling, hi_res))


def match_map(vol: np.ndarray, origin, sampling: float, hi_res: float) -> np.ndarray:
    """Prepared reference transform (diam, diam, diam) complex128."""
    N = vol.shape[0]
    v = np.ascontiguousarray(vol, dtype=np.float32)
    spec = np.zeros(2 * N ** 3)
    d = C.c_int(0)
    o = np.asarray(origin, dtype=np.float64)
    rc = lib().orc_match_map(N, v.ctypes.data_as(C.POINTER(C.c_float)), _dp(o), sampling, hi_res, _dp(spec),
                             C.byref(d))
    if rc:
        raise RuntimeError(f"orc_match_map failed: {rc}")
    D = d.value
    return spec[:2 * D ** 3].view(np.complex128).reshape(D, D, D)


def central_section(spec: np.ndarray, mat: np.ndarray, real_size: float, resolution: float,
                    kernel: np.ndarray) -> np.ndarray:
    D = spec.shape[0]
    s = np.ascontiguousarray(spec, dtype=np.complex128)
    m = np.ascontiguousarray(mat, dtype=np.float64).reshape(9)
    k = np.ascontiguousarray(kernel, dtype=np.float64)
    out = np.zeros(2 * D * D)
    rc = lib().orc_central_section(D, _dp(s.view(np.float64)), _dp(m), real_size, resolution, _dp(k),
                                   k.shape[1], _dp(out))
    if rc:
        raise RuntimeError(f"orc_central_section failed: {rc}")
    return out.view(np.complex128).reshape(D, D)


def match_particle(image: np.ndarray, diam: int, file_avg: float = 0.0, file_std: float = 0.0) -> np.ndarray:
    """Prepared particle transform; file_avg/file_std are the stack's header
    statistics (file_std 0: the image's own)."""
    n = image.shape[0]
    img = np.ascontiguousarray(image, dtype=np.float32)
    out = np.zeros(2 * diam * diam)
    rc = lib().orc_match_particle(n, img.ctypes.data_as(C.POINTER(C.c_float)), diam, file_avg, file_std,
                                  _dp(out))
    if rc:
        raise RuntimeError(f"orc_match_particle failed: {rc}")
    return out.view(np.complex128).reshape(diam, diam)


def phase_shift_2d(spec: np.ndarray, origin) -> np.ndarray:
    s = np.ascontiguousarray(spec, dtype=np.complex128).copy()
    o = np.asarray(origin, dtype=np.float64)
    lib().orc_phase_shift_2d(s.shape[0], _dp(s.view(np.float64)), _dp(o))
    return s


def recip_space_fom(img: np.ndarray, ref: np.ndarray, img_real_size: float, ref_real_size: float,
                    ref_sampling: float, hi_res: float, lo_res: float = 0.0, fom_type: int = 0,
                    ctf=None, invert: bool = False):
    """(fom, cv) of img_recip_space_fom."""
    a = np.ascontiguousarray(img, dtype=np.complex128)
    b = np.ascontiguousarray(ref, dtype=np.complex128)
    c = None if ctf is None else np.ascontiguousarray(ctf, dtype=np.float64)
    cv = np.zeros(1)
    f = lib().orc_recip_space_fom(a.shape[0], _dp(a.view(np.float64)), _dp(b.view(np.float64)), img_real_size,
                                  ref_real_size, ref_sampling, hi_res, lo_res, fom_type, _dp(c), int(invert),
                                  _dp(cv))
    return float(f), float(cv[0])


def fsc(vol1: np.ndarray, vol2: np.ndarray, real_size: float, hi_res: float, nshell: int) -> np.ndarray:
    """Bimage::fsc of two complex (N, N, N) transforms."""
    a = np.ascontiguousarray(vol1, dtype=np.complex128)
    b = np.ascontiguousarray(vol2, dtype=np.complex128)
    out = np.zeros(nshell)
    lib().orc_fsc(a.shape[0], _dp(a.view(np.float64)), _dp(b.view(np.float64)), real_size, hi_res, nshell, _dp(out))
    return out
