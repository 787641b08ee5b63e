"""Host-side mirror of the reference's projection-matching operators on the
GPU (brefine's scoring path, bsoft/src/mg/mg_refine.cpp).

``Matcher`` holds one prepared reference map and a set of prepared particle
images on the device and scores (image, view, origin) hypotheses with the
reference's FRC figure of merit:

    m = Matcher(n=128, map=128, map_sampling=1.5, pixel=1.5, hi_res=3.75)
    m.set_reference(volume, origin=(64, 64, 64))      # project_refine_orientations
    m.set_images(images, ctf_records)                 # part_refine_orientation
    fom, cv = m.score(hypotheses)                     # img_recip_space_fom

Hypotheses are rows of 12 doubles: image index, the view matrix (row-major,
as View::matrix) and the origin (x, y) in pixels of the particle image.
CTF records are rows of 8 doubles: volt, abw00, abw20, abw22, abw2m2, abw40,
flags (MATCH_APPLY_CTF | MATCH_INVERT), 0.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import MATCH_APPLY_CTF, MATCH_INVERT, MATCH_CTF_DOUBLES, MATCH_HYP_DOUBLES  # noqa: F401


def _ptr(a):
    if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
        return C.c_void_p(a.data_ptr()), True
    return C.c_void_p(a.ctypes.data), False


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Matcher:
    def __init__(self, n: int, map: int, map_sampling: float, pixel: float, hi_res: float, lo_res: float = 0.0,
                 kernel_width: int = 8, kernel_power: int = 2, batch: int = 0, device: int = 0):
        L = _lib.load()
        cfg = _lib.MatchConfig(n, map, map_sampling, pixel, hi_res, lo_res, kernel_width, kernel_power, batch, device)
        h = C.c_void_p()
        _lib.check(L.bsg_match_create(C.byref(cfg), C.byref(h)), "bsg_match_create")
        self._h = h
        info = _lib.MatchInfo()
        _lib.check(L.bsg_match_info(h, C.byref(info)), "bsg_match_info")
        self.info = info
        self.diam = info.diam
        self.n = n
        self.N = map
        self.nimg = 0

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().bsg_match_destroy(self._h)
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

    @property
    def stream(self) -> int:
        """The context's cudaStream_t (for events around its work)."""
        return int(_lib.load().bsg_match_stream(self._h) or 0)

    def set_reference(self, volume, origin=None) -> None:
        if origin is None:
            origin = (self.N // 2,) * 3
        o = np.ascontiguousarray(origin, dtype=np.float64)
        if not (hasattr(volume, "data_ptr") and getattr(volume, "is_cuda", False)):
            volume = np.ascontiguousarray(volume, dtype=np.float32)
        p, dev = _ptr(volume)
        _lib.check(_lib.load().bsg_match_set_reference(self._h, p, _dp(o), _lib.BSG_DEVICE_PTR if dev else 0),
                   "bsg_match_set_reference")

    def reference_transform(self) -> np.ndarray:
        D = self.diam
        out = np.empty((D, D, D), dtype=np.complex64)
        _lib.check(_lib.load().bsg_match_reference_transform(self._h, C.c_void_p(out.ctypes.data), 0),
                   "bsg_match_reference_transform")
        return out

    def sections(self, mats) -> np.ndarray:
        m = np.ascontiguousarray(mats, dtype=np.float64).reshape(-1, 9)
        D = self.diam
        out = np.empty((len(m), D, D), dtype=np.complex64)
        _lib.check(_lib.load().bsg_match_sections(self._h, _dp(m), len(m), C.c_void_p(out.ctypes.data), 0),
                   "bsg_match_sections")
        return out

    def project(self, mats, resolution: float = 0.0, origins=None, ctf=None, out=None):
        """Real-space projections (nviews, N, N) of the reference through its
        transform (Bimage::project); `out` may be a CUDA tensor."""
        m = np.ascontiguousarray(mats, dtype=np.float64).reshape(-1, 9)
        o = None if origins is None else np.ascontiguousarray(origins, dtype=np.float64).reshape(-1, 2)
        c = None if ctf is None else np.ascontiguousarray(ctf, dtype=np.float64).reshape(-1, MATCH_CTF_DOUBLES)
        if out is None:
            out = np.empty((len(m), self.N, self.N), dtype=np.float32)
        p, dev = _ptr(out)
        _lib.check(_lib.load().bsg_match_project(self._h, _dp(m), len(m), float(resolution),
                                                 None if o is None else _dp(o), None if c is None else _dp(c), p,
                                                 _lib.BSG_DEVICE_PTR if dev else 0), "bsg_match_project")
        return out

    def set_images(self, images, ctf, file_avg: float = 0.0, file_std: float = 0.0) -> None:
        """Prepare particle images (nimg, n, n) with their CTF records
        (nimg, 8).  file_std > 0: normalise by the stack file's statistics,
        as the reference does for particles read from a stack."""
        c = np.ascontiguousarray(ctf, dtype=np.float64).reshape(-1, MATCH_CTF_DOUBLES)
        if not (hasattr(images, "data_ptr") and getattr(images, "is_cuda", False)):
            images = np.ascontiguousarray(images, dtype=np.float32)
        nimg = images.shape[0]
        if len(c) != nimg:
            raise ValueError("one CTF record per image")
        p, dev = _ptr(images)
        _lib.check(_lib.load().bsg_match_set_images(self._h, p, nimg, _dp(c), float(file_avg), float(file_std),
                                                    _lib.BSG_DEVICE_PTR if dev else 0), "bsg_match_set_images")
        self.nimg = nimg

    def prepared(self, first: int = 0, count: int | None = None) -> np.ndarray:
        count = self.nimg - first if count is None else count
        D = self.diam
        out = np.empty((count, D, D), dtype=np.complex64)
        _lib.check(_lib.load().bsg_match_prepared(self._h, first, count, C.c_void_p(out.ctypes.data), 0),
                   "bsg_match_prepared")
        return out

    def score(self, hyps, fp64: bool = False, dpr: bool = False):
        """Figure of merit and cross-validation figure of each hypothesis: the
        FRC form, or with dpr the DPR form (brefine -fomtype dpr)."""
        h = np.ascontiguousarray(hyps, dtype=np.float64).reshape(-1, MATCH_HYP_DOUBLES)
        fom = np.empty(len(h))
        cv = np.empty(len(h))
        flags = (_lib.MATCH_SCORE_FP64 if fp64 else 0) | (_lib.MATCH_SCORE_DPR if dpr else 0)
        _lib.check(_lib.load().bsg_match_score(self._h, _dp(h), len(h), _dp(fom), _dp(cv), flags), "bsg_match_score")
        return fom, cv

    def refine(self, start, alpha_step: float, accuracy: float, shift_step: float = 0.4,
               shift_accuracy: float = 0.1, def_std: float = 0.0, dpr: bool = False,
               max_mag: float = 0.0) -> np.ndarray:
        """img_refine_grid for every start record (n, 7): image index, view
        x, y, z, angle (radians), origin x, y (particle pixels).  Angular
        step and accuracy in radians, shift step and accuracy in pixels of
        the cut transform (the reference's arguments); def_std > 0 adds
        brefine's defocus search (angstrom); max_mag > 0 its magnification
        search (brefine -magnification).  Returns (n, 12): view x, y, z,
        angle, origin x, y, figure of merit, cross-validation figure,
        hypotheses scored, defocus (0 without the search), pixel size x, y
        after refinement.  dpr scores with the DPR figure of merit (brefine
        -fomtype dpr)."""
        s = np.ascontiguousarray(start, dtype=np.float64).reshape(-1, _lib.MATCH_REFINE_START_DOUBLES)
        out = np.empty((len(s), _lib.MATCH_REFINE_RESULT_DOUBLES))
        _lib.check(_lib.load().bsg_match_refine(self._h, _dp(s), len(s), float(alpha_step), float(accuracy),
                                                float(shift_step), float(shift_accuracy), float(def_std),
                                                float(max_mag), _dp(out),
                                                _lib.MATCH_SCORE_DPR if dpr else 0), "bsg_match_refine")
        return out


    # ---- exhaustive search ----
    def refine_monte(self, start, max_iter: int, def_std: float = 0.0, shift_std: float = 0.0,
                     view_std: float = 0.0, max_angle: float = 0.0, max_mag: float = 0.0, seed: int = 1,
                     dpr: bool = False) -> np.ndarray:
        """img_refine_monte for every start record (brefine -monte); max_angle
        in radians, shift_std in pixels of the cut transform; random() seeded
        with `seed`.  Returns (n, 12) as refine()."""
        s = np.ascontiguousarray(start, dtype=np.float64).reshape(-1, _lib.MATCH_REFINE_START_DOUBLES)
        out = np.empty((len(s), _lib.MATCH_REFINE_RESULT_DOUBLES))
        _lib.check(_lib.load().bsg_match_refine_monte(self._h, _dp(s), len(s), int(max_iter), float(def_std),
                                                      float(shift_std), float(view_std), float(max_angle),
                                                      float(max_mag), int(seed), _dp(out),
                                                      _lib.MATCH_SCORE_DPR if dpr else 0), "bsg_match_refine_monte")
        return out

    def set_shell_weights(self, w=None) -> None:
        """Per-shell weights of the figure of merit (None: unit weights)."""
        a = np.ascontiguousarray([] if w is None else w, dtype=np.float64)
        _lib.check(_lib.load().bsg_match_set_shell_weights(self._h, _dp(a) if a.size else None, int(a.size)),
                   "bsg_match_set_shell_weights")

    def set_c_curve_weights(self) -> None:
        """brefine's default weighting: C_curve(diam, 1 / real size of the cut
        map) (mg_refine.cpp:366-367, ctf.cpp:795-810)."""
        self.set_shell_weights(c_curve(self.diam, 1.0 / (self.diam * self.info.map_sampling_cut)))

    def set_panel(self, mats, exact_sections: bool = True) -> None:
        """Search panel of central sections for row-major view matrices (nsec,
        3, 3).  exact_sections keeps the panel's FP32 sections for the exact
        rescoring (when they fit); False makes the rescoring gather them."""
        m = np.ascontiguousarray(mats, dtype=np.float64).reshape(-1, 9)
        flags = 0 if exact_sections else _lib.MATCH_PANEL_GATHER
        _lib.check(_lib.load().bsg_match_set_panel(self._h, _dp(m), len(m), flags), "bsg_match_set_panel")
        self.nsec = len(m)

    def search(self, origins, topk: int = 8) -> np.ndarray:
        """Every held image at every trial origin (norigin, 2) against the
        panel; returns (nimg, topk, 5): section, origin index, correlation
        score, FRC figure of merit, cross-validation figure, best first."""
        o = np.ascontiguousarray(origins, dtype=np.float64).reshape(-1, 2)
        out = np.empty((self.nimg, topk, _lib.MATCH_RESULT_DOUBLES))
        _lib.check(_lib.load().bsg_match_search(self._h, _dp(o), len(o), topk, _dp(out), 0), "bsg_match_search")
        return out

    def search_local(self, proposals, origins, radius_deg: float = 10.0, origin_radius: float = 1.5,
                     topk: int = 8) -> np.ndarray:
        """Like search(), restricted per image to the panel sections within
        radius_deg of its proposed rotation and the trial origins within
        origin_radius pixels of its proposed origin; proposals (nimg, 11) as
        the proposer predicts them (host array or CUDA tensor)."""
        import math
        o = np.ascontiguousarray(origins, dtype=np.float64).reshape(-1, 2)
        if not (hasattr(proposals, "data_ptr") and getattr(proposals, "is_cuda", False)):
            proposals = np.ascontiguousarray(proposals, dtype=np.float32)
        p, dev = _ptr(proposals)
        out = np.empty((self.nimg, topk, _lib.MATCH_RESULT_DOUBLES))
        _lib.check(_lib.load().bsg_match_search_local(self._h, p, math.radians(radius_deg), _dp(o), len(o),
                                                      float(origin_radius), topk, _dp(out),
                                                      _lib.BSG_DEVICE_PTR if dev else 0), "bsg_match_search_local")
        return out

    def stats(self) -> dict:
        st = _lib.MatchStats()
        _lib.check(_lib.load().bsg_match_get_stats(self._h, C.byref(st)), "bsg_match_get_stats")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def reset_stats(self) -> None:
        _lib.check(_lib.load().bsg_match_reset_stats(self._h), "bsg_match_reset_stats")


def ctf_record(volt: float, coefs, apply: bool = True, invert: bool = False) -> np.ndarray:
    """CTF record from the aberration weights [abw00, abw20, abw22, abw2m2, abw40, ...]."""
    c = np.asarray(coefs, dtype=np.float64)
    flags = (MATCH_APPLY_CTF if apply else 0) | (MATCH_INVERT if invert else 0)
    return np.array([volt, c[0], c[1], c[2], c[3], c[4], flags, 0.0])


def hypothesis(img: int, mat, origin) -> np.ndarray:
    m = np.asarray(mat, dtype=np.float64).reshape(9)
    return np.array([img, *m, origin[0], origin[1]], dtype=np.float64)


def c_curve(n: int, freq_step: float) -> np.ndarray:
    """The reference's C_curve (bsoft/src/util/ctf.cpp:795-810): a sum of five
    Gaussians in s^2 at s = i * freq_step."""
    s2 = (np.arange(n) * freq_step) ** 2
    return (0.893 * np.exp(-0.2465 * s2) + 0.2563 * np.exp(-1.7100 * s2) + 0.7570 * np.exp(-6.4094 * s2)
            + 1.0487 * np.exp(-18.6113 * s2) + 0.3575 * np.exp(-50.2523 * s2))
