"""Host-side mirror of the reference's reconstruction operators on the GPU.

``Reconstructor`` is the object form of the reference's
``particle_reconstruct`` -> ``img_reconstruction_sum_weigh`` -> ``fft_back``
sequence (bsoft/include/mg_reconstruct.h:16-20, bsoft/src/breconstruct.cpp:
280-359), driven through libbsgpu's C ABI:

    plan = plan_reconstruction(read_project("in.star"), ReconOptions(interp=2))
    with Reconstructor(plan) as rec:
        rec.insert(images, plan.params)       # any number of calls, any batch
        volume = rec.finish()                 # (N, N, N) float32, z, y, x

Images may be host numpy arrays (copied to the device through the context's
staging buffers, overlapped with compute) or CUDA tensors (anything with
``data_ptr()`` on the device), in which case nothing is copied.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .plan import ReconPlan


def _ptr(a):
    """(address, is_device) of a numpy array or a CUDA tensor."""
    if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
        return C.c_void_p(a.data_ptr()), True
    return C.c_void_p(a.ctypes.data), False


class Reconstructor:
    def __init__(self, plan: ReconPlan, fom: bool = False, batch: int = 0, device: int = 0):
        L = _lib.load()
        self.plan = plan
        self.N = plan.map
        self.ft = plan.ft
        cfg = _lib.ReconConfig(plan.n, plan.ft, plan.map, plan.map_sampling, plan.hi_res, plan.interp,
                               plan.ctf_action, plan.wiener, plan.nmaps, int(fom), batch, device)
        h = C.c_void_p()
        _lib.check(L.bsg_recon_create(C.byref(cfg), C.byref(h)), "bsg_recon_create")
        self._h = h
        sym = getattr(plan, "symmetry", "C1") or "C1"
        if sym != "C1":
            mode = getattr(plan, "sym_mode", 0)
            if mode == 1:
                self.set_symmetrize(sym)
            elif mode == 0:
                self.set_symmetry(sym)
            # mode 2: the plan's records already carry each particle's random
            # symmetry-related view
        if getattr(plan, "rescale", None):
            self.set_rescale(*plan.rescale)
        self.fom = fom

    # context management
    def close(self):
        if getattr(self, "_h", None):
            _lib.load().bsg_recon_destroy(self._h)
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

    # operators
    def insert(self, images, params: np.ndarray) -> None:
        params = np.ascontiguousarray(params, dtype=np.float64)
        n = params.shape[0]
        if hasattr(images, "data_ptr"):
            if tuple(images.shape[-2:]) != (self.plan.n, self.plan.n) or images.shape[0] != n:
                raise ValueError("images must be (P, n, n) matching params")
            if not images.is_contiguous():
                raise ValueError("images must be contiguous")
            ptr, dev = _ptr(images)
        else:
            images = np.ascontiguousarray(images, dtype=np.float32)
            if images.shape != (n, self.plan.n, self.plan.n):
                raise ValueError(f"images {images.shape} do not match ({n}, {self.plan.n}, {self.plan.n})")
            ptr, dev = _ptr(images)
        flags = _lib.BSG_DEVICE_PTR if dev else 0
        _lib.check(_lib.load().bsg_recon_insert(self._h, ptr, C.c_void_p(params.ctypes.data), n, flags),
                   "bsg_recon_insert")
        self._keep = images   # host buffers must outlive the asynchronous upload

    def synchronize(self):
        _lib.check(_lib.load().bsg_recon_synchronize(self._h), "bsg_recon_synchronize")
        self._keep = None

    def finish(self, imap: int = 0, sinc: bool | None = None, out=None, with_fom: bool = False):
        if sinc is None:
            sinc = self.plan.interp == 2
        N = self.N
        flags = _lib.BSG_SINC if sinc else 0
        fom = np.empty((N, N, N), dtype=np.float32) if with_fom else None
        if out is not None and hasattr(out, "data_ptr"):
            flags |= _lib.BSG_DEVICE_PTR
            mp, _ = _ptr(out)
            fp = C.c_void_p(0)
            if with_fom:
                raise ValueError("device output with FOM is not supported from Python")
            _lib.check(_lib.load().bsg_recon_finish(self._h, imap, mp, fp, flags), "bsg_recon_finish")
            return out
        vol = np.empty((N, N, N), dtype=np.float32) if out is None else out
        _lib.check(_lib.load().bsg_recon_finish(self._h, imap, C.c_void_p(vol.ctypes.data),
                                                C.c_void_p(fom.ctypes.data) if with_fom else C.c_void_p(0),
                                                flags), "bsg_recon_finish")
        self._keep = None
        return (vol, fom) if with_fom else vol

    def accumulators(self, half: int = 0):
        N = self.N
        vol = np.empty((N, N, N, 2), dtype=np.float64)
        w = np.empty((N, N, N), dtype=np.float64)
        _lib.check(_lib.load().bsg_recon_accumulators(self._h, half, C.c_void_p(vol.ctypes.data),
                                                      C.c_void_p(w.ctypes.data), 0), "bsg_recon_accumulators")
        return vol[..., 0] + 1j * vol[..., 1], w

    def add_partial(self, vol: np.ndarray, weight: np.ndarray, half: int = 0) -> None:
        """Add another shard's accumulators (as `accumulators` returns them:
        complex vol, weight) into half `half` of this context, the
        reference's partial-map sum before weighing."""
        N = self.N
        v = np.empty((N, N, N, 2), dtype=np.float64)
        v[..., 0] = np.real(vol)
        v[..., 1] = np.imag(vol)
        w = np.ascontiguousarray(weight, dtype=np.float64)
        if w.size != N ** 3:
            raise ValueError(f"weight has {w.size} values, the map {N ** 3}")
        _lib.check(_lib.load().bsg_recon_add_partial(self._h, half, C.c_void_p(v.ctypes.data),
                                                     C.c_void_p(w.ctypes.data), None, None, 0),
                   "bsg_recon_add_partial")

    def fsc(self, nshell: int | None = None) -> np.ndarray:
        nshell = nshell or self.N // 2
        out = np.zeros(nshell)
        _lib.check(_lib.load().bsg_recon_fsc(self._h, nshell, out.ctypes.data_as(C.POINTER(C.c_double))),
                   "bsg_recon_fsc")
        return out

    def statistics(self, imap: int = 0, resolution: float | None = None) -> dict:
        """Reconstruction statistics of map imap as breconstruct prints them
        (bsg_recon_statistics): Friedel residual, coverage, the shell table
        (columns radius, s, resolution, weight, power, signal, noise, SNR,
        FSC) and the SNR(0.5) / FSC(0.3) resolution estimates.  resolution:
        breconstruct's limit before checks (default: the plan's)."""
        res = self.plan.resolution if resolution is None else resolution
        st = _lib.ShellStats()
        rows = max(1, int(self.plan.map * self.plan.map_sampling / res) + 1) if res > 0.1 else self.N
        table = np.zeros((rows, _lib.STATS_COLUMNS))
        _lib.check(_lib.load().bsg_recon_statistics(self._h, imap, float(res), C.byref(st),
                                                    table.ctypes.data_as(C.POINTER(C.c_double)), rows),
                   "bsg_recon_statistics")
        return dict(friedel=st.friedel, coverage=st.coverage, coverage_pct=st.coverage_pct, res_snr=st.res_snr,
                    res_fsc=st.res_fsc, table=table[:st.rows].copy())

    def spectra(self, images, params: np.ndarray) -> np.ndarray:
        params = np.ascontiguousarray(params, dtype=np.float64)
        images = np.ascontiguousarray(images, dtype=np.float32)
        n = params.shape[0]
        out = np.empty((n, self.ft, self.ft, 2), dtype=np.float32)
        _lib.check(_lib.load().bsg_particle_spectra(self._h, C.c_void_p(images.ctypes.data),
                                                    C.c_void_p(params.ctypes.data), n,
                                                    C.c_void_p(out.ctypes.data), 0), "bsg_particle_spectra")
        return out[..., 0] + 1j * out[..., 1]

    def autotune(self, images, params: np.ndarray):
        """Time every gridding tile shape on these particles, keep the
        fastest, then clear the accumulators (call before inserting)."""
        params = np.ascontiguousarray(params, dtype=np.float64)
        ptr, dev = _ptr(images if hasattr(images, "data_ptr") else np.ascontiguousarray(images, np.float32))
        keep = images
        ms = np.zeros(8)
        best = C.c_int(0)
        _lib.check(_lib.load().bsg_recon_autotune(self._h, ptr, C.c_void_p(params.ctypes.data), params.shape[0],
                                                  _lib.BSG_DEVICE_PTR if dev else 0,
                                                  ms.ctypes.data_as(C.POINTER(C.c_double)), C.byref(best)),
                   "bsg_recon_autotune")
        del keep
        return best.value, ms[:4]

    def set_symmetry(self, sym):
        """Point group (label, or (n, 3, 3) operator matrices) inserted during
        reconstruction, as breconstruct -symmetry does."""
        from .symmetry import operators
        ops = operators(sym) if isinstance(sym, str) else np.asarray(sym, dtype=np.float64)
        ops = np.ascontiguousarray(ops, dtype=np.float64).reshape(-1, 9)
        _lib.check(_lib.load().bsg_recon_set_symmetry(self._h, ops.ctypes.data_as(C.POINTER(C.c_double)), len(ops)),
                   "bsg_recon_set_symmetry")

    def set_symmetrize(self, sym):
        """Point group applied to the finished map in real space
        (breconstruct -symmetry with -mode 1); "C1" or None turns it off."""
        from .symmetry import generator_axes
        ops = [] if not sym or sym == "C1" else generator_axes(sym)
        axes = np.ascontiguousarray([a for a, _ in ops] or [[0.0, 0.0, 1.0]], dtype=np.float64)
        orders = np.ascontiguousarray([k for _, k in ops] or [1], dtype=np.int32)
        _lib.check(_lib.load().bsg_recon_set_symmetrize(self._h, axes.ctypes.data_as(C.POINTER(C.c_double)),
                                                        orders.ctypes.data_as(C.POINTER(C.c_int)), len(ops)),
                   "bsg_recon_set_symmetrize")

    def set_rescale(self, avg: float = 0.0, std: float = 0.0):
        """breconstruct -rescale avg,std of the finished map (std <= 0: off)."""
        _lib.check(_lib.load().bsg_recon_set_rescale(self._h, float(avg), float(std)), "bsg_recon_set_rescale")

    def set_tile_shape(self, shape: int):
        _lib.check(_lib.load().bsg_recon_set_tile_shape(self._h, shape), "bsg_recon_set_tile_shape")

    def set_half_space(self, on: bool = True) -> int:
        """Half-space gridding (on by default for trilinear insertion without
        the FOM channels): about half the gridding work, the full map's sums
        when read.  Switching on needs empty accumulators.  Returns the split
        zsplit (0: the full map)."""
        z = C.c_int(0)
        _lib.check(_lib.load().bsg_recon_set_half_space(self._h, int(on), C.byref(z)), "bsg_recon_set_half_space")
        return z.value

    def reset(self):
        _lib.check(_lib.load().bsg_recon_reset(self._h), "bsg_recon_reset")

    def set_timing(self, on: bool = True):
        _lib.check(_lib.load().bsg_recon_set_timing(self._h, int(on)), "bsg_recon_set_timing")

    def stats(self) -> dict:
        st = _lib.ReconStats()
        _lib.check(_lib.load().bsg_recon_get_stats(self._h, C.byref(st)), "bsg_recon_get_stats")
        return {k: getattr(st, k) for k, _ in _lib.ReconStats._fields_}

    @property
    def stream(self) -> int:
        return _lib.load().bsg_recon_stream(self._h) or 0


def reconstruct(plan: ReconPlan, images, params=None, nmap: int = 0, **kw) -> np.ndarray:
    """One-shot GPU reconstruction of all plan particles (map ``nmap``)."""
    with Reconstructor(plan, **kw) as rec:
        rec.insert(images, plan.params if params is None else params)
        return rec.finish(nmap)
