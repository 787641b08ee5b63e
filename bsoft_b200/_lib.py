"""ctypes binding of libbsgpu.so (the C ABI in include/bsgpu.h).

The library is built in-tree (bsoft_b200/_build/libbsgpu.so) by
``bsoft_b200.build.build()``.  There is no CPU fallback: if the library or a
usable sm_100 device is missing, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libbsgpu.so")

BSG_DEVICE_PTR = 1
BSG_SINC = 2
PARTICLE_DOUBLES = 32


class ReconConfig(C.Structure):
    _fields_ = [("n", C.c_int), ("ft", C.c_int), ("map", C.c_int), ("map_sampling", C.c_double),
                ("hi_res", C.c_double), ("interp", C.c_int), ("ctf_action", C.c_int), ("wiener", C.c_double),
                ("nmaps", C.c_int), ("fom", C.c_int), ("batch", C.c_int), ("device", C.c_int)]


class ReconStats(C.Structure):
    _fields_ = [("launches", C.c_long), ("insert_launches", C.c_long), ("insert_ms", C.c_double),
                ("fft2d_ms", C.c_double), ("h2d_ms", C.c_double), ("particles", C.c_long)]


class MatchConfig(C.Structure):
    _fields_ = [("n", C.c_int), ("map", C.c_int), ("map_sampling", C.c_double), ("pixel", C.c_double),
                ("hi_res", C.c_double), ("lo_res", C.c_double), ("kernel_width", C.c_int),
                ("kernel_power", C.c_int), ("batch", C.c_int), ("device", C.c_int)]


class MatchInfo(C.Structure):
    _fields_ = [("diam", C.c_int), ("npix", C.c_int), ("nshell", C.c_int), ("hi_res", C.c_double),
                ("max_rad", C.c_double), ("section_res", C.c_double), ("map_sampling_cut", C.c_double),
                ("pixel_cut", C.c_double)]


class MatchStats(C.Structure):
    _fields_ = [("panel_ms", C.c_double), ("agen_ms", C.c_double), ("gemm_ms", C.c_double),
                ("merge_ms", C.c_double), ("rescore_ms", C.c_double), ("local_ms", C.c_double),
                ("gemm_flops", C.c_double),
                ("hypotheses", C.c_double), ("launches", C.c_long), ("gemm_launches", C.c_long),
                ("images", C.c_long), ("rescored", C.c_long), ("coarse_k", C.c_int), ("kpad", C.c_int),
                ("refine_ms", C.c_double), ("refine_launches", C.c_long),
                ("panel_exact_ms", C.c_double), ("panel_exact_bytes", C.c_double)]


class BackprojConfig(C.Structure):
    _fields_ = [("n", C.c_int), ("map", C.c_int), ("pixel", C.c_double), ("resolution", C.c_double),
                ("nmaps", C.c_int), ("batch", C.c_int), ("device", C.c_int)]


BACKPROJ_DOUBLES = 16


class CnnConfig(C.Structure):
    _fields_ = [("box", C.c_int), ("channels", C.c_int * 6), ("hidden", C.c_int), ("batch", C.c_int),
                ("shift_weight", C.c_float), ("device", C.c_int), ("seed", C.c_ulonglong)]


CNN_RESULT_FLOATS = 11
MATCH_RESULT_DOUBLES = 5
MATCH_TOPK_MAX = 8
MATCH_APPLY_CTF = 1
MATCH_INVERT = 2
MATCH_CTF_DOUBLES = 8
MATCH_HYP_DOUBLES = 12
MATCH_REFINE_START_DOUBLES = 7
MATCH_SCORE_FP64 = 4
MATCH_SCORE_DPR = 8
MATCH_REFINE_RESULT_DOUBLES = 12
MATCH_PANEL_GATHER = 1


class BsgError(RuntimeError):
    pass


_lib = None


class ShellStats(C.Structure):
    """bsg_recon_shell_stats"""
    _fields_ = [("friedel", C.c_double), ("coverage", C.c_long), ("coverage_pct", C.c_double),
                ("res_snr", C.c_double), ("res_fsc", C.c_double), ("rows", C.c_int)]


STATS_COLUMNS = 9


def load():
    """Load libbsgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise BsgError(f"{LIB_PATH} is missing: run bsoft_b200.build.build() (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    vp, fp, dp = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_double)
    sig = {
        "bsg_recon_create": ([C.POINTER(ReconConfig), C.POINTER(vp)], C.c_int),
        "bsg_recon_destroy": ([vp], None),
        "bsg_recon_insert": ([vp, vp, vp, C.c_long, C.c_int], C.c_int),
        "bsg_recon_finish": ([vp, C.c_int, vp, vp, C.c_int], C.c_int),
        "bsg_recon_accumulators": ([vp, C.c_int, vp, vp, C.c_int], C.c_int),
        "bsg_recon_add_partial": ([vp, C.c_int, vp, vp, vp, vp, C.c_int], C.c_int),
        "bsg_recon_fsc": ([vp, C.c_int, dp], C.c_int),
        "bsg_recon_set_symmetrize": ([vp, dp, C.POINTER(C.c_int), C.c_int], C.c_int),
        "bsg_recon_set_rescale": ([vp, C.c_double, C.c_double], C.c_int),
        "bsg_recon_statistics": ([vp, C.c_int, C.c_double, C.POINTER(ShellStats), dp, C.c_int], C.c_int),
        "bsg_particle_spectra": ([vp, vp, vp, C.c_long, vp, C.c_int], C.c_int),
        "bsg_recon_set_timing": ([vp, C.c_int], C.c_int),
        "bsg_recon_set_tile_shape": ([vp, C.c_int], C.c_int),
        "bsg_recon_set_half_space": ([vp, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "bsg_recon_set_symmetry": ([vp, dp, C.c_int], C.c_int),
        "bsg_recon_autotune": ([vp, vp, vp, C.c_long, C.c_int, dp, C.POINTER(C.c_int)], C.c_int),
        "bsg_recon_get_stats": ([vp, C.POINTER(ReconStats)], C.c_int),
        "bsg_recon_reset": ([vp], C.c_int),
        "bsg_recon_synchronize": ([vp], C.c_int),
        "bsg_recon_stream": ([vp], vp),
        "bsg_match_create": ([C.POINTER(MatchConfig), C.POINTER(vp)], C.c_int),
        "bsg_match_destroy": ([vp], None),
        "bsg_match_info": ([vp, C.POINTER(MatchInfo)], C.c_int),
        "bsg_match_set_reference": ([vp, vp, dp, C.c_int], C.c_int),
        "bsg_match_reference_transform": ([vp, vp, C.c_int], C.c_int),
        "bsg_match_sections": ([vp, dp, C.c_long, vp, C.c_int], C.c_int),
        "bsg_match_set_images": ([vp, vp, C.c_long, dp, C.c_double, C.c_double, C.c_int], C.c_int),
        "bsg_match_prepared": ([vp, C.c_long, C.c_long, vp, C.c_int], C.c_int),
        "bsg_match_score": ([vp, dp, C.c_long, dp, dp, C.c_int], C.c_int),
        "bsg_match_set_shell_weights": ([vp, dp, C.c_int], C.c_int),
        "bsg_match_project": ([vp, dp, C.c_long, C.c_double, dp, dp, vp, C.c_int], C.c_int),
        "bsg_match_set_panel": ([vp, dp, C.c_long, C.c_int], C.c_int),
        "bsg_match_search": ([vp, dp, C.c_int, C.c_int, dp, C.c_int], C.c_int),
        "bsg_match_search_local": ([vp, vp, C.c_double, dp, C.c_int, C.c_double, C.c_int, dp, C.c_int], C.c_int),
        "bsg_match_get_stats": ([vp, C.POINTER(MatchStats)], C.c_int),
        "bsg_match_reset_stats": ([vp], C.c_int),
        "bsg_match_stream": ([vp], vp),
        "bsg_match_refine": ([vp, dp, C.c_long, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                              C.c_double, dp,
                              C.c_int],
                             C.c_int),
        "bsg_backproj_create": ([C.POINTER(BackprojConfig), C.POINTER(vp)], C.c_int),
        "bsg_backproj_destroy": ([vp], None),
        "bsg_backproj_add": ([vp, vp, dp, C.c_long, C.c_int], C.c_int),
        "bsg_backproj_finish": ([vp, C.c_int, vp, C.c_int], C.c_int),
        "bsg_backproj_set_symmetrize": ([vp, dp, C.POINTER(C.c_int), C.c_int], C.c_int),
        "bsg_backproj_set_rescale": ([vp, C.c_double, C.c_double], C.c_int),
        "bsg_backproj_reset": ([vp], C.c_int),
        "bsg_match_refine_monte": ([vp, dp, C.c_long, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_ulonglong, dp, C.c_int], C.c_int),
        "bsg_cnn_create": ([C.POINTER(CnnConfig), C.POINTER(vp)], C.c_int),
        "bsg_cnn_destroy": ([vp], None),
        "bsg_cnn_num_params": ([vp], C.c_long),
        "bsg_cnn_get_params": ([vp, fp], C.c_int),
        "bsg_cnn_set_params": ([vp, fp], C.c_int),
        "bsg_cnn_predict": ([vp, vp, C.c_long, vp, C.c_int], C.c_int),
        "bsg_cnn_loss_grad": ([vp, fp, fp, C.c_long, dp, fp], C.c_int),
        "bsg_cnn_train": ([vp, vp, vp, C.c_long, C.c_int, C.c_float, fp, C.c_int], C.c_int),
        "bsg_add_noise": ([vp, C.c_long, C.c_int, C.c_double, C.c_ulonglong, vp], C.c_int),
        "bsg_last_error": ([], C.c_char_p),
        "bsg_version": ([], C.c_char_p),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().bsg_last_error().decode(errors="replace")
        raise BsgError(f"{what} failed ({rc}): {msg}")
