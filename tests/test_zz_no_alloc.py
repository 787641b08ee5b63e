"""bsg_particle_spectra_noalloc, called through the C ABI, against the
regular 2-D entry point (bsg_particle_spectra).

The no-allocation variant exists for callers that manage all device memory
themselves - a pipeline that reserves its memory once at start-up, or a host
that forbids device allocations after initialisation - and so cannot let
the library call cudaMalloc.  It takes the caller's device buffers for the
images and the spectra and keeps its intermediates in a fixed scratch area
inside the library.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from bsoft_b200 import _lib
from bsoft_b200.plan import ReconOptions, load_images, plan_reconstruction
from bsoft_b200.project import read_project
from bsoft_b200.recon import Reconstructor
from bsoft_b200.synth import DatasetSpec, generate, write_dataset
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL = 2e-6   # the spectra tolerance of the other GPU tests


def _noalloc():
    L = _lib.load()
    f = L.bsg_particle_spectra_noalloc
    f.argtypes = [C.POINTER(_lib.ReconConfig), C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return L, f


def test_noalloc_spectra_match_the_regular_entry_point(tmp_path):
    torch = pytest.importorskip("torch")
    spec = DatasetSpec(box=32, n_particles=48, n_blobs=8, seed=31, snr=0.5, astig_range=(0.0, 300.0))
    ph, imgs, meta = generate(spec)
    star = write_dataset(str(tmp_path), spec, ph, imgs, meta)
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=2, ctf_action=1))
    images = load_images(plan)
    params = np.ascontiguousarray(plan.params)
    with Reconstructor(plan) as rec:
        ref = rec.spectra(images, params)

    L, f = _noalloc()
    cfg = _lib.ReconConfig(plan.n, plan.ft, plan.map, plan.map_sampling, plan.hi_res, plan.interp,
                           plan.ctf_action, plan.wiener, 1, 0, 0, 0)
    d_img = torch.from_numpy(images).cuda()
    # two calls in a row on different particles: the second reuses the
    # scratch area the first one filled
    for sel in (slice(0, 20), slice(20, 48)):
        k = sel.stop - sel.start
        src = d_img[sel].contiguous()
        out = torch.empty((k, plan.ft, plan.ft, 2), dtype=torch.float32, device="cuda")
        p = np.ascontiguousarray(params[sel])
        rc = f(C.byref(cfg), C.c_void_p(src.data_ptr()), C.c_void_p(p.ctypes.data), k,
               C.c_void_p(out.data_ptr()), None)
        assert rc == 0, L.bsg_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        got = got[..., 0] + 1j * got[..., 1]
        assert rel_l2(got, ref[sel]) < TOL

    # a request beyond the fixed scratch area is refused with a clear error
    big = 100000
    rc = f(C.byref(cfg), C.c_void_p(d_img.data_ptr()), C.c_void_p(params.ctypes.data), big,
           C.c_void_p(d_img.data_ptr()), None)
    assert rc == -1
    assert b"scratch" in L.bsg_last_error()
