"""Half-space gridding (bsg_recon_set_half_space): below z = zsplit the
tiles grid the pixels that have a Friedel mate in the stored transform and,
apart, the unpaired ones (row and column -ft/2); past the split only the
unpaired ones, the rest being read as the conjugate of the mirrored voxels.
Against gridding the full map on the same particles: the accumulators and
the finished maps agree to rounding (bit for bit in the tiles that no
unpaired pixel reaches), and so through every path that reads the sums
(finish, half maps and FSC, accumulators to the host and to the device,
partial-map sums); an Ewald batch switches the context to the full map
without losing what was gridded before it."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from bsoft_b200 import _lib
from bsoft_b200.plan import P_MAP, ReconPlan
from bsoft_b200.recon import Reconstructor
from bsoft_b200.synth import batched_insertion_workload
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def work():
    w = batched_insertion_workload(n_particles=96, box=64, pool=96, seed=12)
    return w, np.ascontiguousarray(w["pool"])


def _plan(w, nmaps=1, interp=2):
    return ReconPlan(n=64, ft=128, map=64, map_sampling=w["pixel"], hi_res=w["hi_res"], interp=interp,
                     ctf_action=1, wiener=0.0, params=w["params"], nmaps=nmaps)


def _run(plan, images, params, half_space, shape=0, batch=None):
    kw = {} if batch is None else {"batch": batch}
    with Reconstructor(plan, **kw) as rec:
        rec.set_tile_shape(shape)
        z = rec.set_half_space(half_space)
        rec.insert(images, params)
        v, wt = rec.accumulators(0)
        m = rec.finish(0)
    return z, v, wt, m


@pytest.mark.parametrize("shape", range(4))
def test_half_space_equals_full_map(work, shape):
    w, images = work
    plan = _plan(w)
    z1, v1, w1, m1 = _run(plan, images, w["params"], True, shape)
    z0, v0, w0, m0 = _run(plan, images, w["params"], False, shape)
    assert z1 == 40 and z0 == 0
    assert rel_l2(v1, v0) < 1e-6 and rel_l2(w1, w0) < 1e-6
    # the central tiles below the split, which no unpaired pixel reaches,
    # are gridded the same way, bit for bit; where the full map has nothing,
    # neither has the half-space one (but for a voxel reached only by a
    # trilinear corner whose FP32 weight rounds to zero in one of the two)
    c = np.r_[0:8, 56:64]
    core = np.ix_(np.arange(8), c, c)
    assert np.array_equal(v1[core], v0[core]) and np.array_equal(w1[core], w0[core])
    assert np.count_nonzero((w1 == 0) != (w0 == 0)) <= 4
    # finished maps: the FP32 tile sums' rounding, divided by small weights
    # at the fringe of the coverage, within the reference-parity bar
    assert rel_l2(m1, m0) < 1e-5
    # and the FP64 oracle's map
    ov, ow, _, _ = oracle.insert(plan, images, w["params"])
    assert rel_l2(v1.reshape(-1), ov.view(np.complex128)) < 1e-6
    om, _ = oracle.finish(plan, ov, ow)
    assert rel_l2(m1, om) < 1e-5


def test_half_space_only_for_trilinear(work):
    w, _ = work
    for interp in (0, 1):
        with Reconstructor(_plan(w, interp=interp)) as rec:
            assert rec.set_half_space(True) == 0


def test_half_space_reproducible_and_batch_invariant(work):
    w, images = work
    plan = _plan(w)
    a = _run(plan, images, w["params"], True)
    b = _run(plan, images, w["params"], True)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
    c = _run(plan, images, w["params"], True, batch=17)
    assert rel_l2(c[1], a[1]) < 1e-6 and rel_l2(c[3], a[3]) < 1e-6


def test_half_space_half_maps_and_fsc(work):
    w, images = work
    P = w["params"].copy()
    P[:, P_MAP] = np.arange(len(P)) % 2
    out = {}
    for hs in (True, False):
        with Reconstructor(_plan(w, nmaps=3)) as rec:
            rec.set_half_space(hs)
            rec.insert(images, P)
            out[hs] = ([rec.finish(i) for i in range(3)], rec.fsc())
    for i in range(3):
        assert rel_l2(out[True][0][i], out[False][0][i]) < 1e-5
    assert np.abs(out[True][1] - out[False][1]).max() < 1e-6


def test_half_space_device_accumulators(work):
    w, images = work
    plan = _plan(w)
    N = plan.map
    with Reconstructor(plan) as rec:
        assert rec.set_half_space(True) > 0
        rec.insert(images, w["params"])
        v, wt = rec.accumulators(0)
        dv = torch.empty((N, N, N, 2), dtype=torch.float64, device="cuda")
        dw = torch.empty((N, N, N), dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().bsg_recon_accumulators(rec._h, 0, C.c_void_p(dv.data_ptr()),
                                                      C.c_void_p(dw.data_ptr()), _lib.BSG_DEVICE_PTR),
                   "bsg_recon_accumulators")
        torch.cuda.synchronize()
        hv = dv.cpu().numpy()
        assert np.array_equal(hv[..., 0] + 1j * hv[..., 1], v) and np.array_equal(dw.cpu().numpy(), wt)


def test_half_space_partial_maps(work):
    """Shard 1's accumulators (the map's sums) added into a half-space
    context that gridded shard 0: the one-pass sums to FP64 rounding."""
    w, images = work
    plan = _plan(w)
    P = w["params"]
    s0, s1 = np.arange(0, 48), np.arange(48, 96)
    with Reconstructor(plan) as a, Reconstructor(plan) as b, Reconstructor(plan) as one:
        a.insert(images[s0], P[s0])
        b.insert(images[s1], P[s1])
        one.insert(images[s0], P[s0])
        one.insert(images[s1], P[s1])
        vb, wb = b.accumulators(0)
        a.add_partial(vb, wb, 0)                # a now holds a full map's sums
        va, wa = a.accumulators(0)
        vo, wo = one.accumulators(0)
        assert rel_l2(va, vo) < 1e-13 and rel_l2(wa, wo) < 1e-13
        assert np.array_equal(wa == 0, wo == 0)  # the same contributions, none subtracted
        assert rel_l2(a.finish(0), one.finish(0)) < 1e-6
        with pytest.raises(_lib.BsgError):
            a.set_half_space(True)              # only with empty accumulators
        a.reset()
        assert a.set_half_space(True) == 40


def test_half_space_not_switched_on_over_added_sums(work):
    """A fresh context given another's sums by add_partial holds a full map:
    half-space gridding stays off until reset, as after inserting."""
    w, images = work
    plan = _plan(w)
    with Reconstructor(plan) as a, Reconstructor(plan) as b:
        b.insert(images, w["params"])
        vb, wb = b.accumulators(0)
        a.add_partial(vb, wb, 0)
        with pytest.raises(_lib.BsgError):
            a.set_half_space(True)
        va, wa = a.accumulators(0)
        assert np.array_equal(va, vb) and np.array_equal(wa, wb)


def test_ewald_batch_switches_to_full_map(work):
    """A plane batch gridded in half-space form, then an Ewald batch: the
    context switches to the full map and holds both batches' sums."""
    w, images = work
    plan = _plan(w)
    P = w["params"].copy()
    P[48:, 26] = 0.025079336205768955
    with Reconstructor(plan) as rec:
        assert rec.set_half_space(True) > 0
        rec.insert(images[:48], P[:48])
        rec.insert(images[48:], P[48:])
        assert rec.set_half_space(True) == 0       # off for good
        v, wt = rec.accumulators(0)
    with Reconstructor(plan) as ref:
        ref.set_half_space(False)
        ref.insert(images[:48], P[:48])
        ref.insert(images[48:], P[48:])
        v0, w0 = ref.accumulators(0)
    assert rel_l2(v, v0) < 1e-6 and rel_l2(wt, w0) < 1e-6
    ov, ow, _, _ = oracle.insert(plan, images, P)
    assert rel_l2(v.reshape(-1), ov.view(np.complex128)) < 1e-6


def test_full_size_half_space_against_full_map():
    """At the batched-insertion size (256^2, ft 512, 256^3)."""
    w = batched_insertion_workload(n_particles=64, box=256, pool=64, seed=5)
    images = np.ascontiguousarray(w["pool"])
    plan = ReconPlan(n=256, ft=512, map=256, map_sampling=w["pixel"], hi_res=w["hi_res"], interp=2,
                     ctf_action=1, wiener=0.0, params=w["params"], nmaps=1)
    z1, v1, w1, m1 = _run(plan, images, w["params"], True)
    z0, v0, w0, m0 = _run(plan, images, w["params"], False)
    assert z1 == 136 and z0 == 0
    assert rel_l2(v1, v0) < 1e-6 and rel_l2(w1, w0) < 1e-6 and rel_l2(m1, m0) < 1e-5
