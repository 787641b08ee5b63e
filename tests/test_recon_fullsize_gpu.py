"""Gridding at the batched-insertion workload's full size (256^2 particles,
pad 2 -> 512^2 transforms, 256^3 map, trilinear, CTF flip), through
properties that do not need a full reference run: agreement with the FP64
oracle on a subset, bitwise reproducibility, invariance to batching and
call splitting, and half maps that sum to the full map."""
import numpy as np
import pytest

import oracle
from bsoft_b200.plan import P_MAP, ReconPlan
from bsoft_b200.recon import Reconstructor
from bsoft_b200.synth import batched_insertion_workload
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu
BOX = 256


@pytest.fixture(scope="module")
def work():
    w = batched_insertion_workload(n_particles=320, box=BOX, pool=32, seed=5)
    images = np.ascontiguousarray(w["pool"][np.arange(320) % 32])
    return w, images


def _plan(w, nmaps=1):
    return ReconPlan(n=BOX, ft=2 * BOX, map=BOX, map_sampling=w["pixel"], hi_res=w["hi_res"], interp=2,
                     ctf_action=1, wiener=0.0, params=w["params"], nmaps=nmaps)


def test_full_size_against_fp64_oracle(work):
    w, images = work
    plan = _plan(w)
    n = 12
    with Reconstructor(plan) as rec:
        rec.insert(images[:n], w["params"][:n])
        v, wt = rec.accumulators(0)
    ov, ow, _, _ = oracle.insert(plan, images[:n], w["params"][:n])
    assert rel_l2(v.reshape(-1), ov.view(np.complex128)) < 1e-6
    assert rel_l2(wt.reshape(-1), ow) < 1e-6


def test_full_size_reproducible_and_batch_invariant(work):
    w, images = work
    plan = _plan(w)
    P = w["params"]
    runs = []
    for _ in range(2):
        with Reconstructor(plan) as rec:
            rec.insert(images, P)
            runs.append(rec.accumulators(0))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    with Reconstructor(plan, batch=77) as rec:
        rec.insert(images[:150], P[:150])
        rec.insert(images[150:], P[150:])
        v, wt = rec.accumulators(0)
    assert rel_l2(v, runs[0][0]) < 1e-6 and rel_l2(wt, runs[0][1]) < 1e-6


def test_full_size_half_maps(work):
    """Half maps hold the even and odd particles' sums; the full map made
    from them equals a full-map reconstruction."""
    w, images = work
    P = w["params"].copy()
    P[:, P_MAP] = np.arange(len(P)) % 2
    with Reconstructor(_plan(w, nmaps=3)) as rec:
        rec.insert(images, P)
        halves = [rec.accumulators(h) for h in (0, 1)]
        full_from_halves = rec.finish(0)
    for h, sel in ((0, slice(0, None, 2)), (1, slice(1, None, 2))):
        with Reconstructor(_plan(w)) as rec:
            rec.insert(images[sel], P[sel])
            v, wt = rec.accumulators(0)
        assert rel_l2(halves[h][0], v) < 1e-6 and rel_l2(halves[h][1], wt) < 1e-6
    with Reconstructor(_plan(w)) as rec:
        rec.insert(images, P)
        full = rec.finish(0)
    assert rel_l2(full_from_halves, full) < 1e-5
