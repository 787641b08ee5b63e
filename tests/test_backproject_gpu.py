"""Real-space weighted back-projection on the GPU (bsg_backproj_*,
bsoft_b200/csrc/backproj.cu) against the reference's own maps: the
back-projection probe's (Bimage::back_project over seeded images and views,
tests/golden/backproject.npz) and bbackproj's on STAR projects, with half
maps, symmetry and rescaling (tests/golden/bbackproj.npz), and against the
FP64 oracle (oracle/backproject_oracle.py).  Tolerance: relative L2 <= 1e-5
(the reference transforms in float; the oracle is within 1e-7 of it)."""
import os

import numpy as np
import pytest

from bsoft_b200.backproj import (B_MAP, BackProjector, BackprojPlan, load_images, plan_backprojection,
                                 records_from_views)
from bsoft_b200.project import read_project
from oracle.backproject_oracle import back_projection
from tests.helpers import GOLDEN, backproj_options_from_args, materialize_dataset, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _probe_case(key):
    z = np.load(os.path.join(GOLDEN, "backproject.npz"))
    pixel, res, N = (float(v) for v in z[f"{key}_scalars"])
    imgs, params = z[f"{key}_images"], z[f"{key}_params"]
    n = imgs.shape[1]
    plan = BackprojPlan(n=n, map=int(N), map_sampling=pixel, pixel=pixel, resolution=res,
                        records=records_from_views(params[:, :2], params[:, 2:]))
    return plan, imgs, params, z[f"{key}_map"]


@pytest.mark.parametrize("key", ["a", "b"])
def test_backprojection_matches_reference_probe(key):
    """Even images into an equal map (power-of-two transforms) and odd
    images (15 = 3 x 5: the mixed-radix transforms) into a larger map."""
    plan, imgs, params, ref = _probe_case(key)
    with BackProjector(plan) as bp:
        bp.add(imgs, plan.records)
        m = bp.finish()
    assert rel_l2(m, ref) <= TOL, rel_l2(m, ref)
    orc = back_projection(imgs, params, plan.map, plan.resolution, plan.pixel)
    assert rel_l2(m, orc) <= TOL


def test_backprojection_batch_invariant():
    """The map is the same to the bit whatever the batch size: the float
    accumulation runs image by image in order."""
    plan, imgs, _, _ = _probe_case("b")
    maps = []
    for batch in (0, 1, 4):
        with BackProjector(plan, batch=batch) as bp:
            bp.add(imgs[:2], plan.records[:2])
            bp.add(imgs[2:], plan.records[2:])
            maps.append(bp.finish())
    assert np.array_equal(maps[0], maps[1]) and np.array_equal(maps[0], maps[2])


BBACKPROJ_CASES = ["ctf16_bp", "plain24_bp", "plain24_bp_half", "plain24_bp_full_half", "plain24_bp_d2",
                   "ctf16_bp_rs"]


@pytest.mark.parametrize("case", BBACKPROJ_CASES)
def test_bbackproj_matches_reference(case, tmp_path):
    """bbackproj on a STAR project: origins, views and pixel sizes resolved
    as project_back_projection does, half maps from the round-robin partial
    maps, -symmetry and -rescale of the finished map."""
    z = np.load(os.path.join(GOLDEN, "bbackproj.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    plan = plan_backprojection(read_project(star), backproj_options_from_args(str(z[case + "__options"])))
    images = load_images(plan)
    keys = [k for k in z.files if k.startswith(case + "__map")]
    assert keys
    with BackProjector(plan) as bp:
        bp.add(images, plan.records)
        for k in keys:
            tag = k[len(case) + 5:]
            imap = 0 if not tag else int(tag[1:])
            m = bp.finish(imap)
            assert rel_l2(m, z[k]) <= TOL, (k, rel_l2(m, z[k]))


def test_backprojection_larger_map_against_oracle():
    """64^2 images into a 64^3 map at a fine limit, and 48^2 (mixed radix)
    images with origins off centre and magnification 1, against the FP64
    oracle."""
    rng = np.random.default_rng(7)
    for n, N, K in ((64, 64, 12), (48, 56, 10)):
        imgs = rng.standard_normal((K, n, n)).astype(np.float32)
        imgs[:, n // 3:n // 2, n // 4:n // 2] += 2.0
        v = rng.standard_normal((K, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        views = np.concatenate([v, rng.uniform(-np.pi, np.pi, (K, 1))], axis=1)
        origins = n / 2 + rng.uniform(-2, 2, (K, 2))
        plan = BackprojPlan(n=n, map=N, map_sampling=1.2, pixel=1.2, resolution=3.0,
                            records=records_from_views(origins, views))
        with BackProjector(plan) as bp:
            bp.add(imgs, plan.records)
            m = bp.finish()
        params = np.concatenate([origins, views], axis=1)
        orc = back_projection(imgs, params, N, 3.0, 1.2)
        assert rel_l2(m, orc) <= TOL, (n, rel_l2(m, orc))


def test_backprojection_rejects_bad_records():
    plan, imgs, _, _ = _probe_case("a")
    r = plan.records.copy()
    r[0, B_MAP] = 1        # a second half map without half maps
    with BackProjector(plan) as bp:
        with pytest.raises(Exception):
            bp.add(imgs, r)
