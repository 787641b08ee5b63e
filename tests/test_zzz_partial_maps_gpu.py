"""bsg_recon_add_partial on the GPU: the partial-map sum of a reconstruction
split into shards (bsoft_b200.shard).  A context that grids shard 0 and then
adds shard 1's accumulators must hold exactly the sums of one context that
grids shard 0 and then shard 1 as its two batches (each batch's sums are
added to the FP64 accumulators once, so both orders of operations are the
same additions); the finished maps then match the FP64 oracle."""
import numpy as np
import pytest

import oracle
from bsoft_b200._lib import BsgError
from bsoft_b200.recon import Reconstructor
from bsoft_b200.shard import shard_indices
from tests.helpers import load_case, rel_l2

pytestmark = pytest.mark.gpu


def test_add_partial_equals_one_pass(tmp_path):
    plan, images, _ = load_case("ctf16_tri_flip", str(tmp_path))
    n = len(plan.params)
    s0, s1 = shard_indices(n, 0, 2), shard_indices(n, 1, 2)
    with Reconstructor(plan) as a, Reconstructor(plan) as b, Reconstructor(plan) as one:
        a.insert(images[s0], plan.params[s0])
        b.insert(images[s1], plan.params[s1])
        one.insert(images[s0], plan.params[s0])
        one.insert(images[s1], plan.params[s1])
        vb, wb = b.accumulators(0)
        a.add_partial(vb, wb, 0)
        va, wa = a.accumulators(0)
        vo, wo = one.accumulators(0)
        assert np.array_equal(va, vo) and np.array_equal(wa, wo)
        m = a.finish(0)
    order = np.concatenate([s0, s1])
    vol, w, _, _ = oracle.insert(plan, images[order], plan.params[order])
    orc, _ = oracle.finish(plan, vol, w)
    assert rel_l2(m, orc) < 1e-5, rel_l2(m, orc)


def test_add_partial_rejects_bad_arguments(tmp_path):
    plan, images, _ = load_case("ctf16_tri_flip", str(tmp_path))
    with Reconstructor(plan) as a:
        v, w = a.accumulators(0)
        with pytest.raises(BsgError):
            a.add_partial(v, w, 1)          # one map: no half 1
        with pytest.raises(ValueError):
            a.add_partial(v, w[:2], 0)
