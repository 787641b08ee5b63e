"""The CUDA orientation-proposer network against its FP64 oracle (loss and
every parameter gradient), and training on projections made by the
library's own projector."""
import math

import numpy as np
import pytest

from oracle import cnn_oracle as co

pytestmark = pytest.mark.gpu

BOX, CH, HID = 64, (4, 8, 8, 16, 16, 16), 32


def _case(seed=0, B=5):
    rng = np.random.default_rng(seed)
    lay = co.layout(BOX, CH, HID)
    n = sum(int(np.prod(s)) for _, s in lay)
    w = np.zeros(n, dtype=np.float32)
    off = 0
    for name, shape in lay:
        k = int(np.prod(shape))
        fan = int(np.prod(shape[1:])) if len(shape) > 1 else 1
        if name.endswith(".W"):
            w[off:off + k] = rng.normal(scale=math.sqrt(2.0 / fan), size=k)
        else:
            w[off:off + k] = rng.normal(scale=0.1, size=k)
        off += k
    imgs = rng.normal(size=(B, BOX, BOX)).astype(np.float32)
    from bsoft_b200.geometry import random_views, views_to_matrices
    R = views_to_matrices(random_views(rng, B))
    t = rng.uniform(-2, 2, size=(B, 2))
    tgt = np.concatenate([R.reshape(B, 9), t], axis=1).astype(np.float32)
    return w, imgs, tgt


def test_parameter_count():
    from bsoft_b200.cnn import Proposer
    with Proposer(box=BOX, channels=CH, hidden=HID, batch=8) as net:
        lay = co.layout(BOX, CH, HID)
        assert net.nparams == sum(int(np.prod(s)) for _, s in lay)
    with Proposer(box=128) as net:
        assert 0.9e6 < net.nparams < 1.1e6


def test_loss_and_gradients_match_oracle():
    from bsoft_b200.cnn import Proposer
    w, imgs, tgt = _case()
    with Proposer(box=BOX, channels=CH, hidden=HID, batch=8) as net:
        net.set_params(w)
        assert np.array_equal(net.get_params(), w)
        loss, g = net.loss_grad(imgs, tgt)
    R, t, L, go = co.forward_backward(w, imgs, tgt, BOX, CH, HID)
    assert abs(loss - L) < 1e-4 * max(1.0, abs(L))
    off = 0
    for name, shape in co.layout(BOX, CH, HID):
        k = int(np.prod(shape))
        a, b = g[off:off + k].astype(np.float64), go[off:off + k]
        off += k
        nb = np.linalg.norm(b)
        if nb == 0:
            assert np.linalg.norm(a) < 1e-6, name
            continue
        assert np.linalg.norm(a - b) / nb < 2e-3, name


def test_predict_matches_oracle():
    from bsoft_b200.cnn import Proposer
    w, imgs, tgt = _case(3)
    with Proposer(box=BOX, channels=CH, hidden=HID, batch=4) as net:
        net.set_params(w)
        out = net.predict(imgs)          # two chunks of 4 and 1
    R, t, _, _ = co.forward_backward(w, imgs, None, BOX, CH, HID)
    assert np.abs(out[:, :9].reshape(-1, 3, 3) - R).max() < 2e-3
    assert np.abs(out[:, 9:] - t).max() < 2e-3 * max(1.0, np.abs(t).max())


def test_training_reduces_loss():
    """A few hundred Adam steps on projections of one map (the library's
    projector with CTF) bring the pose loss well below its start."""
    import torch
    from bsoft_b200.cnn import Proposer, pose_targets
    from bsoft_b200.match import Matcher, ctf_record
    from bsoft_b200.geometry import random_views, views_to_matrices
    from tests.match_helpers import load
    d = load("match64")
    rng = np.random.default_rng(5)
    n = 4096
    mats = views_to_matrices(random_views(rng, n))
    shifts = rng.uniform(-2, 2, size=(n, 2))
    m = Matcher(n=64, map=64, map_sampling=d["pixel"], pixel=d["pixel"], hi_res=2 * d["pixel"])
    m.set_reference(d["map"], d["map_origin"])
    ctf = np.stack([ctf_record(200000.0, d["ctf_rows"][i % 4][1:6]) for i in range(n)])
    imgs = torch.empty((n, 64, 64), dtype=torch.float32, device="cuda")
    m.project(mats, origins=32 + shifts, ctf=ctf, out=imgs)
    m.close()
    tg = torch.from_numpy(pose_targets(mats, shifts)).cuda()
    with Proposer(box=64, channels=(16, 32, 32, 64, 64, 64), hidden=256, batch=128, seed=3) as net:
        losses = net.train(imgs, tg, steps=400, lr=1e-3)
        again = Proposer(box=64, channels=(16, 32, 32, 64, 64, 64), hidden=256, batch=128, seed=3)
        l2 = again.train(imgs, tg, steps=20, lr=1e-3)
        again.close()
    assert np.all(np.isfinite(losses))
    assert losses[-50:].mean() < 0.6 * losses[:20].mean()
    assert np.array_equal(l2, losses[:20])          # reproducible for a seed
