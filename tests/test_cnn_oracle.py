"""The FP64 oracle of the orientation-proposer network: its analytic
gradients against central finite differences of its own loss."""
import numpy as np

from oracle import cnn_oracle as co

BOX, CH, HID = 64, (3, 4, 4, 5, 5, 6), 7


def _setup(seed=0, B=3):
    rng = np.random.default_rng(seed)
    lay = co.layout(BOX, CH, HID)
    n = sum(int(np.prod(s)) for _, s in lay)
    w = rng.normal(scale=0.4, size=n)
    imgs = rng.normal(size=(B, BOX, BOX))
    q = rng.normal(size=(B, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    from bsoft_b200.geometry import quaternion_to_matrix
    R = np.stack([quaternion_to_matrix(x) for x in q])
    t = rng.uniform(-2, 2, size=(B, 2))
    tgt = np.concatenate([R.reshape(B, 9), t], axis=1)
    return w, imgs, tgt


def test_layout_counts():
    lay = co.layout(128, (32, 64, 64, 128, 128, 128), 1024)
    n = sum(int(np.prod(s)) for _, s in lay)
    assert 0.9e6 < n < 1.1e6          # ~1M parameters


def test_gradients_finite_differences():
    w, imgs, tgt = _setup()
    _, _, L, g = co.forward_backward(w, imgs, tgt, BOX, CH, HID, rounded=False)
    rng = np.random.default_rng(1)
    idx = rng.choice(w.size, size=40, replace=False)
    eps = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        lp = co.forward_backward(wp, imgs, tgt, BOX, CH, HID, rounded=False)[2]
        lm = co.forward_backward(wm, imgs, tgt, BOX, CH, HID, rounded=False)[2]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) < 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_head_is_a_rotation():
    o = np.random.default_rng(2).normal(size=(5, 8))
    R, t, _, _ = co._head(o, None, 0.05)
    for r in R:
        assert np.allclose(r.T @ r, np.eye(3), atol=1e-10)
        assert abs(np.linalg.det(r) - 1) < 1e-10


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.001953125, -3.1415927, 1e-3], dtype=np.float32)
    r = co.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0078125 or r[1] == 1.0       # ties to even
    assert r[2] == 1.0                                             # below half an ulp
    assert abs(r[3] + 3.140625) < 1e-7
