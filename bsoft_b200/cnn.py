"""Learned orientation proposer (libbsgpu's bsg_cnn_*): a convolutional
network trained on the GPU by the library's own kernels to map a particle
image to a rotation and a shift, used to restrict the orientation search to
the neighbourhood of its proposal.

    net = Proposer(box=128)
    net.train(images_dev, targets_dev, steps=2000, lr=1e-3)   # CUDA tensors
    pose = net.predict(images)          # (n, 11): R row-major (9), shift (2)

Targets are rows of 11 floats: the true rotation (row-major) and the shift
of the particle from the box centre in pixels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

DEFAULT_CHANNELS = (32, 64, 64, 128, 128, 128)


def _ptr(a):
    if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
        return C.c_void_p(a.data_ptr()), True
    return C.c_void_p(a.ctypes.data), False


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Proposer:
    def __init__(self, box: int = 128, channels=DEFAULT_CHANNELS, hidden: int = 1024, batch: int = 256,
                 shift_weight: float = 0.05, seed: int = 1, device: int = 0):
        L = _lib.load()
        ch = (C.c_int * 6)(*channels)
        cfg = _lib.CnnConfig(box, ch, hidden, batch, shift_weight, device, seed)
        h = C.c_void_p()
        _lib.check(L.bsg_cnn_create(C.byref(cfg), C.byref(h)), "bsg_cnn_create")
        self._h = h
        self.box = box
        self.channels = tuple(channels)
        self.hidden = hidden
        self.nparams = int(L.bsg_cnn_num_params(h))

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().bsg_cnn_destroy(self._h)
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

    def get_params(self) -> np.ndarray:
        out = np.empty(self.nparams, dtype=np.float32)
        _lib.check(_lib.load().bsg_cnn_get_params(self._h, _fp(out)), "bsg_cnn_get_params")
        return out

    def set_params(self, p) -> None:
        a = np.ascontiguousarray(p, dtype=np.float32)
        if a.size != self.nparams:
            raise ValueError(f"expected {self.nparams} parameters, got {a.size}")
        _lib.check(_lib.load().bsg_cnn_set_params(self._h, _fp(a)), "bsg_cnn_set_params")

    def predict(self, images, out=None):
        if not (hasattr(images, "data_ptr") and getattr(images, "is_cuda", False)):
            images = np.ascontiguousarray(images, dtype=np.float32)
        n = images.shape[0]
        if out is None:
            out = np.empty((n, _lib.CNN_RESULT_FLOATS), dtype=np.float32)
        p, dev = _ptr(images)
        q, qdev = _ptr(out)
        if dev != qdev:
            raise ValueError("images and out must both be on the host or both on the device")
        _lib.check(_lib.load().bsg_cnn_predict(self._h, p, n, q, _lib.BSG_DEVICE_PTR if dev else 0),
                   "bsg_cnn_predict")
        return out

    def loss_grad(self, images, targets):
        x = np.ascontiguousarray(images, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.empty(self.nparams, dtype=np.float32)
        loss = C.c_double()
        _lib.check(_lib.load().bsg_cnn_loss_grad(self._h, _fp(x), _fp(t), len(x), C.byref(loss), _fp(g)),
                   "bsg_cnn_loss_grad")
        return loss.value, g

    def train(self, images, targets, steps: int, lr: float = 1e-3) -> np.ndarray:
        """`steps` Adam steps; images (n, box, box) and targets (n, 11) are
        CUDA tensors.  Returns the mean loss of each step."""
        losses = np.empty(steps, dtype=np.float32)
        p, _ = _ptr(images)
        q, _ = _ptr(targets)
        _lib.check(_lib.load().bsg_cnn_train(self._h, p, q, images.shape[0], steps, lr, _fp(losses),
                                             _lib.BSG_DEVICE_PTR), "bsg_cnn_train")
        return losses


def pose_targets(mats: np.ndarray, shifts: np.ndarray) -> np.ndarray:
    """Targets (n, 11) from rotation matrices (n, 3, 3) and shifts (n, 2)."""
    m = np.asarray(mats, dtype=np.float64).reshape(-1, 9)
    return np.concatenate([m, np.asarray(shifts, dtype=np.float64).reshape(-1, 2)], axis=1).astype(np.float32)


def add_noise(images, snr: float, seed: int = 1) -> None:
    """Add Gaussian noise in place to CUDA images (n, box, box) at `snr`."""
    n, box = images.shape[0], images.shape[1]
    _lib.check(_lib.load().bsg_add_noise(C.c_void_p(images.data_ptr()), n, box, float(snr), seed, None),
               "bsg_add_noise")
