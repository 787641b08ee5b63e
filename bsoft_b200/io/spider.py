"""SPIDER image / stack reading (host side, numpy).

Follows the reference's SPIDER reader (bsoft/src/rwimg/rwSPIDER.cpp:82-243)
for real-space float stacks, the form particle stacks take:

* 1024-float header words as floats: nslice (0), nrow (1), iform (4), av (8),
  sig (9), nsam (11), xoff/yoff/zoff (17-19), scale (20), labbyt (21),
  istack (23), maxim (25);
* byte order: the header's 4-byte words are swapped when |nslice| or |iform|
  exceeds 65535 or |nslice| < 1 (the reference's test), and so is the data;
* a stack (istack > 0) holds maxim images after the global header; image i
  is a labbyt-byte image header followed by its data at
  labbyt + i (labbyt + 4 nsam nrow nslice);
* sampling = scale on every axis; each image's origin comes from its own
  header (xoff, yoff, zoff), the centre the reference uses for the
  background estimate.

Fourier-transform files (iform < 0) are not particle stacks and are refused.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SWAPTRIG = 65535
HEADER_WORDS = 256          # floats of the SPIDERhead structure read (1024 bytes)


@dataclass
class SpiderHeader:
    nx: int
    ny: int
    nz: int
    iform: float
    labbyt: int
    istack: float
    maxim: int
    scale: float
    av: float
    sig: float
    swap: bool
    origins: np.ndarray = field(default_factory=lambda: np.zeros((1, 3)))   # per image (pixels)

    @property
    def sampling(self):
        s = self.scale
        return (s, s, s)

    @property
    def n_images(self):
        return self.maxim if self.istack > 0 else 1

    @property
    def image_bytes(self):
        return self.labbyt + 4 * self.nx * self.ny * self.nz

    def data_offset(self, i: int) -> int:
        """Byte offset of image i's data."""
        if self.istack > 0:
            return self.labbyt + i * self.image_bytes + self.labbyt
        return self.labbyt

    @property
    def file_stats(self):
        """(average, standard deviation) read_img attaches (the global header's)."""
        return float(self.av), float(self.sig)

    def image_origin_of(self, i: int):
        return tuple(float(v) for v in self.origins[min(i, len(self.origins) - 1)])


def _words(raw: bytes, swap: bool) -> np.ndarray:
    return np.frombuffer(raw[:4 * HEADER_WORDS], dtype=">f4" if swap else "<f4").astype(np.float64)


def is_spider(path: str) -> bool:
    p = path.lower()
    return p.endswith(".spi") or p.endswith(".spider")


def read_header(path: str) -> SpiderHeader:
    with open(path, "rb") as f:
        raw = f.read(4 * HEADER_WORDS)
        if len(raw) < 4 * HEADER_WORDS:
            raise ValueError(f"{path}: short SPIDER header")
        w = _words(raw, False)
        swap = abs(w[0]) > SWAPTRIG or abs(w[4]) > SWAPTRIG or abs(w[0]) < 1
        if swap:
            w = _words(raw, True)
        h = SpiderHeader(nx=int(w[11]), ny=int(w[1]), nz=int(w[0]), iform=float(w[4]), labbyt=int(w[21]),
                         istack=float(w[23]), maxim=int(w[25]), scale=float(w[20]), av=float(w[8]),
                         sig=float(w[9]), swap=swap)
        if h.nx < 1 or h.ny < 1 or h.nz < 1 or h.labbyt < 4 * 36:
            raise ValueError(f"{path}: not a valid SPIDER image (nsam={h.nx} nrow={h.ny} nslice={h.nz})")
        if h.iform < 0:
            raise ValueError(f"{path}: SPIDER Fourier transforms are not particle stacks")
        org = np.zeros((h.n_images, 3))
        if h.istack > 0:
            for i in range(h.n_images):
                f.seek(h.labbyt + i * h.image_bytes)
                wi = _words(f.read(4 * HEADER_WORDS), swap)
                org[i] = wi[17:20]
        else:
            org[0] = w[17:20]
        h.origins = org
    return h


def read_stack(path: str, first: int = 0, count: int | None = None) -> tuple[np.ndarray, SpiderHeader]:
    """Float32 images [first, first+count) -> (n, ny, nx) (slices of a volume
    image stay along the first axis of each image)."""
    h = read_header(path)
    n = h.n_images
    count = n - first if count is None else count
    if first < 0 or count < 0 or first + count > n:
        raise ValueError(f"{path}: images [{first}, {first + count}) outside the {n} images of the file")
    per = h.nx * h.ny * h.nz
    out = np.empty((count, h.nz * h.ny, h.nx) if h.nz > 1 else (count, h.ny, h.nx), dtype=np.float32)
    dt = ">f4" if h.swap else "<f4"
    with open(path, "rb") as f:
        for j in range(count):
            f.seek(h.data_offset(first + j))
            a = np.frombuffer(f.read(4 * per), dtype=dt)
            if a.size != per:
                raise ValueError(f"{path}: truncated data")
            out[j] = a.astype(np.float32).reshape(out.shape[1:])
    return out, h
