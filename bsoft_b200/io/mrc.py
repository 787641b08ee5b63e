"""MRC image / stack reading and writing (host side, numpy).

Mirrors the subset of the reference's MRC reader that the reconstruction path
relies on (bsoft/src/rwimg/rwMRC.cpp:60-215):

* 1024-byte header, mode 2 (float32) data, x fastest;
* header version >= 20140: ``nz / mz`` sub-images of ``mz`` slices each, so a
  particle stack is written with ``mz = 1``;
* sampling = cell / m{x,y,z};
* image origin (pixels) = -origin_field / sampling (rwMRC.cpp:195), which is
  the centre the reference uses for its background estimate
  (bsoft/src/img/Bimage_background.cpp:27-80).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np

HEADER_BYTES = 1024


@dataclass
class MRCHeader:
    nx: int
    ny: int
    nz: int
    mode: int
    mx: int
    my: int
    mz: int
    cell: tuple
    origin: tuple          # the header's origin field (angstrom)
    nsymbt: int
    nversion: int
    dmean: float = 0.0     # header average and rms: the statistics read_img
    rms: float = 0.0       # attaches to an image read from the file (rwMRC.cpp:181-184)

    @property
    def sampling(self):
        mx, my, mz = self.mx or 1, self.my or 1, self.mz or 1
        return (self.cell[0] / mx if self.cell[0] else 1.0,
                self.cell[1] / my if self.cell[1] else 1.0,
                self.cell[2] / mz if self.cell[2] else 1.0)

    @property
    def n_images(self):
        if self.nversion >= 20140 and self.nversion <= 20209 and self.mz:
            return self.nz // self.mz
        return self.nz

    @property
    def image_origin(self):
        """Image origin in pixels, as the reference derives it (rwMRC.cpp:195)."""
        s = self.sampling
        return tuple(-self.origin[i] / s[i] for i in range(3))

    def image_origin_of(self, i: int):
        """The origin of image i of the stack: the header's, for every image."""
        return self.image_origin

    @property
    def file_stats(self):
        """(average, standard deviation) read_img attaches to an image of the file."""
        return float(self.dmean), float(self.rms)


def read_header(path: str) -> MRCHeader:
    with open(path, "rb") as f:
        raw = f.read(HEADER_BYTES)
    if len(raw) < HEADER_BYTES:
        raise ValueError(f"{path}: short MRC header")
    ints = struct.unpack("<10i", raw[:40])
    nx, ny, nz, mode, _, _, _, mx, my, mz = ints
    if nx < 1 or ny < 1 or nz < 1 or mode < 0 or mode > 16:
        raise ValueError(f"{path}: not a valid little-endian MRC image "
                         f"(nx={nx} ny={ny} nz={nz} mode={mode})")
    cell = struct.unpack("<3f", raw[40:52])
    nsymbt = struct.unpack("<i", raw[92:96])[0]
    nversion = struct.unpack("<i", raw[108:112])[0]
    origin = struct.unpack("<3f", raw[196:208])
    dmean = struct.unpack("<f", raw[84:88])[0]
    rms = struct.unpack("<f", raw[216:220])[0]
    return MRCHeader(nx, ny, nz, mode, mx, my, mz, cell, origin, nsymbt, nversion, dmean, rms)


def read_stack(path: str, first: int = 0, count: int | None = None) -> tuple[np.ndarray, MRCHeader]:
    """Read float32 images [first, first+count) of a mode-2 stack -> (n, ny, nx)."""
    h = read_header(path)
    if h.mode != 2:
        raise ValueError(f"{path}: only mode 2 (float32) stacks are supported, got mode {h.mode}")
    per = h.nx * h.ny * (h.mz if h.nversion >= 20140 and h.mz else 1)
    nimg = h.n_images
    if count is None:
        count = nimg - first
    if first < 0 or first + count > nimg:
        raise IndexError(f"{path}: images [{first},{first + count}) outside stack of {nimg}")
    data = np.fromfile(path, dtype="<f4", count=count * per,
                       offset=HEADER_BYTES + h.nsymbt + first * per * 4)
    if data.size != count * per:
        raise ValueError(f"{path}: truncated data")
    return data.reshape(count, h.ny, h.nx), h


def write_stack(path: str, images: np.ndarray, pixel_size: float,
                origin_pixels=(0.0, 0.0, 0.0), volume: bool = False) -> None:
    """Write float32 images (n, ny, nx) as a stack (mz = 1), or a volume (nz, ny, nx)."""
    a = np.ascontiguousarray(images, dtype="<f4")
    if a.ndim == 2:
        a = a[None]
    nz, ny, nx = a.shape
    mz = nz if volume else 1
    hdr = bytearray(HEADER_BYTES)
    struct.pack_into("<10i", hdr, 0, nx, ny, nz, 2, 0, 0, 0, nx, ny, mz)
    struct.pack_into("<3f", hdr, 40, nx * pixel_size, ny * pixel_size, mz * pixel_size)
    struct.pack_into("<3f", hdr, 52, 90.0, 90.0, 90.0)
    struct.pack_into("<3i", hdr, 64, 1, 2, 3)
    struct.pack_into("<3f", hdr, 76, float(a.min()), float(a.max()), float(a.mean()))
    struct.pack_into("<i", hdr, 104, 0)
    struct.pack_into("<i", hdr, 108, 20140)
    struct.pack_into("<3f", hdr, 196, *[-o * pixel_size for o in origin_pixels])
    hdr[208:212] = b"MAP "
    hdr[212:216] = bytes([0x44, 0x44, 0x00, 0x00])
    struct.pack_into("<f", hdr, 216, float(a.std()))
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(hdr)
        f.write(a.tobytes())
    os.replace(tmp, path)


def read_volume(path: str) -> tuple[np.ndarray, MRCHeader]:
    h = read_header(path)
    if h.mode != 2:
        raise ValueError(f"{path}: only mode 2 (float32) maps are supported")
    data = np.fromfile(path, dtype="<f4", count=h.nx * h.ny * h.nz,
                       offset=HEADER_BYTES + h.nsymbt)
    return data.reshape(h.nz, h.ny, h.nx), h
