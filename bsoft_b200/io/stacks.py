"""Particle stack reading by file format, as the reference's read_img picks
the reader from the file extension (bsoft/src/rwimg/rwimg.cpp:79-130):
``.spi`` / ``.spider`` -> SPIDER (spider.py), otherwise MRC (mrc.py).  Both
headers answer nx, ny, sampling, n_images and image_origin_of(i)."""
from __future__ import annotations

from . import mrc, spider


def read_header(path: str):
    return spider.read_header(path) if spider.is_spider(path) else mrc.read_header(path)


def read_stack(path: str, first: int = 0, count: int | None = None):
    if spider.is_spider(path):
        return spider.read_stack(path, first, count)
    return mrc.read_stack(path, first, count)
