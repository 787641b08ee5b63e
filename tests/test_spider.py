"""SPIDER particle stacks (bsoft/src/rwimg/rwSPIDER.cpp:82-243): the readers
against stacks written by the reference's own SPIDER writer, and the
reconstruction from a SPIDER project against the reference's breconstruct
on the same project (tests/golden/spider.npz, make_spider_golden.py)."""
import os
import subprocess

import numpy as np
import pytest

from bsoft_b200.io import mrc, spider, stacks
from bsoft_b200.plan import ReconOptions, load_images, plan_reconstruction
from bsoft_b200.project import read_project
from tests.helpers import GOLDEN, materialize_dataset, rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "bsoft_b200", "_build", "breconstruct")


def _spider_project(d):
    z = np.load(os.path.join(GOLDEN, "spider.npz"))
    for name in z["names"]:
        z["file_" + str(name)].tofile(os.path.join(d, str(name)))
    star = os.path.join(d, "particles.star")
    with open(star, "w") as f:
        f.write(str(z["star"]))
    return star, z


def test_reader_reads_the_reference_stacks(tmp_path):
    sd, md = tmp_path / "spi", tmp_path / "mrc"
    sd.mkdir()
    md.mkdir()
    _, z = _spider_project(str(sd))
    materialize_dataset("ctf16", str(md))
    for name in z["names"]:
        s, h = spider.read_stack(str(sd / str(name)))
        m, hm = mrc.read_stack(str(md / (str(name)[:-4] + ".mrcs")))
        assert np.array_equal(s, m)
        assert h.sampling == hm.sampling and h.n_images == hm.n_images == len(m)
        for i in range(h.n_images):
            assert h.image_origin_of(i) == hm.image_origin
        # one image at a time, as read_img(file, 1, index) reads it
        k = h.n_images - 1
        assert np.array_equal(spider.read_stack(str(sd / str(name)), k, 1)[0][0], m[k])


def test_reader_swaps_other_byte_order(tmp_path):
    """A big-endian copy (every 4-byte word of the headers and data swapped)
    reads the same, by the reference's test on nslice and iform."""
    _, z = _spider_project(str(tmp_path))
    name = str(z["names"][0])
    raw = z["file_" + name]
    be = raw.reshape(-1, 4)[:, ::-1].reshape(-1).copy()
    be.tofile(str(tmp_path / "be.spi"))
    a, h = spider.read_stack(str(tmp_path / name))
    b, hb = spider.read_stack(str(tmp_path / "be.spi"))
    assert hb.swap and not h.swap
    assert np.array_equal(a, b)


def test_plan_from_spider_equals_mrc(tmp_path):
    sd, md = tmp_path / "spi", tmp_path / "mrc"
    sd.mkdir()
    md.mkdir()
    star_s, z = _spider_project(str(sd))
    star_m = materialize_dataset("ctf16", str(md))
    opt = ReconOptions(interp=2, ctf_action=1)
    ps, pm = plan_reconstruction(read_project(star_s), opt), plan_reconstruction(read_project(star_m), opt)
    assert (ps.n, ps.ft, ps.map, ps.map_sampling, ps.hi_res) == (pm.n, pm.ft, pm.map, pm.map_sampling, pm.hi_res)
    assert np.array_equal(ps.params, pm.params)
    assert np.array_equal(load_images(ps), load_images(pm))
    assert stacks.read_header(os.path.join(str(sd), str(z["names"][0]))).n_images > 0


def test_drop_in_plan_from_spider(tmp_path):
    """The C++ drop-in's plan (-plan) from the SPIDER project equals the one
    from the MRC project."""
    if not os.path.exists(EXE):
        from bsoft_b200 import build
        build.build()
    sd, md = tmp_path / "spi", tmp_path / "mrc"
    sd.mkdir()
    md.mkdir()
    star_s, z = _spider_project(str(sd))
    star_m = materialize_dataset("ctf16", str(md))
    args = str(z["options"]).split()
    rs = subprocess.run([EXE, *args, "-plan", star_s], capture_output=True, text=True, check=True)
    rm = subprocess.run([EXE, *args, "-plan", star_m], capture_output=True, text=True, check=True)
    assert rs.stdout == rm.stdout and len(rs.stdout.splitlines()) > 60


@pytest.mark.gpu
def test_reconstruction_from_spider_matches_reference(tmp_path):
    from bsoft_b200.recon import Reconstructor
    star, z = _spider_project(str(tmp_path))
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=2, ctf_action=1))
    with Reconstructor(plan) as rec:
        rec.insert(load_images(plan), plan.params)
        m = rec.finish()
    assert rel_l2(m, z["map"]) < 1e-5
    out = os.path.join(str(tmp_path), "map.mrc")
    subprocess.run([EXE, *str(z["options"]).split(), "-reconstruction", out, star], capture_output=True, text=True,
                   check=True)
    v, _ = mrc.read_volume(out)
    assert rel_l2(v, z["map"]) < 1e-5
