"""Host-side logic: STAR/MRC I/O, planning rules and orientation conventions."""
import math
import os

import numpy as np

from bsoft_b200.geometry import angle_set_negpi_to_pi, matrix_to_view, random_views, view_to_matrix
from bsoft_b200.io import mrc
from bsoft_b200.plan import check_resolution, part_ft_size
from bsoft_b200.project import read_project, write_project
from bsoft_b200.synth import DatasetSpec, generate, write_dataset


def test_part_ft_size():
    # mg_reconstruct.cpp:38-64: next power of two of pad * box
    assert part_ft_size(64, 1, 2) == 128
    assert part_ft_size(256, 1, 2) == 512
    assert part_ft_size(384, 1, 2) == 1024
    assert part_ft_size(100, 1, 0) == 100
    assert part_ft_size(100, 1, 3) == 512


def test_check_resolution():
    # default resolution = sampling -> 2u/sqrt(3) in 3-D (Bimage.cpp:633-648)
    assert abs(check_resolution(1.5, 64, 1.5) - 3.0 / math.sqrt(3)) < 1e-12
    assert check_resolution(10.0, 64, 1.5) == 10.0
    assert check_resolution(1e4, 64, 1.5) == 64 * 1.5


def test_angle_wrap_matches_reference_rule():
    for a in (-7.0, -3.5, -1.0, 0.0, 1.0, 3.5, 7.0, 10.0):
        r = angle_set_negpi_to_pi(a)
        assert -math.pi - 1e-12 <= r <= math.pi + 1e-12
        assert abs(math.sin(r) - math.sin(a)) < 1e-12 and abs(math.cos(r) - math.cos(a)) < 1e-12


def test_view_matrix_conventions():
    rng = np.random.default_rng(0)
    for v in random_views(rng, 50):
        R = view_to_matrix(v)
        assert np.allclose(R @ R.T, np.eye(3), atol=1e-12)
        assert abs(np.linalg.det(R) - 1) < 1e-12
        assert np.allclose(R[:, 2], v[:3] / np.linalg.norm(v[:3]), atol=1e-12)
        back = matrix_to_view(R)
        assert np.allclose(view_to_matrix(back), R, atol=1e-10)
    # identity view
    assert np.allclose(view_to_matrix((0, 0, 1, 0)), np.eye(3))


def test_star_mrc_roundtrip(tmp_path):
    spec = DatasetSpec(box=16, n_particles=20, n_blobs=4, seed=5, mean_per_micrograph=6, astig_range=(0, 300))
    ph, imgs, meta = generate(spec)
    star = write_dataset(str(tmp_path), spec, ph, imgs, meta)
    proj = read_project(star)
    assert proj.n_particles == 20
    got = np.concatenate([mrc.read_stack(os.path.join(str(tmp_path), m.particle_file))[0] for m in proj.micrographs])
    assert np.array_equal(got, imgs)
    views = np.concatenate([m.view for m in proj.micrographs])
    assert np.allclose(views[:, :3], meta["views"][:, :3])
    assert np.allclose(np.cos(views[:, 3]), np.cos(meta["views"][:, 3]))
    origins = np.concatenate([m.origin for m in proj.micrographs])
    assert np.allclose(origins[:, :2], meta["origins"][:, :2])
    write_project(str(tmp_path / "again.star"), proj)
    proj2 = read_project(str(tmp_path / "again.star"))
    assert np.allclose(np.concatenate([m.view for m in proj2.micrographs]), views)


def test_origin_reset_rule(tmp_path):
    # rwmg.cpp:655-659: a cubic particle.box_size makes every origin too far
    # from box/2 (z included) and resets it to the box centre
    spec = DatasetSpec(box=16, n_particles=3, n_blobs=2, seed=1)
    ph, imgs, meta = generate(spec)
    star = write_dataset(str(tmp_path), spec, ph, imgs, meta)
    lines = open(star).read().splitlines()
    lines = ["_particle.box_size 16" if l.startswith("_particle.box_size_x") else l for l in lines
             if not l.startswith(("_particle.box_size_y", "_particle.box_size_z"))]
    text = "\n".join(lines) + "\n"
    open(star, "w").write(text)
    proj = read_project(star)
    assert np.allclose(proj.micrographs[0].origin[:, :2], 8.0)


def test_mrc_header_origin(tmp_path):
    p = str(tmp_path / "x.mrcs")
    mrc.write_stack(p, np.zeros((2, 8, 8), np.float32), 1.5, origin_pixels=(4.0, 3.0, 0.0))
    h = mrc.read_header(p)
    assert h.n_images == 2 and h.sampling[0] == 1.5
    assert np.allclose(h.image_origin[:2], (4.0, 3.0))
