"""The C++ drop-in `breconstruct` (bsoft_b200/host/breconstruct.cpp) over
libbsgpu: its planning against the Python host mirror (CPU) and its maps
against the compiled reference's breconstruct output (GPU)."""
import os
import shlex
import subprocess

import numpy as np
import pytest

from bsoft_b200.plan import PARTICLE_DOUBLES
from bsoft_b200.io import mrc
from tests.helpers import CASES, GOLDEN, load_case, materialize_dataset, ref_tol, rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "bsoft_b200", "_build", "breconstruct")


@pytest.fixture(scope="module")
def exe():
    if not os.path.exists(EXE):
        from bsoft_b200 import build
        build.build()
    return EXE


def _args(case):
    return shlex.split(str(np.load(os.path.join(GOLDEN, case + ".npz"))["options"]))


@pytest.mark.parametrize("case", CASES)
def test_plan_matches_host_mirror(case, exe, tmp_path):
    plan, _, _ = load_case(case, str(tmp_path))
    star = materialize_dataset(str(np.load(os.path.join(GOLDEN, case + ".npz"))["dataset"]), str(tmp_path))
    r = subprocess.run([exe, *_args(case), "-plan", star], capture_output=True, text=True, check=True)
    lines = r.stdout.strip().splitlines()
    head = lines[0].split()
    kv = {head[i]: head[i + 1] for i in range(0, len(head), 2)}
    assert int(kv["n"]) == plan.n and int(kv["ft"]) == plan.ft and int(kv["map"]) == plan.map
    assert float(kv["map_sampling"]) == plan.map_sampling and float(kv["hi_res"]) == plan.hi_res
    assert int(kv["nmaps"]) == plan.nmaps and float(kv["wiener"]) == plan.wiener
    from bsoft_b200.symmetry import operators
    assert int(kv["nsym"]) == len(operators(plan.symmetry))
    rec = np.array([[float(t) for t in ln.split()] for ln in lines[1:]]).reshape(-1, PARTICLE_DOUBLES)
    assert rec.shape == plan.params.shape
    assert np.abs(rec - plan.params).max() <= 1e-12 * max(1.0, np.abs(plan.params).max())


def test_rejects_unknown_option(exe, tmp_path):
    r = subprocess.run([exe, "-nonsense", "x.star"], capture_output=True, text=True)
    assert r.returncode != 0 and "unknown option" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_maps_match_reference(case, exe, tmp_path):
    z = np.load(os.path.join(GOLDEN, case + ".npz"))
    star = materialize_dataset(str(z["dataset"]), str(tmp_path))
    out = os.path.join(str(tmp_path), "map.mrc")
    subprocess.run([exe, *_args(case), "-reconstruction", out, star], capture_output=True, text=True, check=True)
    keys = [k for k in z.files if k.startswith("map")]
    for k in keys:
        name = out if k == "map" else out.replace(".mrc", k[3:] + ".mrc")   # map_01 -> map_01.mrc
        h = mrc.read_header(name)
        assert (h.nx, h.ny, h.nz) == z[k].shape[::-1]
        m = np.fromfile(name, dtype="<f4", offset=1024 + h.nsymbt).reshape(z[k].shape)
        assert rel_l2(m, z[k]) < ref_tol(case), (k, rel_l2(m, z[k]))


# ---- brefine: the reference's grid refinement fixtures through the drop-in
def _write_refine_project(d, tmp_path):
    import math
    from bsoft_b200.ctf import CTFParams, electron_wavelength
    from bsoft_b200.project import Micrograph, Project, write_project
    N, n = d["N"], d["n"]
    mrc.write_stack(os.path.join(tmp_path, "ref.mrc"), d["map"], d["pixel"], origin_pixels=(N // 2,) * 3, volume=True)
    mrc.write_stack(os.path.join(tmp_path, "parts.mrcs"), d["images"], d["pixel"])
    proj = Project(base_dir=str(tmp_path))
    for i, st in enumerate(d["start"]):
        ctf = None
        if d["def_std"] > 0:
            r = d["ctf_rows"][i]
            wl = electron_wavelength(r[0])
            t1, t2 = math.pi / 2 * wl ** 3, -math.pi * wl
            ctf = CTFParams(volt=r[0], cs=r[5] / t1, amp_shift=-r[1], defocus=r[2] / t2,
                            def_dev=math.hypot(r[3], r[4]) / abs(t2), ast_angle=math.atan2(r[4] / t2, r[3] / t2) / 2)
        # one micrograph per particle: each carries its own CTF
        proj.micrographs.append(Micrograph(
            id=f"mg{i}", particle_file="parts.mrcs", box_size=n, pixel_size=d["pixel"], ctf=ctf,
            part_id=np.array([i + 1]), origin=np.array([[st[4], st[5], 0.0]]), view=st[None, :4].copy(),
            defocus=np.zeros(1), magnification=np.zeros(1), select=np.ones(1, dtype=np.int64),
            pixel=np.array([d["pixel"]])))
    star = os.path.join(tmp_path, "in.star")
    write_project(star, proj)
    return star


@pytest.mark.gpu
@pytest.mark.parametrize("fomtype", ["frc", "dpr", "mag"])
@pytest.mark.parametrize("case", ["refine64", "refine32", "refine64ctf"])
def test_brefine_matches_reference(case, fomtype, exe, tmp_path):
    """The drop-in brefine against the compiled reference brefine program on
    the same STAR project (tests/golden/refine_ccurve.npz and
    refine_mag.npz, ``<case>_brefine*``): the FRC and DPR figures of merit
    with brefine's C_curve shell weights, and -magnification (the refined
    pixel sizes x, y written with the particles).  The program writes six
    decimals."""
    import math
    from bsoft_b200.project import read_project
    from tests.refine_helpers import GOLDEN, load
    d = load(case)
    star = _write_refine_project(d, str(tmp_path))
    out = os.path.join(str(tmp_path), "out.star")
    args = [os.path.join(ROOT, "bsoft_b200", "_build", "brefine"), "-reference", os.path.join(str(tmp_path), "ref.mrc"),
            "-grid", f"{round(d['alpha'] * 180 / math.pi, 6)},{round(d['accuracy'] * 180 / math.pi, 6)}",
            "-step", f"{d['shift_step']},{d['shift_accuracy']}", "-resolution", repr(d["hi_res"]), "-output", out, star]
    if d["def_std"] > 0:
        args[1:1] = ["-defocus", repr(d["def_std"])]
    if fomtype == "dpr":
        args[1:1] = ["-fomtype", "dpr"]
    zmag = np.load(os.path.join(GOLDEN, "refine_mag.npz"))
    if fomtype == "mag":
        args[1:1] = ["-magnification", repr(float(zmag[case + "_max_mag"]))]
    subprocess.run(args, capture_output=True, text=True, check=True)
    proj = read_project(out)
    if fomtype == "mag":
        ref = zmag[case + "_brefine"]
    else:
        ref = np.load(os.path.join(GOLDEN, "refine_ccurve.npz"))[f"{case}_brefine_{fomtype}"]
    fom = _star_column(out, "particle.fom")
    for i, mg in enumerate(proj.micrographs):
        v = mg.view[0]
        assert np.abs(v - ref[i, :4]).max() < 2e-6, (i, v, ref[i, :4])
        assert np.abs(mg.origin[0, :2] - ref[i, 4:6]).max() < 2e-6
        assert abs(fom[i] - ref[i, 7]) < 2e-6
        if d["def_std"] > 0:
            assert abs(mg.defocus[0] - ref[i, 6]) < 2e-6 * ref[i, 6]
        if fomtype == "mag":
            assert abs(mg.pixel[0] - ref[i, 9]) < 2e-6 and abs(mg.pixel_y[0] - ref[i, 10]) < 2e-6


def _star_column(path, tag):
    """Values of a STAR loop column over all blocks, in order."""
    from bsoft_b200.io.star import read_star
    vals = []
    for b in read_star(path):
        for lp in b.loops:
            if lp.index(tag) >= 0:
                vals.extend(float(v) for v in lp.column(tag))
    return np.array(vals)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["fom_ctf16_tri_flip", "fom_plain24_tri", "fom_ctf16_tri_flip_half"])
def test_verbose_statistics_match_reference(case, exe, tmp_path):
    """breconstruct -verbose 1: the Friedel residual, coverage and shell
    table the drop-in prints against what the reference prints
    (tests/golden/fom_stats.npz)."""
    from tests.test_recon_gpu import close_to_printed, parse_reference_stats
    z = np.load(os.path.join(GOLDEN, "fom_stats.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    out = os.path.join(str(tmp_path), "map.mrc")
    r = subprocess.run([exe, "-verbose", "1", *shlex.split(str(z[case + "__options"])), "-reconstruction", out, star],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = {d["map"]: d for d in parse_reference_stats(r.stdout)}
    want = {d["map"]: d for d in parse_reference_stats(str(z[case + "__stdout"]))}
    assert set(got) == set(want)
    for k, w in want.items():
        g = got[k]
        assert g["coverage"] == w["coverage"]
        assert close_to_printed(float(g["friedel"]), w["friedel"], 1e-3, 1.0)
        assert close_to_printed(float(g["coverage_pct"]), w["coverage_pct"], 1e-3, 1.0)
        assert len(g["rows"]) == len(w["rows"])
        for a, b in zip(g["rows"], w["rows"]):
            for c in range(1, 9):
                assert close_to_printed(float(a[c]), b[c], 1e-3, 1.0), (k, a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["plain24_tri_d2_m1", "plain24_tri_i_m1"])
def test_symmetry_mode1_matches_reference(case, exe, tmp_path):
    """The drop-in with -symmetry X -mode 1 against the reference's map."""
    z = np.load(os.path.join(GOLDEN, "mode1.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    out = os.path.join(str(tmp_path), "map.mrc")
    r = subprocess.run([exe, *shlex.split(str(z[case + "__options"])), "-reconstruction", out, star],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    v, _ = mrc.read_volume(out)
    assert rel_l2(v, z[case + "__map"]) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ctf16_tri_flip_rs", "plain24_tri_d2_m1_rs"])
def test_rescale_matches_reference(case, exe, tmp_path):
    """The drop-in with -rescale avg,std against the reference's map."""
    z = np.load(os.path.join(GOLDEN, "mode1.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    out = os.path.join(str(tmp_path), "map.mrc")
    r = subprocess.run([exe, *shlex.split(str(z[case + "__options"])), "-reconstruction", out, star],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    v, _ = mrc.read_volume(out)
    assert rel_l2(v, z[case + "__map"]) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ctf16_tri_flip_ew", "ctf16_tri_flip_d3_ew"])
def test_ewald_matches_reference(case, exe, tmp_path):
    """The drop-in with -ewald against the reference's map."""
    z = np.load(os.path.join(GOLDEN, "mode1.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    out = os.path.join(str(tmp_path), "map.mrc")
    r = subprocess.run([exe, *shlex.split(str(z[case + "__options"])), "-reconstruction", out, star],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    v, _ = mrc.read_volume(out)
    assert rel_l2(v, z[case + "__map"]) <= 1e-5


M2_CASES = ["ctf16_tri_flip_d3_m2", "plain24_tri_i_m2", "plain24_near_t_m2_half"]


@pytest.mark.parametrize("case", M2_CASES)
def test_mode2_plan_matches_host_mirror(case, exe, tmp_path):
    """-mode 2 -seed S: the drop-in's random symmetric views (its own
    srandom/random) equal the Python planner's, record for record."""
    from bsoft_b200.plan import plan_reconstruction
    from bsoft_b200.project import read_project
    from tests.helpers import options_from_args
    z = np.load(os.path.join(GOLDEN, "mode2.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    args = shlex.split(str(z[case + "__options"])) + ["-seed", str(int(z[case + "__seed"]))]
    plan = plan_reconstruction(read_project(star), options_from_args(" ".join(args)))
    r = subprocess.run([exe, *args, "-plan", star], capture_output=True, text=True, check=True)
    rec = np.array([[float(t) for t in ln.split()] for ln in r.stdout.strip().splitlines()[1:]])
    assert rec.shape == plan.params.shape
    assert np.abs(rec - plan.params).max() <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("case", M2_CASES)
def test_symmetry_mode2_matches_reference(case, exe, tmp_path):
    """The drop-in with -symmetry X -mode 2 -seed S against the reference's
    map drawn with the same seed."""
    z = np.load(os.path.join(GOLDEN, "mode2.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    out = os.path.join(str(tmp_path), "map.mrc")
    args = shlex.split(str(z[case + "__options"])) + ["-seed", str(int(z[case + "__seed"]))]
    r = subprocess.run([exe, *args, "-reconstruction", out, star], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for k in [k for k in z.files if k.startswith(case + "__map")]:
        tag = k[len(case) + 5:]
        v, _ = mrc.read_volume(out.replace(".mrc", tag + ".mrc"))
        assert rel_l2(v, z[k]) <= 1e-5, (k, rel_l2(v, z[k]))


# ---- bbackproj: the reference's back-projection maps through the drop-in
BP_EXE = os.path.join(ROOT, "bsoft_b200", "_build", "bbackproj")
BP_CASES = ["ctf16_bp", "plain24_bp", "plain24_bp_half", "plain24_bp_full_half", "plain24_bp_d2", "ctf16_bp_rs"]


@pytest.mark.parametrize("case", BP_CASES)
def test_bbackproj_plan_matches_host_mirror(case, exe, tmp_path):
    """The drop-in's records (origins, matrices, magnification, half maps,
    pixel sizes) equal the Python planner's."""
    from bsoft_b200.backproj import plan_backprojection
    from bsoft_b200.project import read_project
    from tests.helpers import backproj_options_from_args
    z = np.load(os.path.join(GOLDEN, "bbackproj.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    args = shlex.split(str(z[case + "__options"]))
    plan = plan_backprojection(read_project(star), backproj_options_from_args(str(z[case + "__options"])))
    r = subprocess.run([BP_EXE, *args, "-plan", star], capture_output=True, text=True, check=True)
    lines = r.stdout.strip().splitlines()
    head = lines[0].split()
    kv = {head[i]: head[i + 1] for i in range(0, len(head), 2)}
    assert int(kv["n"]) == plan.n and int(kv["map"]) == plan.map and int(kv["nmaps"]) == plan.nmaps
    rec = np.array([[float(t) for t in ln.split()] for ln in lines[1:]])
    assert rec.shape == plan.records.shape
    assert np.abs(rec - plan.records).max() <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("case", BP_CASES)
def test_bbackproj_matches_reference(case, exe, tmp_path):
    """The drop-in bbackproj against the reference's maps (every map it
    writes: full, half maps)."""
    z = np.load(os.path.join(GOLDEN, "bbackproj.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    out = os.path.join(str(tmp_path), "map.mrc")
    r = subprocess.run([BP_EXE, *shlex.split(str(z[case + "__options"])), "-reconstruction", out, star],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for k in [k for k in z.files if k.startswith(case + "__map")]:
        tag = k[len(case) + 5:]
        v, _ = mrc.read_volume(out.replace(".mrc", tag + ".mrc"))
        assert rel_l2(v, z[k]) <= 1e-5, (k, rel_l2(v, z[k]))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["refine64", "refine32", "refine64ctf"])
def test_brefine_monte_matches_reference(case, exe, tmp_path):
    """The drop-in brefine -monte -seed S against the compiled brefine with
    its process id pinned to S (tests/golden/refine_monte.npz,
    ``<case>_brefine``): one random() stream over the run, the particles
    drawing one after another."""
    from bsoft_b200.project import read_project
    from tests.refine_helpers import GOLDEN, load
    d = load(case)
    z = np.load(os.path.join(GOLDEN, "refine_monte.npz"))
    it, sh, vw, ang, mag, seed = z[case + "_params"]
    ref = z[case + "_brefine"]
    star = _write_refine_project(d, str(tmp_path))
    out = os.path.join(str(tmp_path), "out.star")
    args = [os.path.join(ROOT, "bsoft_b200", "_build", "brefine"), "-reference", os.path.join(str(tmp_path), "ref.mrc"),
            "-monte", str(int(it)), "-shift", repr(float(sh)), "-view", repr(float(vw)), "-angle", repr(float(ang)),
            "-seed", str(int(seed)), "-resolution", repr(d["hi_res"]), "-output", out, star]
    if mag > 0:
        args[1:1] = ["-magnification", repr(float(mag))]
    if d["def_std"] > 0:
        args[1:1] = ["-defocus", repr(d["def_std"])]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    proj = read_project(out)
    fom = _star_column(out, "particle.fom")
    for i, mg in enumerate(proj.micrographs):
        assert np.abs(mg.view[0] - ref[i, :4]).max() < 2e-6, (i, mg.view[0], ref[i, :4])
        assert np.abs(mg.origin[0, :2] - ref[i, 4:6]).max() < 2e-6
        assert abs(fom[i] - ref[i, 7]) < 2e-6
        if d["def_std"] > 0:
            assert abs(mg.defocus[0] - ref[i, 6]) < 2e-6 * ref[i, 6]
        if mag > 0:
            assert abs(mg.pixel[0] - ref[i, 9]) < 2e-6 and abs(mg.pixel_y[0] - ref[i, 10]) < 2e-6


@pytest.mark.gpu
@pytest.mark.parametrize("case,sym", [("refine32", "D2"), ("refine64", "C3")])
def test_brefine_symmetry_matches_reference(case, sym, exe, tmp_path):
    """The drop-in brefine -symmetry X against the compiled brefine
    (tests/golden/refine_sym.npz): every particle refined from each view of
    symmetry_get_all_views, the best kept and its view number written as
    the selection."""
    import math
    from bsoft_b200.project import read_project
    from tests.refine_helpers import GOLDEN, load
    d = load(case)
    ref = np.load(os.path.join(GOLDEN, "refine_sym.npz"))[f"{case}_{sym}"]
    star = _write_refine_project(d, str(tmp_path))
    out = os.path.join(str(tmp_path), "out.star")
    args = [os.path.join(ROOT, "bsoft_b200", "_build", "brefine"), "-reference", os.path.join(str(tmp_path), "ref.mrc"),
            "-grid", f"{round(d['alpha'] * 180 / math.pi, 6)},{round(d['accuracy'] * 180 / math.pi, 6)}",
            "-step", f"{d['shift_step']},{d['shift_accuracy']}", "-resolution", repr(d["hi_res"]),
            "-symmetry", sym, "-output", out, star]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    proj = read_project(out)
    fom = _star_column(out, "particle.fom")
    sel = _star_column(out, "particle.select")
    for i, mg in enumerate(proj.micrographs):
        assert np.abs(mg.view[0] - ref[i, :4]).max() < 2e-6, (i, mg.view[0], ref[i, :4])
        assert np.abs(mg.origin[0, :2] - ref[i, 4:6]).max() < 2e-6
        assert abs(fom[i] - ref[i, 6]) < 2e-6
        assert sel[i] == ref[i, 7]

