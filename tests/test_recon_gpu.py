"""CUDA reconstruction path against the FP64 oracle and the reference's own
breconstruct outputs (golden fixtures).  Tolerance for maps: relative L2
<= 1e-5, FSC >= 0.999."""
import os

import numpy as np
import pytest

import oracle
from bsoft_b200.plan import P_MAP, ReconOptions, load_images, plan_reconstruction
from bsoft_b200.project import read_project
from bsoft_b200.recon import Reconstructor
from bsoft_b200.synth import DatasetSpec, generate, write_dataset
from tests.helpers import CASES, GOLDEN, load_case, materialize_dataset, ref_tol, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def fsc(a, b):
    A, B = np.fft.fftn(a), np.fft.fftn(b)
    N = a.shape[0]
    f = np.fft.fftfreq(N) * N
    r = np.rint(np.sqrt(f[:, None, None] ** 2 + f[None, :, None] ** 2 + f[None, None, :] ** 2)).astype(int)
    out = []
    for s in range(1, N // 2):
        m = r == s
        out.append(np.real(np.sum(A[m] * np.conj(B[m]))) / np.sqrt(np.sum(abs(A[m]) ** 2) * np.sum(abs(B[m]) ** 2)))
    return np.array(out)


@pytest.mark.parametrize("case", CASES)
def test_gpu_matches_reference_and_oracle(case, tmp_path):
    plan, images, refs = load_case(case, str(tmp_path))
    with Reconstructor(plan) as rec:
        rec.insert(images, plan.params)
        if plan.nmaps == 2:
            for h, key in ((1, "map_01"), (2, "map_02")):
                m = rec.finish(h)
                sel = np.nonzero(plan.params[:, P_MAP] == h - 1)[0]
                orc = oracle.reconstruct(plan, images, sel)
                assert rel_l2(m, orc) < TOL, (key, rel_l2(m, orc))
                assert rel_l2(m, refs[key]) < ref_tol(case), (key, rel_l2(m, refs[key]))
        else:
            m = rec.finish(0)
            orc = oracle.reconstruct(plan, images)
            assert rel_l2(m, orc) < TOL, rel_l2(m, orc)
            assert rel_l2(m, refs["map"]) < ref_tol(case), rel_l2(m, refs["map"])
            assert fsc(m, refs["map"]).min() > 0.999


@pytest.mark.parametrize("probe", ["probe_ctf16_0", "probe_ctf16_37"])
def test_gpu_particle_spectrum_matches_reference(probe, tmp_path):
    z = np.load(os.path.join(GOLDEN, probe + ".npz"))
    star = materialize_dataset(str(z["dataset"]), str(tmp_path))
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=int(z["interp"]),
                                                                ctf_action=int(z["ctf_action"])))
    i = int(z["index"])
    img = load_images(plan, [i])
    with Reconstructor(plan) as rec:
        S = rec.spectra(img, plan.params[i:i + 1])[0]
    ref = z["ctf"][..., 0] + 1j * z["ctf"][..., 1]
    assert rel_l2(S, ref) < 2e-6
    F = oracle.particle_transform(plan, img[0], plan.params[i])
    assert rel_l2(S, F) < 2e-6


def _dataset(tmp_path, **kw):
    spec = DatasetSpec(**kw)
    ph, imgs, meta = generate(spec)
    star = write_dataset(str(tmp_path), spec, ph, imgs, meta)
    return star


@pytest.mark.parametrize("shape", [0, 2])
def test_gpu_c1_scale_against_oracle(tmp_path, shape):
    # 64^2 images -> 64^3, CTF flip, trilinear, 300 particles
    star = _dataset(tmp_path, box=64, n_particles=300, n_blobs=50, seed=21, snr=0.1)
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=2, ctf_action=1))
    images = load_images(plan)
    with Reconstructor(plan) as rec:
        rec.set_tile_shape(shape)
        rec.insert(images, plan.params)
        m = rec.finish()
    orc = oracle.reconstruct(plan, images)
    assert rel_l2(m, orc) < TOL
    assert fsc(m, orc).min() > 0.999


@pytest.mark.parametrize("shape", [0, 1, 3])
def test_gpu_bitwise_deterministic_and_batch_invariant(tmp_path, shape):
    star = _dataset(tmp_path, box=32, n_particles=120, n_blobs=12, seed=22, snr=0.3)
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=2, ctf_action=1))
    images = load_images(plan)
    outs = []
    for _ in range(2):
        with Reconstructor(plan) as rec:
            rec.set_tile_shape(shape)
            rec.insert(images, plan.params)
            outs.append(rec.accumulators(0))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    # different device batch sizes and split insert calls: same sums within rounding
    with Reconstructor(plan, batch=7) as rec:
        rec.set_tile_shape(shape)
        rec.insert(images[:50], plan.params[:50])
        rec.insert(images[50:], plan.params[50:])
        v, w = rec.accumulators(0)
    assert rel_l2(v, outs[0][0]) < 1e-6 and rel_l2(w, outs[0][1]) < 1e-6
    # and the FP64 oracle's accumulators
    ov, ow, _, _ = oracle.insert(plan, images, plan.params)
    assert rel_l2(v.reshape(-1), ov.view(np.complex128)) < 1e-6 and rel_l2(w.reshape(-1), ow) < 1e-6


@pytest.mark.parametrize("shape", range(4))
@pytest.mark.parametrize("case", ["ctf16_tri_flip", "ctf16_tri_flip_res", "plain24_tri", "ctf16_near_apply"])
def test_gpu_tile_shapes_match_reference(case, shape, tmp_path):
    """Every gridding tile shape against the compiled reference's map."""
    plan, images, refs = load_case(case, str(tmp_path))
    with Reconstructor(plan) as rec:
        rec.set_tile_shape(shape)
        rec.insert(images, plan.params)
        m = rec.finish(0)
    assert rel_l2(m, refs["map"]) < ref_tol(case), rel_l2(m, refs["map"])


def test_gpu_autotune_reports_every_shape(tmp_path):
    star = _dataset(tmp_path, box=32, n_particles=40, n_blobs=8, seed=26)
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=2, ctf_action=1))
    images = load_images(plan)
    with Reconstructor(plan) as rec:
        best, ms = rec.autotune(images, plan.params)
        assert len(ms) == 4 and np.all(ms > 0) and 0 <= best < 4
        rec.insert(images, plan.params)
        m = rec.finish()
    assert rel_l2(m, oracle.reconstruct(plan, images)) < TOL


def test_gpu_device_pointer_input(tmp_path):
    torch = pytest.importorskip("torch")
    star = _dataset(tmp_path, box=32, n_particles=40, n_blobs=8, seed=23)
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=2, ctf_action=1))
    images = load_images(plan)
    with Reconstructor(plan) as rec:
        rec.insert(images, plan.params)
        host = rec.finish()
    dev = torch.from_numpy(images).cuda()
    with Reconstructor(plan) as rec:
        rec.insert(dev, plan.params)
        rec.synchronize()
        devm = rec.finish()
    assert np.array_equal(host, devm)


def test_gpu_half_maps_fsc(tmp_path):
    star = _dataset(tmp_path, box=32, n_particles=200, n_blobs=12, seed=24, snr=1.0)
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=2, ctf_action=1, nmaps=3))
    images = load_images(plan)
    with Reconstructor(plan) as rec:
        rec.insert(images, plan.params)
        full = rec.finish(0)
        f = rec.fsc()
        halves = [rec.accumulators(h) for h in (0, 1)]
    assert rel_l2(full, oracle.reconstruct(plan, images)) < TOL
    assert f.shape == (16,) and f[0] == 1.0 and f[1] > 0.5 and np.all(f <= 1.0 + 1e-9)
    # Bimage::fsc of the two weighed half-map transforms (F / w where w > 1e-30)
    wv = [np.where(w > 1e-30, v / np.where(w > 1e-30, w, 1.0), 0.0) for v, w in halves]
    ref = oracle.fsc(wv[0], wv[1], plan.map * plan.map_sampling, plan.hi_res, 16)
    assert np.abs(f - ref).max() < 1e-6


def test_gpu_rejects_bad_sizes(tmp_path):
    from bsoft_b200._lib import BsgError
    star = _dataset(tmp_path, box=16, n_particles=4, n_blobs=2, seed=25)
    plan = plan_reconstruction(read_project(star), ReconOptions())
    plan.ft = 48
    with pytest.raises(BsgError):
        Reconstructor(plan)


FOM_CASES = [("fom_ctf16_tri_flip", ("",)), ("fom_plain24_tri", ("",)), ("fom_ctf16_near_apply", ("",)),
             ("fom_ctf16_tri_flip_half", ("_01", "_02"))]


@pytest.mark.parametrize("case,suffixes", FOM_CASES)
def test_gpu_fom_map_matches_reference(case, suffixes, tmp_path):
    """The -fom map (fspace_reconstruction_snr after fspace_reconstruction_weigh,
    Bimage_reconstruct.cpp:486-515, 610-634) against the reference's own
    (tests/golden/fom_stats.npz, make_fom_golden.py).  The GPU forms it from
    FP64 channel sums and the reference from FP32 ones (measured agreement
    3e-7 to 9e-7 relative L2); every voxel kept or zeroed alike."""
    from tests.helpers import options_from_args
    z = np.load(os.path.join(GOLDEN, "fom_stats.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    plan = plan_reconstruction(read_project(star), options_from_args(str(z[case + "__options"])))
    images = load_images(plan)
    with Reconstructor(plan, fom=True) as rec:
        rec.insert(images, plan.params)
        for i, suf in enumerate(suffixes):
            imap = i + 1 if len(suffixes) > 1 else 0
            m, f = rec.finish(imap, with_fom=True)
            ref_m, ref_f = z[case + "__map" + suf], z[case + "__fom" + suf]
            assert rel_l2(m, ref_m) < ref_tol(case)
            err = rel_l2(f, ref_f)
            kept = np.mean((f != 0) == (ref_f != 0))
            print(case, suf, "fom rel L2", err, "same nonzero voxels", kept)
            assert err < 1e-5
            assert kept == 1.0


def parse_reference_stats(text: str) -> list:
    """The reconstruction reports breconstruct -verbose 1 prints
    (img_reconstruction_sum_weigh, fspace_reconstruction_stats): one dict per
    map with the printed strings of every number."""
    import re
    out = []
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        m = re.match(r"(Full|Half) reconstruction\s*(\d*):", lines[i])
        if not m:
            i += 1
            continue
        d = {"map": 0 if m.group(1) == "Full" else int(m.group(2)), "rows": []}
        d["friedel"] = lines[i + 1].split(":")[1].strip()
        cov = lines[i + 2].split(":")[1].split()
        d["coverage"], d["coverage_pct"] = cov[0], cov[1].strip("(")
        i += 3
        while i < len(lines) and not lines[i].startswith("Radius") and not re.match(r"(Full|Half) rec", lines[i]):
            i += 1
        if i < len(lines) and lines[i].startswith("Radius"):
            i += 1
            while i < len(lines) and lines[i].strip():
                d["rows"].append(lines[i].split("\t"))
                i += 1
            while not lines[i].startswith("SNR(0.5)"):
                i += 1
            d["res_snr"] = lines[i].split(":")[1].split()[0]
            d["res_fsc"] = lines[i + 1].split(":")[1].split()[0]
        out.append(d)
    # the table is printed only for the first map of a set (imap % nmaps == 0,
    # mg_reconstruct.cpp:347); with parallel weighing it can follow another
    # map's lines, so it belongs to the lowest map index
    rows = [d for d in out if d["rows"]]
    if rows and out:
        first = min(out, key=lambda d: d["map"])
        if rows[0] is not first:
            for k in ("rows", "res_snr", "res_fsc"):
                first[k] = rows[0].pop(k)
            rows[0]["rows"] = []
    return out


def close_to_printed(value: float, printed: str, rel: float = 1e-4, units: float = 0.5) -> bool:
    """|value - printed| within `units` of the printed last decimal (half a
    unit for an unrounded value, one for a value printed the same way), plus
    a relative slack for the FP32 (reference) against FP64 (here) sums."""
    dec = len(printed.split(".")[1]) if "." in printed else 0
    ref = float(printed)
    return abs(value - ref) <= units * 10.0 ** -dec + rel * abs(ref) + 1e-12


@pytest.mark.parametrize("case,suffixes", FOM_CASES)
def test_gpu_reconstruction_statistics_match_reference(case, suffixes, tmp_path):
    """Friedel residual, coverage and the shell table against what the
    reference prints for the same reconstruction (fom_stats.npz)."""
    from tests.helpers import options_from_args
    z = np.load(os.path.join(GOLDEN, "fom_stats.npz"))
    reports = parse_reference_stats(str(z[case + "__stdout"]))
    assert len(reports) == len(suffixes)
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    plan = plan_reconstruction(read_project(star), options_from_args(str(z[case + "__options"])))
    with Reconstructor(plan, fom=True) as rec:
        rec.insert(load_images(plan), plan.params)
        for rep in reports:
            st = rec.statistics(rep["map"])
            assert st["coverage"] == int(rep["coverage"])
            assert close_to_printed(st["coverage_pct"], rep["coverage_pct"])
            assert close_to_printed(st["friedel"], rep["friedel"])
            if not rep["rows"]:
                continue
            assert len(st["table"]) == len(rep["rows"])
            for got, want in zip(st["table"], rep["rows"]):
                assert int(want[0]) == int(got[0])
                for c in range(1, 9):
                    assert close_to_printed(got[c], want[c]), (int(got[0]), c, got[c], want[c])
            assert close_to_printed(st["res_snr"], rep["res_snr"], 1e-3)
            assert close_to_printed(st["res_fsc"], rep["res_fsc"], 1e-3)


MODE1_CASES = ["plain24_tri_d2_m1", "ctf16_tri_flip_c3_m1", "plain24_near_t_m1", "plain24_tri_i_m1"]


@pytest.mark.parametrize("case", MODE1_CASES)
def test_gpu_symmetry_after_reconstruction_matches_reference(case, tmp_path):
    """breconstruct -symmetry X -mode 1 (tests/golden/mode1.npz): particles
    inserted once, the finished map symmetrized in real space
    (bsg_recon_set_symmetrize), then the sinc weight; against the reference's
    map (rel L2 <= 1e-5, FSC >= 0.999).  The symmetrization itself equals the
    FP64 oracle's restatement of Bimage::symmetrize applied to the GPU's own
    unsymmetrized map, to the last bit in all but the voxels the background
    fill reaches."""
    from oracle.symmetrize_oracle import symmetrize
    from tests.helpers import options_from_args
    z = np.load(os.path.join(GOLDEN, "mode1.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    opt = options_from_args(str(z[case + "__options"]))
    plan = plan_reconstruction(read_project(star), opt)
    assert plan.sym_mode == 1
    ref = z[case + "__map"]
    with Reconstructor(plan) as rec:
        rec.insert(load_images(plan), plan.params)
        m = rec.finish()
        assert rel_l2(m, ref) <= 1e-5
        assert fsc(m, ref).min() >= 0.999
        sym_nosinc = rec.finish(sinc=False)
        rec.set_symmetrize(None)
        plain = rec.finish(sinc=False)
    N = plain.shape[0]
    orc = symmetrize(plain, (N / 2, N / 2, N / 2), opt.symmetry)
    same = np.mean(orc == sym_nosinc)
    print(case, "bitwise equal voxels", same, "rel L2", rel_l2(sym_nosinc, orc))
    assert rel_l2(sym_nosinc, orc) < 1e-7
    assert same > 0.99


@pytest.mark.parametrize("case", ["ctf16_tri_flip_rs", "plain24_tri_d2_m1_rs"])
def test_gpu_rescale_matches_reference(case, tmp_path):
    """breconstruct -rescale avg,std (tests/golden/mode1.npz): every particle
    normalised with the statistics read_img attaches before its transform,
    and the finished real map rescaled (after any -mode 1 symmetrization,
    before the sinc weight)."""
    from tests.helpers import options_from_args
    z = np.load(os.path.join(GOLDEN, "mode1.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    plan = plan_reconstruction(read_project(star), options_from_args(str(z[case + "__options"])))
    assert plan.rescale and np.all(plan.params[:, 24] > 0)
    ref = z[case + "__map"]
    with Reconstructor(plan) as rec:
        rec.insert(load_images(plan), plan.params)
        m = rec.finish()
    assert rel_l2(m, ref) <= 1e-5
    assert fsc(m, ref).min() >= 0.999


EWALD_CASES = ["ctf16_tri_flip_ew", "ctf16_near_apply_ew", "ctf16_tri_flip_d3_ew"]


@pytest.mark.parametrize("case", EWALD_CASES)
def test_gpu_ewald_matches_reference(case, tmp_path):
    """breconstruct -ewald (tests/golden/mode1.npz): every pixel inserted on
    both Ewald-sphere surfaces s_z = +-(lambda/2) s^2; against the
    reference's map and the FP64 oracle.  The maps differ from the plane
    insertion's by ~20%, so the test tells the two apart."""
    from tests.helpers import options_from_args
    z = np.load(os.path.join(GOLDEN, "mode1.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    plan = plan_reconstruction(read_project(star), options_from_args(str(z[case + "__options"])))
    assert np.all(plan.params[:, 26] > 0.02)
    images = load_images(plan)
    ref = z[case + "__map"]
    with Reconstructor(plan) as rec:
        rec.insert(images, plan.params)
        m = rec.finish()
    assert rel_l2(m, ref) <= 1e-5
    assert fsc(m, ref).min() >= 0.999
    assert rel_l2(m, oracle.reconstruct(plan, images)) <= 1e-5


def test_gpu_ewald_full_size_against_fp64_oracle():
    """Ewald insertion at the batched-insertion size (256^2, ft 512, 256^3,
    lambda of 200 kV: up to ~1 voxel of curvature at the transform's corners)
    against the FP64 oracle's accumulators on a few particles."""
    from bsoft_b200.plan import ReconPlan
    from bsoft_b200.synth import batched_insertion_workload
    w = batched_insertion_workload(n_particles=8, box=256, pool=8, seed=5)
    P = w["params"].copy()
    P[:, 26] = 0.025079336205768955
    plan = ReconPlan(n=256, ft=512, map=256, map_sampling=w["pixel"], hi_res=w["hi_res"], interp=2,
                     ctf_action=1, wiener=0.0, params=P, nmaps=1)
    images = np.ascontiguousarray(w["pool"])
    with Reconstructor(plan) as rec:
        rec.insert(images, P)
        v, wt = rec.accumulators(0)
    ov, ow, _, _ = oracle.insert(plan, images, P)
    assert rel_l2(v.reshape(-1), ov.view(np.complex128)) < 1e-6
    assert rel_l2(wt.reshape(-1), ow) < 1e-6


MODE2_CASES = ["ctf16_tri_flip_d3_m2", "plain24_tri_i_m2", "plain24_near_t_m2_half"]


@pytest.mark.parametrize("case", MODE2_CASES)
def test_gpu_symmetry_mode2_matches_reference(case, tmp_path):
    """breconstruct -symmetry X -mode 2 (tests/golden/mode2.npz): each
    particle inserted once with a random symmetry-related view, drawn with
    the seed the reference's random() had; against the reference's maps
    (half maps too) and the FP64 oracle."""
    from tests.helpers import options_from_args
    z = np.load(os.path.join(GOLDEN, "mode2.npz"))
    star = materialize_dataset(str(z[case + "__dataset"]), str(tmp_path))
    opt = options_from_args(str(z[case + "__options"]))
    opt.seed = int(z[case + "__seed"])
    plan = plan_reconstruction(read_project(star), opt)
    assert plan.sym_mode == 2
    images = load_images(plan)
    with Reconstructor(plan) as rec:
        rec.insert(images, plan.params)
        if plan.nmaps == 2:
            for h in (1, 2):
                m = rec.finish(h)
                assert rel_l2(m, z[f"{case}__map_0{h}"]) <= 1e-5
        else:
            m = rec.finish()
            ref = z[case + "__map"]
            assert rel_l2(m, ref) <= 1e-5
            assert fsc(m, ref).min() >= 0.999
            plan.symmetry = "C1"
            assert rel_l2(m, oracle.reconstruct(plan, images)) <= 1e-5
