"""Benchmark: batched Fourier-space insertion (particles/s).

Workload (one B200): 50,000 float32 256x256 particle images of a 256^3
blob phantom (400 blobs), micrographs of Poisson(200) particles, per-particle
defocus U[0.8, 3.5] um with astigmatism U[0, 0.1] um, SNR 0.05, inserted with
trilinear interpolation and CTF phase flipping (pad 2 -> 512^2 transforms)
into a 256^3 complex64 map with float32 weights.

A step = one batch of `--batch` particles through the whole hot path: image
upload (e2e leg only), background + padded 2-D FFT + origin shift + CTF, and
gridding into the map.  The timed region is `--steps` steps after
`--warmup` untimed ones.  Inputs are synthetic (seeded); each step's images
(524 MB for 2,000 particles) are larger than L2.

Legs reported on one JSON line:
  value       particles/s with images already resident in HBM (CUDA events
              on the library stream, barrier + synchronize around the region)
  e2e         particles/s through the C ABI with pinned HOST images: every
              step uploads its images; the finished map (weigh, 3-D inverse
              FFT, sinc) is read back at the end of the region
  roofline    the gridding kernel against measured HBM bandwidth, with the
              per-particle algorithmic bytes 22 N^2 (Hermitian-half complex64
              + float32 weight read and written over 0.75 N^2 voxels, plus the
              4 n^2 image)
  cpu_baseline  the reference's own breconstruct (compiled from its sources,
              oracle/_ref) on a bounded sample of the same workload, all host
              threads

Search leg (the "search" object of the same line): 128x128 noisy CTF images
(SNR 0.1) of a 128^3 blob phantom against 4,586 view directions (the
reference's asymmetric_unit_views, C1, 3 degrees) x 120 in-plane angles =
550,320 central sections, 5 x 5 trial origins (+-2 pixels), shells up to
0.8 Nyquist.  A step = one batch of `--search-batch` images: preparation
(FFT, CTF, shell norms), the BF16 tensor-core correlation with top-8
selection, and exact rescoring of the 8 candidates.  Its roofline is the
correlation kernel against the measured sustained BF16 rate; its CPU
baseline is the reference's own central_section + img_recip_space_fom per
hypothesis (oracle/_ref/match_probe), extrapolated to the exhaustive search.

Refinement leg (the search object's "refine"): `--refine-images` images of
the last search step refined from their best search pose by the reference's
grid refinement (img_refine_grid: 27 views, 2 -> 0.5 degrees; 3 x 3 origins,
0.4 -> 0.1 pixel; defocus search +-5 x 100 angstrom, as brefine -defocus),
scored in FP64 on the GPU; its CPU baseline is the reference's own
img_refine_grid on one of those particles at a single angular level
(oracle/_ref/refine_probe, one thread), timed per hypothesis and
extrapolated to the GPU leg's hypotheses per particle; the GPU refines the
same particle with the same steps and the two results are compared.

`--impl reference` times only the reference CPU implementation (rank 0).
Multi-GPU (`torchrun --nproc-per-node N`): replicas only.  Every rank runs
the same insertion workload on its own GPU (weak scaling, no collective
while inserting); timing is the max over ranks.  The partial-map sum that a
particle split across GPUs would need (the reference's sum of per-thread
maps, mg_reconstruct.cpp:306-324) is bsoft_b200.shard, not part of the
timed step.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_PARTICLES = 50000
BOX = 256
WORKLOAD = "batched-insertion-256"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    self.samples.append([t.strip() for t in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        sm = [float(s[0]) for s in self.samples if len(s) >= 6 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) >= 6 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples if len(s) >= 6 for i in range(4)
                          if s[2 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def make_workload(n_particles, rank=0, world=1):
    from bsoft_b200.synth import batched_insertion_workload
    w = batched_insertion_workload(n_particles=n_particles, box=BOX, pool=512)
    # every rank inserts the same synthetic particles (replicas; weak
    # scaling keeps the per-rank count fixed)
    return w


def plan_for(w):
    from bsoft_b200.plan import ReconPlan
    return ReconPlan(n=BOX, ft=2 * BOX, map=BOX, map_sampling=w["pixel"], hi_res=w["hi_res"], interp=2,
                     ctf_action=1, wiener=0.0, params=w["params"], nmaps=1)


def reference_project(w, n_sample: int) -> str:
    """The first `n_sample` particles of the workload as an MRC stack and a
    STAR project in a new temporary directory (returned); the project file
    is p.star."""
    from bsoft_b200.ctf import CTFParams
    from bsoft_b200.geometry import matrix_to_view
    from bsoft_b200.io import mrc
    from bsoft_b200.plan import P_CTF, P_MAT, P_ORIGIN
    from bsoft_b200.project import Micrograph, Project, write_project
    d = tempfile.mkdtemp(prefix="bench_ref_")
    P = w["params"][:n_sample]
    imgs = w["pool"][np.arange(n_sample) % w["pool"].shape[0]]
    mrc.write_stack(os.path.join(d, "p.mrcs"), imgs, w["pixel"])
    views = np.array([matrix_to_view(P[i, P_MAT:P_MAT + 9].reshape(3, 3)) for i in range(n_sample)])
    # defocus from the CTF coefficient (abw20 = -pi lambda def)
    from bsoft_b200.ctf import electron_wavelength
    lam = electron_wavelength(200000.0)
    defocus = P[:, P_CTF + 1] / (-math.pi * lam)
    proj = Project(base_dir=d)
    proj.micrographs.append(Micrograph(
        id="mg1", particle_file="p.mrcs", box_size=BOX, pixel_size=w["pixel"],
        ctf=CTFParams.from_amp_contrast(200000.0, 2.7e7, 0.07, float(defocus[0])),
        part_id=np.arange(1, n_sample + 1), origin=np.concatenate([P[:, P_ORIGIN:P_ORIGIN + 2],
                                                                   np.zeros((n_sample, 1))], 1),
        view=views, defocus=defocus, magnification=np.ones(n_sample), select=np.ones(n_sample, dtype=np.int64),
        pixel=np.full(n_sample, w["pixel"])))
    write_project(os.path.join(d, "p.star"), proj)
    return d


def reference_sample(w, n_sample: int, threads: int):
    """Run the reference's breconstruct on `n_sample` particles of the
    workload written as MRC + STAR (writing is not timed).  Returns
    (wall seconds, project directory holding ref.mrc, error text)."""
    import oracle
    exe = oracle.ref_binary("breconstruct")
    if not os.path.exists(exe):
        return None, None, "oracle/_ref/breconstruct not built"
    d = reference_project(w, n_sample)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    t0 = time.perf_counter()
    r = subprocess.run([exe, "-interp", "trilinear", "-CTF", "flip", "-threads", str(threads), "-recon",
                        os.path.join(d, "ref.mrc"), os.path.join(d, "p.star")], cwd=d, env=env,
                       capture_output=True, text=True)
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        return None, d, f"breconstruct failed: {r.stderr[-200:]}"
    return dt, d, None


def reference_steady(w, threads: int, per_thread=(4, 12)):
    """Steady-state rate of the reference: two runs of per_thread[0] and
    per_thread[1] particles per thread; the rate is the slope between them,
    so each thread's map set-up, the partial-map sum and the final transform
    (the intercept) are reported apart.  Returns (cpu_baseline dict, project
    directory of the larger run)."""
    n0, n1 = threads * per_thread[0], threads * per_thread[1]
    t0, d0, err = reference_sample(w, n0, threads)
    if t0 is None:
        return {"value": None, "unit": "particles/s", "cores": threads, "kind": "reference", "sample": err}, None
    shutil.rmtree(d0, ignore_errors=True)
    t1, d1, err = reference_sample(w, n1, threads)
    if t1 is None:
        return {"value": None, "unit": "particles/s", "cores": threads, "kind": "reference", "sample": err}, None
    slope = (n1 - n0) / max(t1 - t0, 1e-9)
    setup = max(0.0, t0 - n0 / slope)
    return {"value": round(slope, 2), "unit": "particles/s", "cores": threads, "kind": "reference",
            "sample": (f"steady state: slope between {n0} and {n1} particles of the workload ({BOX}^2 -> {BOX}^3, "
                       f"trilinear, CTF flip), walls {t0:.1f} s and {t1:.1f} s"),
            "setup_s": round(setup, 2), "single_run_particles_per_s": round(n1 / t1, 2)}, d1


def gpu_parity(d):
    """The GPU path on the reference run's own STAR project and stacks,
    against the reference's map: relative L2 and the smallest shell FSC."""
    from bsoft_b200.io import mrc
    from bsoft_b200.plan import ReconOptions, load_images, plan_reconstruction
    from bsoft_b200.project import read_project
    from bsoft_b200.recon import Reconstructor
    ref, _ = mrc.read_volume(os.path.join(d, "ref.mrc"))
    plan = plan_reconstruction(read_project(os.path.join(d, "p.star")), ReconOptions(interp=2, ctf_action=1))
    images = load_images(plan)
    with Reconstructor(plan) as rec:
        rec.insert(images, plan.params)
        m = rec.finish().reshape(ref.shape)
    a, b = m.astype(np.float64), ref.astype(np.float64)
    rel = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    A, Bf = np.fft.rfftn(a), np.fft.rfftn(b)
    N = a.shape[0]
    fz = np.fft.fftfreq(N) * N
    fx = np.arange(N // 2 + 1)
    r = np.rint(np.sqrt(fz[:, None, None] ** 2 + fz[None, :, None] ** 2 + fx[None, None, :] ** 2)).astype(int)
    num = np.bincount(r.ravel(), np.real(A * np.conj(Bf)).ravel(), minlength=N)
    da = np.bincount(r.ravel(), (np.abs(A) ** 2).ravel(), minlength=N)
    db = np.bincount(r.ravel(), (np.abs(Bf) ** 2).ravel(), minlength=N)
    sh = np.arange(1, N // 2)
    fsc = num[sh] / np.sqrt(da[sh] * db[sh])
    return {"against": "reference breconstruct map, same STAR project and stacks", "particles": int(plan.params.shape[0]),
            "rel_l2": float(f"{rel:.3g}"), "fsc_min": round(float(fsc.min()), 7), "fsc_shells": f"1..{N // 2 - 1}"}


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_threads_for_reference():
    # each reference thread holds a 20 B/voxel partial map (335 MB at 256^3)
    return max(1, min(cpu_threads(), 32))


def run_reference(args):
    """The reference processes its particle list in one pass, so the timed
    steps run inside one breconstruct call (one particle per thread per step,
    at least 8 per thread so the map set-up and final transform do not
    dominate); the warm-up is a separate small call."""
    threads = cpu_threads_for_reference()
    w = make_workload(threads * 12)
    if args.warmup:
        t, _, err = reference_sample(w, 2 * threads, threads)
        if t is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return
    cpu, d = reference_steady(w, threads)
    if d is not None:
        shutil.rmtree(d, ignore_errors=True)
    value, sample = cpu["value"], cpu["sample"]
    if value is None:
        print(json.dumps({"impl": "reference", "unavailable": sample}))
        return
    print(json.dumps({
        "impl": "reference", "metric": "particles/s (insertion)", "value": value, "unit": "particles/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "particles": N_PARTICLES, "box": BOX, "map": BOX, "ft": 2 * BOX,
                   "interp": "trilinear", "ctf": "flip"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "vs_baseline": None}))


SEARCH_BOX = 128
SEARCH_PIXEL = 1.5
SEARCH_RES = 3.75            # 0.8 Nyquist at 1.5 angstrom/pixel
SEARCH_PSI = 120             # in-plane angles (3 degrees)
SEARCH_ORIGINS = [(SEARCH_BOX // 2 + dx, SEARCH_BOX // 2 + dy) for dy in range(-2, 3) for dx in range(-2, 3)]


def search_workload(n_images, seed=21):
    from bsoft_b200.synth import DatasetSpec, generate, phantom_volume
    spec = DatasetSpec(box=SEARCH_BOX, n_particles=n_images, n_blobs=100, pixel=SEARCH_PIXEL, snr=0.1, seed=seed,
                       defocus_range=(1.0e4, 3.0e4), shift_range=2.0)
    ph, imgs, meta = generate(spec)
    return dict(spec=spec, volume=phantom_volume(ph).astype(np.float32), images=imgs, meta=meta)


def search_views_mats(npsi: int = SEARCH_PSI):
    from bsoft_b200.geometry import asymmetric_unit_views_c, search_views, views_to_matrices
    dirs = asymmetric_unit_views_c(1, math.radians(3.0), math.radians(3.0))
    views = search_views(dirs, npsi)
    return len(dirs), views_to_matrices(views), views


# grid refinement (brefine without -monte): 2 -> 0.5 degrees, 0.4 -> 0.1 pixel
# of the cut transform, defocus search of +-5 x 100 angstrom (brefine -defocus)
REFINE_ALPHA, REFINE_ACC, REFINE_STEP, REFINE_SACC, REFINE_DEF = 2.0, 0.5, 0.4, 0.1, 100.0


def refine_reference_sample(sw, start_row, ctf_row, alpha=REFINE_ALPHA, accuracy=REFINE_ACC):
    """The reference's img_refine_grid (refine_probe, one thread) on one
    particle of the search workload with the bench's shift and defocus
    steps, the given angular steps (degrees) and brefine's C_curve shell
    weights."""
    import oracle
    from bsoft_b200.io import mrc
    exe = oracle.ref_binary("refine_probe")
    if not os.path.exists(exe):
        return None, None, "oracle/_ref/refine_probe not built"
    d = tempfile.mkdtemp(prefix="bench_refine_")
    N = SEARCH_BOX
    mrc.write_stack(os.path.join(d, "ref.mrc"), sw["volume"], SEARCH_PIXEL, origin_pixels=(N // 2,) * 3, volume=True)
    mrc.write_stack(os.path.join(d, "p.mrcs"), sw["images"][int(start_row[0]):int(start_row[0]) + 1], SEARCH_PIXEL)
    np.savetxt(os.path.join(d, "start.txt"), np.asarray(start_row[1:7])[None], fmt="%.17g")
    np.savetxt(os.path.join(d, "ctf.txt"), np.asarray(ctf_row)[None], fmt="%.17g")
    t0 = time.perf_counter()
    r = subprocess.run([exe, os.path.join(d, "ref.mrc"), os.path.join(d, "p.mrcs"), repr(SEARCH_PIXEL),
                        repr(SEARCH_RES), os.path.join(d, "start.txt"), os.path.join(d, "ctf.txt"),
                        repr(alpha), repr(accuracy), repr(REFINE_STEP), repr(REFINE_SACC), "0",
                        repr(REFINE_DEF), "0", "0", "1"], capture_output=True, text=True)
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        return None, None, f"refine_probe failed: {r.stderr[-200:]}"
    out = np.array([float(t) for t in r.stdout.split()])
    return dt, out, (f"1 particle, img_refine_grid with the defocus search at one angular level "
                     f"({alpha} degrees), one thread, wall {dt:.1f} s including map preparation")


def search_reference_sample(sw, n_views: int = 160):
    """Per-hypothesis time of the reference's own scoring (match_probe:
    central_section once per view, then phase shift + img_recip_space_fom per
    trial origin), one thread, on the search workload's map and images."""
    import oracle
    from bsoft_b200.io import mrc
    exe = oracle.ref_binary("match_probe")
    if not os.path.exists(exe):
        return None, "oracle/_ref/match_probe not built"
    d = tempfile.mkdtemp(prefix="bench_match_")
    N = SEARCH_BOX
    mrc.write_stack(os.path.join(d, "ref.mrc"), sw["volume"], SEARCH_PIXEL, origin_pixels=(N // 2,) * 3, volume=True)
    nimg = 4
    mrc.write_stack(os.path.join(d, "p.mrcs"), sw["images"][:nimg], SEARCH_PIXEL)
    views = sw["meta"]["views"][np.arange(n_views) % len(sw["meta"]["views"])]
    np.savetxt(os.path.join(d, "views.txt"), views, fmt="%.17g")
    coefs = sw["meta"]["coefs"]
    np.savetxt(os.path.join(d, "ctf.txt"), np.array([[200000.0, *coefs[i][:5], 1] for i in range(nimg)]), fmt="%.17g")
    hyps = [[v % nimg, v, ox, oy] for v in range(n_views) for ox, oy in SEARCH_ORIGINS]
    np.savetxt(os.path.join(d, "hyps.txt"), np.array(hyps, float), fmt="%.17g")
    t0 = time.perf_counter()
    r = subprocess.run([exe, os.path.join(d, "ref.mrc"), os.path.join(d, "p.mrcs"), repr(SEARCH_PIXEL),
                        repr(SEARCH_RES), os.path.join(d, "views.txt"), os.path.join(d, "ctf.txt"),
                        os.path.join(d, "hyps.txt"), os.path.join(d, "out")], capture_output=True, text=True)
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        return None, f"match_probe failed: {r.stderr[-200:]}"
    return dt / len(hyps), (f"{len(hyps)} hypotheses ({n_views} central sections x {len(SEARCH_ORIGINS)} origins, "
                            f"img_recip_space_fom each), one thread, wall {dt:.1f} s including map preparation")


def train_proposer(sw, local, torch, n_train: int, epochs: float):
    """The learned proposer for the search map: n_train projections through
    the library's own projector (random views, shifts U[-2, 2] pixels, CTF
    with defocus U[1, 3] um, noise at SNR 0.1), then Adam on the GPU."""
    from bsoft_b200.cnn import Proposer, pose_targets, add_noise
    from bsoft_b200.ctf import CTFParams
    from bsoft_b200.geometry import random_views, views_to_matrices
    from bsoft_b200.match import Matcher, ctf_record
    rng = np.random.default_rng(11)
    mats = views_to_matrices(random_views(rng, n_train))
    shifts = rng.uniform(-2, 2, size=(n_train, 2))
    defocus = rng.uniform(1e4, 3e4, size=n_train)
    ctf = np.stack([ctf_record(200000.0, CTFParams.from_amp_contrast(200000.0, 2.7e7, 0.07, d).coefficients())
                    for d in defocus])
    t0 = time.perf_counter()
    proj = Matcher(n=SEARCH_BOX, map=SEARCH_BOX, map_sampling=SEARCH_PIXEL, pixel=SEARCH_PIXEL,
                   hi_res=2 * SEARCH_PIXEL, device=local)
    proj.set_reference(sw["volume"], (SEARCH_BOX // 2,) * 3)
    imgs = torch.empty((n_train, SEARCH_BOX, SEARCH_BOX), dtype=torch.float32, device="cuda")
    proj.project(mats, origins=SEARCH_BOX // 2 + shifts, ctf=ctf, out=imgs)
    add_noise(imgs, 0.1, seed=5)
    proj.close()
    torch.cuda.synchronize()
    data_s = time.perf_counter() - t0
    tg = torch.from_numpy(pose_targets(mats, shifts)).cuda()
    steps = int(epochs * n_train / 256)
    # two restarts (seeds 1, 2); the one with the lower training loss over its
    # last 100 steps is kept (the training data only; some seeds settle in a
    # worse minimum)
    runs = []
    for seed in (1, 2):
        net = Proposer(box=SEARCH_BOX, batch=256, seed=seed, device=local)
        t0 = time.perf_counter()
        losses = net.train(imgs, tg, steps=steps, lr=1e-3)
        torch.cuda.synchronize()
        runs.append((float(losses[-100:].mean()), seed, net, time.perf_counter() - t0, losses))
    runs.sort(key=lambda r: r[0])
    for r in runs[1:]:
        r[2].close()
    loss_last, seed, net, train_s, losses = runs[0]
    del imgs, tg
    torch.cuda.empty_cache()
    return net, {"train_images": n_train, "epochs": epochs, "steps": steps, "params": net.nparams,
                 "data_s": round(data_s, 2), "train_s": round(train_s, 2), "restarts": len(runs), "seed": seed,
                 "loss_last_per_seed": {str(r[1]): round(r[0], 4) for r in runs},
                 "loss_first": round(float(losses[:100].mean()), 4), "loss_last": round(loss_last, 4)}


def learned_controls(m, net, mats, pviews, origins, radius, torch, n=256):
    """The learned pipeline on the same particles at SNR 0.1, SNR 1 and
    without noise: the proposal, the local search and grid refinement
    (brefine -defocus) from the local search's best pose.  Every set is
    generated from the search map's phantom with the same views, shifts and
    CTFs (the noise is drawn last), so the rows differ only by the noise;
    the medians show what the noise, not the pipeline, limits."""
    from bsoft_b200.synth import DatasetSpec, generate
    from bsoft_b200.match import ctf_record
    from bsoft_b200.geometry import angular_distance_deg, views_to_matrices
    out = {}
    for label, snr in (("snr_0.1", 0.1), ("snr_1", 1.0), ("noise_free", None)):
        spec = DatasetSpec(box=SEARCH_BOX, n_particles=n, n_blobs=100, pixel=SEARCH_PIXEL, snr=snr, seed=21,
                           defocus_range=(1.0e4, 3.0e4), shift_range=2.0)
        _, imgs, meta = generate(spec)
        ctf = np.stack([ctf_record(spec.volt, c) for c in meta["coefs"]])
        dev = torch.from_numpy(np.ascontiguousarray(imgs)).cuda()
        pred = torch.empty((n, 11), dtype=torch.float32, device="cuda")
        net.predict(dev, out=pred)
        m.set_images(dev, ctf)
        res = m.search_local(pred, origins, radius, 1.5, 8)
        best = res[:, 0, 0].astype(int)
        start = np.column_stack([np.arange(n), pviews[best], origins[res[:, 0, 1].astype(int)]])
        m.set_c_curve_weights()             # brefine's shell weights for the refinement
        rout = m.refine(start, REFINE_ALPHA * math.pi / 180.0, REFINE_ACC * math.pi / 180.0, REFINE_STEP,
                        REFINE_SACC, REFINE_DEF)
        m.set_shell_weights(None)
        pr = pred.cpu().numpy()[:, :9].reshape(-1, 3, 3).astype(np.float64)
        e_p = angular_distance_deg(pr, meta["mats"])
        e_l = angular_distance_deg(mats[best], meta["mats"])
        e_r = angular_distance_deg(views_to_matrices(rout[:, :4]), meta["mats"])
        out[label] = {"proposal": round(float(np.median(e_p)), 3), "local_search": round(float(np.median(e_l)), 3),
                      "refined": round(float(np.median(e_r)), 3),
                      "refined_frac_within_1_deg": round(float(np.mean(e_r <= 1.0)), 4)}
    out["particles"] = n
    out["what"] = ("median angular error (degrees) against the true poses: the proposal, the local search from it "
                   "(3-degree panel), and grid refinement from the local search (2 -> 0.5 degrees, defocus search)")
    return out


def fsc_of_poses(sw, sel, mats_by_method, origins_by_method, local):
    """Reconstructions (trilinear, CTF flip, pad 2) of the images `sel` with
    each method's poses, and their Fourier shell correlation with the map
    reconstructed from the true poses: mean over shells up to 0.8 Nyquist and
    the first shell below 0.5."""
    from bsoft_b200.plan import (P_CTF, P_MAP, P_MAT, P_ORIGIN, P_PIXEL, P_SCALE, P_WEIGHT, PARTICLE_DOUBLES,
                                 ReconPlan, check_resolution)
    from bsoft_b200.recon import Reconstructor
    n = len(sel)
    imgs = np.ascontiguousarray(sw["images"][sel])
    meta = sw["meta"]

    def recon(mats, origins):
        P = np.zeros((n, PARTICLE_DOUBLES))
        P[:, P_ORIGIN:P_ORIGIN + 2] = origins
        P[:, P_MAT:P_MAT + 9] = mats.reshape(n, 9)
        P[:, P_PIXEL] = SEARCH_PIXEL
        P[:, P_SCALE] = 1.0
        P[:, P_WEIGHT] = 1.0
        P[:, P_CTF:P_CTF + 7] = meta["coefs"][sel][:, :7]
        P[:, P_MAP] = np.arange(n) % 2
        plan = ReconPlan(n=SEARCH_BOX, ft=2 * SEARCH_BOX, map=SEARCH_BOX, map_sampling=SEARCH_PIXEL,
                         hi_res=check_resolution(SEARCH_PIXEL, SEARCH_BOX, SEARCH_PIXEL), interp=2, ctf_action=1,
                         wiener=0.0, params=P, nmaps=1)
        with Reconstructor(plan, device=local) as rec:
            rec.insert(imgs, P)
            return rec.finish()

    ref = np.fft.fftn(recon(meta["mats"][sel], meta["origins"][sel][:, :2]))
    N = SEARCH_BOX
    f = np.fft.fftfreq(N) * N
    r = np.sqrt(f[:, None, None] ** 2 + f[None, :, None] ** 2 + f[None, None, :] ** 2).astype(int)
    nsh = int(0.8 * N / 2)
    out = {}
    for name in mats_by_method:
        F = np.fft.fftn(recon(mats_by_method[name], origins_by_method[name]))
        num = np.bincount(r.ravel(), (F * np.conj(ref)).real.ravel(), minlength=N)[:nsh]
        d1 = np.bincount(r.ravel(), (np.abs(F) ** 2).ravel(), minlength=N)[:nsh]
        d2 = np.bincount(r.ravel(), (np.abs(ref) ** 2).ravel(), minlength=N)[:nsh]
        fsc = num / np.sqrt(np.maximum(d1 * d2, 1e-300))
        below = np.nonzero(fsc[1:] < 0.5)[0]
        out[name] = {"fsc_mean_to_0.8_nyquist": round(float(fsc[1:].mean()), 4),
                     "first_shell_below_0.5": int(below[0] + 1) if len(below) else None}
    return out


def search_leg(args, local, dist, world, rank, torch):
    """Exhaustive orientation search; returns the "search" object (rank 0)."""
    from bsoft_b200.match import Matcher, ctf_record
    from bsoft_b200.geometry import angular_distance_deg
    B = args.search_batch
    nsteps, nwarm = args.search_steps, args.search_warmup
    pool = 2 * B
    sw = search_workload(pool, seed=21 + rank)
    imgs = sw["images"]
    meta = sw["meta"]
    ctf = np.stack([ctf_record(sw["spec"].volt, c) for c in meta["coefs"]])
    ndir, mats, pviews = search_views_mats(args.search_psi)
    origins = np.array(SEARCH_ORIGINS, float)
    m = Matcher(n=SEARCH_BOX, map=SEARCH_BOX, map_sampling=SEARCH_PIXEL, pixel=SEARCH_PIXEL, hi_res=SEARCH_RES,
                device=local)
    m.set_reference(sw["volume"], (SEARCH_BOX // 2,) * 3)
    m.set_panel(mats)
    pst = m.stats()
    panel_ms = pst["panel_ms"]
    panel_exact = {"ms": round(pst["panel_exact_ms"], 1), "gb": round(pst["panel_exact_bytes"] / 1e9, 2)}
    host = [torch.from_numpy(np.ascontiguousarray(imgs[i * B:(i + 1) * B])).pin_memory() for i in range(2)]
    dev = [h.cuda() for h in host]
    s = torch.cuda.ExternalStream(m.stream)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    results = []
    for i in range(nwarm):
        m.set_images(dev[i % 2], ctf[(i % 2) * B:(i % 2 + 1) * B])
        m.search(origins, topk=8)
    m.reset_stats()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clk:
        ev0.record(s)
        for i in range(nsteps):
            j = (nwarm + i) % 2
            m.set_images(dev[j], ctf[j * B:(j + 1) * B])
            results.append((j, m.search(origins, topk=8)))
        ev1.record(s)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    st = m.stats()
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    images = B * nsteps * world
    value = images / (ms / 1e3)
    # e2e: pinned host images through the C ABI, results back on the host
    barrier()
    t0 = time.perf_counter()
    for i in range(nsteps):
        j = (nwarm + i) % 2
        m.set_images(host[j].numpy(), ctf[j * B:(j + 1) * B])
        m.search(origins, topk=8)
    barrier()
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

    # ---- learned proposal + local search on the same images
    learned = None
    if "learned" in args.legs:
        net, train_info = train_proposer(sw, local, torch, args.train_images, args.train_epochs)
        pred = torch.empty((B, 11), dtype=torch.float32, device="cuda")
        # the network's inference alone, one batch, after two warm-up passes
        # (bsg_cnn_predict returns when its stream is done: wall time)
        for _ in range(2):
            net.predict(dev[0], out=pred)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        net.predict(dev[0], out=pred)
        train_info["predict_ms_per_batch"] = round((time.perf_counter() - t0) * 1e3, 3)
        train_info["predict_batch"] = B
        for i in range(nwarm):
            j = i % 2
            net.predict(dev[j], out=pred)
            m.set_images(dev[j], ctf[j * B:(j + 1) * B])
            m.search_local(pred, origins, args.local_radius, 1.5, 8)
        m.reset_stats()
        lres = []
        barrier()
        ev0.record(s)
        for i in range(nsteps):
            j = (nwarm + i) % 2
            net.predict(dev[j], out=pred)
            m.set_images(dev[j], ctf[j * B:(j + 1) * B])
            lres.append((j, m.search_local(pred, origins, args.local_radius, 1.5, 8), pred.cpu().numpy()))
        ev1.record(s)
        torch.cuda.synchronize()
        barrier()
        lms = ev0.elapsed_time(ev1)
        lst = m.stats()
        if dist is not None:
            t = torch.tensor([lms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            lms = float(t.item())
        learned = {"ms": lms, "stats": lst, "results": lres, "train": train_info}
        if rank == 0 and "refine" in args.legs:
            learned["controls"] = learned_controls(m, net, mats, pviews, origins, args.local_radius, torch)
        net.close()
    # ---- grid refinement of the last step's best poses (brefine -defocus)
    refine = None
    if "refine" in args.legs:
        j, res = results[-1]
        R = min(args.refine_images, B)
        best = res[:R, 0, 0].astype(int)
        start = np.column_stack([np.arange(R), pviews[best], origins[res[:R, 0, 1].astype(int)]])
        m.set_images(dev[j], ctf[j * B:(j + 1) * B])
        m.set_c_curve_weights()             # brefine's shell weights
        # radians as the reference's CLI converts degrees (atof(x) * M_PI / 180.0)
        rargs = (REFINE_ALPHA * math.pi / 180.0, REFINE_ACC * math.pi / 180.0, REFINE_STEP, REFINE_SACC, REFINE_DEF)
        m.refine(start[:16], *rargs)                                # warm-up
        m.reset_stats()
        barrier()
        ev0.record(s)
        rout = m.refine(start, *rargs)
        ev1.record(s)
        torch.cuda.synchronize()
        barrier()
        rms = ev0.elapsed_time(ev1)
        refine = {"ms": rms, "out": rout, "start": start, "j": j, "stats": m.stats(), "R": R}

    m.close()
    if rank != 0:
        return None
    errs = []
    for j, res in results:
        best = res[:, 0, 0].astype(int)
        errs.append(angular_distance_deg(mats[best], meta["mats"][j * B:(j + 1) * B]))
    errs = np.concatenate(errs)
    with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
        pk = json.load(f)
    tpeak = float(pk.get("bf16_tflops_sustained", 1411.5))
    achieved = st["gemm_flops"] / (st["gemm_ms"] / 1e3) / 1e12
    hyp_per_image = len(mats) * len(origins)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        us, sample = search_reference_sample(sw)
        if us is not None:
            cpu = {"value": 1.0 / (us * hyp_per_image), "unit": "particles/s", "cores": 1, "kind": "reference",
                   "sample": sample, "seconds_per_hypothesis": us,
                   "extrapolation": f"{hyp_per_image} hypotheses per particle x measured seconds per hypothesis"}
        else:
            cpu = {"value": None, "unit": "particles/s", "cores": 1, "kind": "reference", "sample": sample}
    refine_obj = None
    if refine is not None:
        from bsoft_b200.geometry import views_to_matrices
        from bsoft_b200.ctf import electron_wavelength
        R, j, rout, start = refine["R"], refine["j"], refine["out"], refine["start"]
        truth = meta["mats"][j * B:j * B + R]
        e0 = angular_distance_deg(views_to_matrices(start[:, 1:5]), truth)
        e1 = angular_distance_deg(views_to_matrices(rout[:, :4]), truth)
        t2 = -math.pi * electron_wavelength(sw["spec"].volt)
        true_def = meta["coefs"][j * B:j * B + R, 1] / t2
        rst = refine["stats"]
        rvalue = R / (refine["ms"] / 1e3)
        rcpu = None
        if world == 1 and not args.no_cpu_baseline:
            # a bounded sample: one particle at a single angular level (alpha =
            # accuracy), timed per hypothesis and extrapolated to the GPU leg's
            # hypotheses per particle; the GPU refines the same particle with the
            # same steps for a bitwise comparison
            ctf_row = [sw["spec"].volt, *meta["coefs"][j * B][:5], 1]
            row = start[0].copy()
            row[0] = j * B                         # the image's index in the workload's stack
            dt, rref, sample = refine_reference_sample(sw, row, ctf_row, REFINE_ALPHA, REFINE_ALPHA)
            if dt is not None:
                m2 = Matcher(n=SEARCH_BOX, map=SEARCH_BOX, map_sampling=SEARCH_PIXEL, pixel=SEARCH_PIXEL,
                             hi_res=SEARCH_RES, device=local)
                m2.set_reference(sw["volume"], (SEARCH_BOX // 2,) * 3)
                m2.set_images(sw["images"][j * B:j * B + 1], ctf[j * B:j * B + 1])
                m2.set_c_curve_weights()
                a1 = REFINE_ALPHA * math.pi / 180.0
                g1 = m2.refine(start[:1], a1, a1, REFINE_STEP, REFINE_SACC, REFINE_DEF)[0]
                m2.close()
                per_hyp = dt / max(1.0, rref[8])
                rcpu = {"value": round(1.0 / (per_hyp * float(rout[:, 8].mean())), 5), "unit": "particles/s",
                        "cores": 1, "kind": "reference", "sample": sample,
                        "seconds_per_hypothesis": per_hyp,
                        "extrapolation": "mean hypotheses per particle of the GPU leg x measured seconds per hypothesis",
                        "same_result_as_gpu": bool(np.abs(rref[:6] - g1[:6]).max() < 1e-9 and rref[8] == g1[8]),
                        "reference_hypotheses": int(rref[8])}
            else:
                rcpu = {"value": None, "unit": "particles/s", "cores": 1, "kind": "reference", "sample": sample}
        refine_obj = {
            "metric": "particles/s (grid refinement, img_refine_grid with defocus search)",
            "value": round(rvalue, 1), "unit": "particles/s", "particles": R,
            "config": {"start": "best pose of the exhaustive search", "shell_weights": "C_curve (brefine)",
                       "alpha_deg": REFINE_ALPHA,
                       "accuracy_deg": REFINE_ACC, "shift_step_px": REFINE_STEP, "shift_accuracy_px": REFINE_SACC,
                       "defocus_step_A": REFINE_DEF, "scoring": "FP64 figure of merit"},
            "hypotheses_per_particle": round(float(rout[:, 8].mean()), 1),
            "fom_ms": round(rst["refine_ms"], 2), "gpu_launches": int(rst["refine_launches"]),
            "accuracy": {"median_angular_error_deg_search": round(float(np.median(e0)), 3),
                         "median_angular_error_deg_refined": round(float(np.median(e1)), 3),
                         "median_defocus_error_A_refined": round(float(np.median(np.abs(rout[:, 9] - true_def))), 1)},
            "cpu_baseline": rcpu,
        }
    learned_obj = None
    if learned is not None:
        lvalue = images / (learned["ms"] / 1e3)
        lerr, perr = [], []
        for j, res, pr in learned["results"]:
            lerr.append(angular_distance_deg(mats[res[:, 0, 0].astype(int)], meta["mats"][j * B:(j + 1) * B]))
            perr.append(angular_distance_deg(pr[:, :9].reshape(-1, 3, 3).astype(np.float64),
                                             meta["mats"][j * B:(j + 1) * B]))
        lerr = np.concatenate(lerr)
        perr = np.concatenate(perr)
        # reconstructions from each method's poses on the last step's images
        j, res_l, _ = learned["results"][-1]
        _, res_e = results[-1]
        sel = np.arange(j * B, (j + 1) * B)
        fsc = fsc_of_poses(sw, sel, {"exhaustive": mats[res_e[:, 0, 0].astype(int)],
                                     "learned": mats[res_l[:, 0, 0].astype(int)]},
                           {"exhaustive": origins[res_e[:, 0, 1].astype(int)],
                            "learned": origins[res_l[:, 0, 1].astype(int)]}, local)
        lst = learned["stats"]
        learned_obj = {
            "metric": "particles/s (learned proposal + local search)", "value": round(lvalue, 1),
            "unit": "particles/s", "speedup_vs_exhaustive": round(lvalue / value, 2),
            "ms_per_step": round(learned["ms"] / nsteps, 2),
            "config": {"radius_deg": args.local_radius, "origin_radius_px": 1.5, "topk_rescored": 8,
                       "network": "6 conv 3x3 stride 2 (32-64-64-128-128-128), fc 1024, 6-D rotation + shift"},
            "hypotheses_per_image": round(lst["hypotheses"] / max(1, lst["images"]), 1),
            "stages_ms": {k: round(lst[k], 2) for k in ("local_ms", "rescore_ms")},
            "accuracy": {"median_angular_error_deg": round(float(np.median(lerr)), 3),
                         "frac_within_5_deg": round(float(np.mean(lerr < 5)), 4),
                         "proposal_median_error_deg": round(float(np.median(perr)), 3),
                         "proposal_frac_within_radius": round(float(np.mean(perr < args.local_radius)), 4)},
            "fsc_vs_true_pose_map": fsc, "training": learned["train"],
            "gpu_launches": int(lst["launches"]),
            "controls": learned.get("controls"),
        }
    return {
        "metric": "particles/s (exhaustive orientation search)", "value": round(value, 1), "unit": "particles/s",
        "steps": nsteps, "warmup": nwarm, "ms_per_step": round(ms / nsteps, 2), "dtype": "bf16 (correlation), f32",
        "config": {"workload": "projection-matching-128", "images_per_step": B, "box": SEARCH_BOX,
                   "map": SEARCH_BOX, "pixel": SEARCH_PIXEL, "hi_res": SEARCH_RES, "directions": ndir,
                   "in_plane": args.search_psi, "sections": len(mats), "origins": len(origins),
                   "hypotheses_per_image": hyp_per_image, "topk_rescored": 8, "snr": 0.1,
                   "l2": "inputs larger than L2 (the 9.4 GB panel is streamed every step)"},
        "e2e": {"value": round(images / e2e_s, 1), "unit": "particles/s", "h2d_bytes_per_step": B * SEARCH_BOX ** 2 * 4,
                "d2h_bytes_per_step": B * 8 * 5 * 8},
        "roofline": {"kernel": "search_gemm_kernel", "bound": "tensor", "achieved": round(achieved, 1),
                     "peak": tpeak, "unit": "TFLOP/s", "frac": round(achieved / tpeak, 4), "traffic": None,
                     "peak_source": "measured (bf16_tflops_sustained)",
                     "flops_per_hypothesis": 2 * st["coarse_k"], "gemm_ms": round(st["gemm_ms"], 2)},
        "stages_ms": {k: round(st[k], 2) for k in ("agen_ms", "gemm_ms", "merge_ms", "rescore_ms")},
        "panel_ms": round(panel_ms, 1),
        "panel_exact_sections": {**panel_exact, "what": "the panel's FP32 sections at the figure-of-merit pixels, "
                                 "built once with the panel; the exact rescoring reads them"},
        "accuracy": {"median_angular_error_deg": round(float(np.median(errs)), 3),
                     "frac_within_5_deg": round(float(np.mean(errs < 5)), 4)},
        "cpu_baseline": cpu, "gpu_launches": int(st["launches"]), "clocks": clk.summary(),
        "learned": learned_obj, "refine": refine_obj,
    }


def iteration384_leg(args, local, torch):
    """The reconstruction half of configs[4]: 384^2 particles (SNR 0.05,
    defocus U[0.5, 4] um) inserted into two 384^3 half maps (ft 1024,
    trilinear, CTF flip), then both halves weighed, inverse-transformed with
    the sinc weight and their FSC computed.  Insertion is timed like the
    main leg (device-resident images, CUDA events); the finishing (weigh,
    3-D inverse FFT of both halves, FSC) separately.  The learned proposal
    and local search of configs[4] are the search leg's, at 128^2."""
    from bsoft_b200.plan import ReconPlan
    from bsoft_b200.recon import Reconstructor
    from bsoft_b200.synth import batched_insertion_workload
    box, B, warm, steps = 384, args.iter_batch, 2, args.iter_steps
    w = batched_insertion_workload(n_particles=B * (warm + steps), box=box, pool=256, snr=0.05,
                                   defocus_range=(5000.0, 40000.0), seed=4)
    plan = ReconPlan(n=box, ft=2 * 512, map=box, map_sampling=w["pixel"], hi_res=w["hi_res"], interp=2,
                     ctf_action=1, wiener=0.0, params=w["params"], nmaps=3)
    P = w["params"]
    pool = w["pool"]
    dev = [torch.from_numpy(np.ascontiguousarray(pool[(np.arange(B) + i * B) % pool.shape[0]])).cuda()
           for i in range(2)]
    rec = Reconstructor(plan, batch=B, device=local)
    shape, shape_ms = rec.autotune(dev[0][: min(B, 256)], P[: min(B, 256)])
    rec.set_tile_shape(shape)
    s = torch.cuda.ExternalStream(rec.stream)
    for i in range(warm):
        rec.insert(dev[i % 2], P[i * B:(i + 1) * B])
    rec.synchronize()
    rec.reset()
    rec.set_timing(True)
    st0 = rec.stats()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(s)
        for i in range(steps):
            j = warm + i
            rec.insert(dev[j % 2], P[j * B:(j + 1) * B])
        ev1.record(s)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    st1 = rec.stats()
    out = torch.empty((box, box, box), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for h in (1, 2):
        rec.finish(h, out=out)
    fsc = rec.fsc()
    torch.cuda.synchronize()
    finish_ms = (time.perf_counter() - t0) * 1e3
    # the same again: the first call also allocates the finishing buffers
    t0 = time.perf_counter()
    for h in (1, 2):
        rec.finish(h, out=out)
    rec.fsc()
    torch.cuda.synchronize()
    finish_again_ms = (time.perf_counter() - t0) * 1e3
    ins_launch = st1["insert_launches"] - st0["insert_launches"]
    ins_ms = st1["insert_ms"] - st0["insert_ms"]
    rec.close()
    peak, peak_kind = peaks()
    per_particle = 22.0 * box * box
    avg = ins_ms / max(1, ins_launch)
    achieved = per_particle * B / (avg / 1e3) / 1e9
    below = np.nonzero(fsc[1:] < 0.5)[0]
    return {
        "metric": "particles/s (insertion into two 384^3 half maps)", "value": round(B * steps / (ms / 1e3), 1),
        "unit": "particles/s", "steps": steps, "warmup": warm, "ms_per_step": round(ms / steps, 2),
        "config": {"workload": "iteration-384", "box": box, "ft": 1024, "map": box, "batch_per_step": B,
                   "interp": "trilinear", "ctf": "flip", "nmaps": "two halves (+ full)", "snr": 0.05,
                   "defocus_um": [0.5, 4.0], "l2": f"inputs larger than L2 ({B * box * box * 4 / 1e6:.0f} MB per step)"},
        "finish_ms": {"weigh_ifft_both_halves_and_fsc": round(finish_ms, 1),
                      "again": round(finish_again_ms, 1), "first_call": "allocates the finishing buffers"},
        "fsc_first_shell_below_0.5": int(below[0] + 1) if below.size else None,
        "roofline": {"kernel": "grid4_kernel", "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "avg_launch_ms": round(avg, 3), "algorithmic_bytes_per_particle": per_particle,
                     "tile_shape": int(shape), "autotune_ms_per_shape": [round(float(x), 2) for x in shape_ms]},
        "gpu_launches": int(st1["launches"] - st0["launches"]), "clocks": clk.summary(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=25)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=2000)
    ap.add_argument("--impl", default="gpu")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--search-batch", type=int, default=2048)
    ap.add_argument("--search-steps", type=int, default=3)
    ap.add_argument("--search-warmup", type=int, default=3)
    ap.add_argument("--search-psi", type=int, default=SEARCH_PSI)
    ap.add_argument("--legs", default="insert,search,refine,learned,iter384")
    ap.add_argument("--iter-batch", type=int, default=1000)
    ap.add_argument("--iter-steps", type=int, default=5)
    ap.add_argument("--refine-images", type=int, default=512)
    ap.add_argument("--tile-shape", type=int, default=-1, help="gridding tile shape (default: autotuned)")
    ap.add_argument("--train-images", type=int, default=200000)
    ap.add_argument("--train-epochs", type=float, default=8.0)
    ap.add_argument("--local-radius", type=float, default=10.0)
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def insertion_leg():
        from bsoft_b200.recon import Reconstructor

        B = args.batch
        per_rank = B * (args.warmup + args.steps)
        w = make_workload(max(per_rank, 2 * B))
        plan = plan_for(w)
        P = w["params"]
        pool = w["pool"]
        npool = pool.shape[0]

        # two distinct step buffers (each > L2), alternating between steps
        def step_images(i):
            idx = (np.arange(B) + i * B) % npool
            return np.ascontiguousarray(pool[idx])

        host = [torch.from_numpy(step_images(i)).pin_memory() for i in range(2)]
        dev = [h.cuda() for h in host]
        stream_of = lambda rec: torch.cuda.ExternalStream(rec.stream)

        def barrier():
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()

        # ---- tile shape from the project's autotuner (untimed, on warm-up
        # data), or the one given (profiling runs fix it)
        if args.tile_shape >= 0:
            shape, shape_ms = args.tile_shape, []
        else:
            rec = Reconstructor(plan, batch=B, device=local)
            shape, shape_ms = rec.autotune(dev[0][: min(B, 512)], P[: min(B, 512)])
            rec.close()

        # ---- value: device-resident inputs
        rec = Reconstructor(plan, batch=B, device=local)
        rec.set_tile_shape(shape)
        s = stream_of(rec)
        for i in range(args.warmup):
            rec.insert(dev[i % 2], P[i * B:(i + 1) * B])
        rec.synchronize()
        rec.set_timing(True)
        st0 = rec.stats()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        with ClockSampler(local) as clk:
            ev0.record(s)
            for i in range(args.steps):
                j = args.warmup + i
                rec.insert(dev[j % 2], P[j * B:(j + 1) * B])
            ev1.record(s)
            torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1)
        st1 = rec.stats()
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        particles = B * args.steps * world
        value = particles / (ms / 1e3)
        launches = st1["launches"] - st0["launches"]
        ins_launch = st1["insert_launches"] - st0["insert_launches"]
        ins_ms = st1["insert_ms"] - st0["insert_ms"]
        fft_ms = st1["fft2d_ms"] - st0["fft2d_ms"]
        rec.close()

        # ---- e2e: pinned host images through the C ABI, map read back at the end
        rec = Reconstructor(plan, batch=B, device=local)
        rec.set_tile_shape(shape)
        for i in range(args.warmup):
            rec.insert(host[i % 2].numpy(), P[i * B:(i + 1) * B])
        rec.synchronize()
        rec.reset()
        out = np.empty((BOX, BOX, BOX), dtype=np.float32)
        barrier()
        t0 = time.perf_counter()
        for i in range(args.steps):
            j = args.warmup + i
            rec.insert(host[j % 2].numpy(), P[j * B:(j + 1) * B])
        if dist is not None:
            rec.synchronize()
        rec.finish(0, out=out)
        barrier()
        e2e_s = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([e2e_s], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = particles / e2e_s
        rec.close()
        # the host-to-device copy rate of one step's pinned images alone (the
        # e2e leg moves them every step): a plain copy, CUDA events
        ev0.record()
        dev[0].copy_(host[0], non_blocking=True)
        ev1.record()
        torch.cuda.synchronize()
        h2d_gbs = host[0].numel() * 4 / (ev0.elapsed_time(ev1) / 1e3) / 1e9
        return dict(value=value, ms=ms, e2e=e2e, launches=launches, ins_launch=ins_launch, ins_ms=ins_ms,
                    fft_ms=fft_ms, shape=shape, shape_ms=shape_ms, clk=clk, w=w, B=B, particles=particles,
                    h2d_gbs=h2d_gbs)

    ins = insertion_leg() if "insert" in args.legs else None
    search = search_leg(args, local, dist, world, rank, torch) if "search" in args.legs else None
    iter384 = iteration384_leg(args, local, torch) if ("iter384" in args.legs and rank == 0) else None

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    if ins is not None:
        value, ms, e2e, launches = ins["value"], ins["ms"], ins["e2e"], ins["launches"]
        ins_launch, ins_ms, fft_ms = ins["ins_launch"], ins["ins_ms"], ins["fft_ms"]
        shape, shape_ms, clk, w, B, particles = ins["shape"], ins["shape_ms"], ins["clk"], ins["w"], ins["B"], ins["particles"]
        # roofline of the gridding kernel
        peak, peak_kind = peaks()
        per_particle = 22.0 * BOX * BOX
        avg_launch_ms = ins_ms / max(1, ins_launch)
        achieved = per_particle * B / (avg_launch_ms / 1e3) / 1e9
        # DRAM bytes of one gridding launch, from one ncu capture of this
        # kernel (8^3 tiles, two replicas, half-space gridding, 256^3 map) on
        # a 256-particle batch of this workload: reads 574.2 MB (mostly the
        # spectra, 2.243 MB per particle: the tiles below the split read each
        # particle's spectrum about once) and writes 922.7 MB (the two
        # replicas' partial sums and the unpaired pixels' sums, fixed per
        # launch); scaled to the launch's batch
        traffic = (2.243e6 * B + 0.923e9) if (int(shape) == 0 and BOX == 256) else None
        roof = {"kernel": "grid4_kernel", "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "traffic_unit": ("bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum of a "
                                 "256-particle launch, reads scaled per particle)"),
                "peak_source": peak_kind, "avg_launch_ms": round(avg_launch_ms, 3),
                "algorithmic_bytes_per_particle": per_particle,
                "fft2d_ms_per_step": round(fft_ms / args.steps, 3), "tile_shape": int(shape),
                "autotune_ms_per_shape": [round(float(x), 2) for x in shape_ms]}

        cpu = None
        parity = None
        if world == 1 and not args.no_cpu_baseline:
            threads = cpu_threads_for_reference()
            cpu, d = reference_steady(w, threads)
            if d is not None:
                parity = gpu_parity(d)
                shutil.rmtree(d, ignore_errors=True)

        line = {
            "metric": "particles/s (insertion)", "value": round(value, 1), "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": N_PARTICLES, "particles_timed": particles,
                       "batch_per_step": B, "box": BOX, "map": BOX, "ft": 2 * BOX, "interp": "trilinear",
                       "ctf": "flip", "l2": "inputs larger than L2 (524 MB per step)", "parallelism": f"dp{world}"},
            "e2e": {"value": round(e2e, 1), "unit": "particles/s", "h2d_bytes_per_step": B * BOX * BOX * 4,
                    "d2h_bytes_per_step": BOX ** 3 * 4 // args.steps,
                    "h2d_copy_gbs": round(ins["h2d_gbs"], 1),
                    "copy_bound_particles_per_s": round(ins["h2d_gbs"] * 1e9 / (BOX * BOX * 4), 1)},
            "roofline": roof, "cpu_baseline": cpu, "parity": parity, "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        if search is not None:
            line["search"] = search
            line["gpu_launches"] = int(launches) + search["gpu_launches"] + (
                search["learned"]["gpu_launches"] if search.get("learned") else 0) + (
                search["refine"]["gpu_launches"] if search.get("refine") else 0)
        if iter384 is not None:
            line["iteration_384"] = iter384
            line["gpu_launches"] += iter384["gpu_launches"]
    else:
        line = {"metric": search["metric"], "value": search["value"], "unit": "particles/s", "n_gpus": world,
                "steps": search["steps"], "warmup": search["warmup"], "ms_per_step": search["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": search["dtype"],
                "data": "synthetic", "config": search["config"], "e2e": search["e2e"], "roofline": search["roofline"],
                "cpu_baseline": search["cpu_baseline"], "gpu_launches": search["gpu_launches"],
                "clocks": search["clocks"], "search": search}
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
