"""GPU maps at the benchmark configurations, against the reference's own
breconstruct and the FP64 oracle.

* The CPU-runnable configuration in full: 2,000 particles of 64^2 projected
  from a 64^3 phantom of 50 Gaussian blobs, views uniform on SO(3), shifts
  U[-2, 2] px, CTF 200 kV / Cs 2.7 mm / amplitude contrast 0.07 / 1.5 A per
  pixel / defocus U[1, 3] um, noise at SNR 0.1, trilinear insertion, CTF
  flip, pad 2 -> 128^2 transforms, 64^3 map.  The compiled reference
  (oracle/_ref/breconstruct, built from the reference sources) reconstructs
  the same STAR project and stacks; the GPU map must agree to relative
  L2 <= 1e-5 with FSC >= 0.999 on every shell.
* The largest configuration's geometry: 384^2 particles, pad 2 -> 1024^2
  transforms, 384^3 map (384 = 2^7 3: the mixed-radix 3-D inverse
  transform), trilinear, CTF flip, on a few dozen particles against the FP64
  oracle (accumulators and finished map).
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
from bsoft_b200.io import mrc
from bsoft_b200.plan import ReconOptions, ReconPlan, load_images, plan_reconstruction
from bsoft_b200.project import read_project
from bsoft_b200.recon import Reconstructor
from bsoft_b200.synth import DatasetSpec, batched_insertion_workload, generate, write_dataset
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def shell_fsc(a, b):
    """FSC between two real maps on integer shells 1 .. N/2 - 1."""
    A, B = np.fft.fftn(a), np.fft.fftn(b)
    N = a.shape[0]
    f = np.fft.fftfreq(N) * N
    r = np.rint(np.sqrt(f[:, None, None] ** 2 + f[None, :, None] ** 2 + f[None, None, :] ** 2)).astype(int)
    out = []
    for s in range(1, N // 2):
        m = r == s
        out.append(np.real(np.sum(A[m] * np.conj(B[m]))) / np.sqrt(np.sum(abs(A[m]) ** 2) * np.sum(abs(B[m]) ** 2)))
    return np.array(out)


def host_threads():
    try:
        n = len(os.sched_getaffinity(0))
    except Exception:
        n = os.cpu_count() or 1
    return max(1, min(n, 32))


def test_cpu_config_in_full_against_reference(tmp_path):
    exe = oracle.ref_binary("breconstruct")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/breconstruct is not built")
    spec = DatasetSpec(box=64, n_particles=2000, n_blobs=50, pixel=1.5, defocus_range=(1.0e4, 3.0e4),
                       shift_range=2.0, snr=0.1, seed=1)
    ph, imgs, meta = generate(spec)
    d = str(tmp_path)
    star = write_dataset(d, spec, ph, imgs, meta)
    t = host_threads()
    r = subprocess.run([exe, "-interp", "trilinear", "-CTF", "flip", "-threads", str(t), "-recon", "ref.mrc",
                        "particles.star"], cwd=d, env=dict(os.environ, OMP_NUM_THREADS=str(t)),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-400:]
    ref, _ = mrc.read_volume(os.path.join(d, "ref.mrc"))
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=2, ctf_action=1))
    assert (plan.n, plan.ft, plan.map) == (64, 128, 64)
    images = load_images(plan)
    with Reconstructor(plan) as rec:
        rec.insert(images, plan.params)
        m = rec.finish()
    m = m.reshape(ref.shape)
    assert rel_l2(m, ref) <= 1e-5
    assert shell_fsc(m, ref).min() >= 0.999
    orc = oracle.reconstruct(plan, images).reshape(ref.shape)
    assert rel_l2(m, orc) <= 1e-5


@pytest.fixture(scope="module")
def big():
    n = 24
    w = batched_insertion_workload(n_particles=n, box=384, n_blobs=400, pool=n, snr=0.05,
                                   defocus_range=(5000.0, 40000.0), seed=9)
    plan = ReconPlan(n=384, ft=1024, map=384, map_sampling=w["pixel"], hi_res=w["hi_res"], interp=2,
                     ctf_action=1, wiener=0.0, params=w["params"], nmaps=1)
    return plan, np.ascontiguousarray(w["pool"]), w["params"]


def test_384_map_ft1024_against_fp64_oracle(big):
    plan, images, params = big
    with Reconstructor(plan) as rec:
        rec.insert(images, params)
        v, wt = rec.accumulators(0)
        m = rec.finish()
    ov, ow, _, _ = oracle.insert(plan, images, params)
    assert rel_l2(v.reshape(-1), ov.view(np.complex128)) < 1e-6
    assert rel_l2(wt.reshape(-1), ow) < 1e-6
    om, _ = oracle.finish(plan, ov, ow)
    assert rel_l2(m.reshape(-1), om.reshape(-1)) <= 1e-5
