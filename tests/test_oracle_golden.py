"""The FP64 oracle against the reference's own breconstruct (golden fixtures
made by tests/golden/make_golden.py from oracle/_ref)."""
import os

import numpy as np
import pytest

import oracle
from tests.helpers import CASES, GOLDEN, load_case, materialize_dataset, ref_tol, rel_l2
from bsoft_b200.plan import P_MAP, ReconOptions, load_images, plan_reconstruction
from bsoft_b200.project import read_project

# float32 reference (FFTW-API stand-in, float maps) vs FP64 restatement
TOL = 1e-5


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference(case, tmp_path):
    plan, images, refs = load_case(case, str(tmp_path))
    if plan.nmaps == 2:
        for h, key in ((0, "map_01"), (1, "map_02")):
            sel = np.nonzero(plan.params[:, P_MAP] == h)[0]
            m = oracle.reconstruct(plan, images, sel)
            assert rel_l2(m, refs[key]) < ref_tol(case), key
    else:
        m = oracle.reconstruct(plan, images)
        assert rel_l2(m, refs["map"]) < ref_tol(case)


@pytest.mark.parametrize("probe", ["probe_ctf16_0", "probe_ctf16_37"])
def test_oracle_particle_stages(probe, tmp_path):
    z = np.load(os.path.join(GOLDEN, probe + ".npz"))
    star = materialize_dataset(str(z["dataset"]), str(tmp_path))
    plan = plan_reconstruction(read_project(star), ReconOptions(interp=int(z["interp"]),
                                                                ctf_action=int(z["ctf_action"])))
    i = int(z["index"])
    img = load_images(plan, [i])[0]
    F = oracle.particle_transform(plan, img, plan.params[i])
    ref = z["ctf"][..., 0] + 1j * z["ctf"][..., 1]
    assert rel_l2(F, ref) < 1e-6
    # that particle's inserted volume and weights
    vol, w, _, _ = oracle.insert(plan, img[None], plan.params[i:i + 1])
    rv = z["vol"].reshape(-1, 2)
    assert rel_l2(vol.reshape(-1, 2), rv) < 1e-6
    assert rel_l2(w, z["w"]) < 1e-6


def test_fsc_matches_reference():
    """orc_fsc against Bimage::fsc of the compiled reference (its shell sums
    are float, hence the tolerance)."""
    z = np.load(os.path.join(GOLDEN, "fsc32.npz"))
    a = np.fft.fftn(z["map1"].astype(np.float64))
    b = np.fft.fftn(z["map2"].astype(np.float64))
    N, u = z["map1"].shape[0], float(z["sampling"])
    for key, res in (("res5", 5.0), ("res3", 3.0)):
        ref = z[key]
        f = oracle.fsc(a, b, N * u, res, len(ref))
        assert len(ref) == int(N * u / res)
        assert np.abs(f - ref[:, 1]).max() < 1e-5
