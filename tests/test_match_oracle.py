"""The FP64 matching oracle against the reference's own brefine steps
(golden fixtures made by tests/golden/make_match_golden.py with the
reference library compiled from source)."""
import numpy as np
import pytest

import oracle
from tests.match_helpers import MATCH_CASES, load, rel_l2

# float32 reference data (FFTW-API stand-in) vs FP64 restatement
TOL = 1e-6


@pytest.fixture(scope="module", params=MATCH_CASES)
def case(request):
    d = load(request.param)
    d["spec"] = oracle.match_map(d["map"], d["map_origin"], d["pixel"], d["hi_res"])
    return d


def test_fsi_kernel_rows():
    k = oracle.fsi_kernel(8, 2)
    assert k.shape == (513, 8)
    assert k[0, 3] == 1 and np.count_nonzero(k[0]) == 1          # identity at tap (w-1)/2
    assert k[512, 4] == 1 and np.count_nonzero(k[512]) == 1      # identity one tap later
    # the window sums close to 1 (a partition of unity up to the cos^2 window)
    assert np.all(np.abs(k[1:512].sum(axis=1) - 1) < 0.05)
    assert oracle.fsi_kernel(8, -1).shape == (513, 1)


def test_cut_edge():
    assert oracle.match_diam(48, 1.5, 3.75) == 42
    assert oracle.match_diam(128, 1.5, 3.75) == 114          # 0.8 Nyquist at 128^3
    assert oracle.match_diam(32, 2.0, 4.0) == 32             # never enlarged


def test_reference_map_transform(case):
    assert case["spec"].shape == (case["diam"],) * 3
    assert rel_l2(case["spec"], case["map_spec"]) < TOL
    assert case["spec"][0, 0, 0] == 0


def test_central_sections(case):
    d = case
    k = oracle.fsi_kernel(8, 2)
    samp = d["pixel"] * d["N"] / d["diam"]
    for m, ref in zip(d["mats"], d["sections"]):
        s = oracle.central_section(d["spec"], m, d["diam"] * samp, d["hi_res"] / 1.11, k)
        assert rel_l2(s, ref) < TOL


def test_particle_preparation(case):
    d = case
    for img, ref in zip(d["images"], d["prepared"]):
        p = oracle.match_particle(img, d["diam"], float(d["file_avg"]), float(d["file_std"]))
        assert rel_l2(p, ref) < TOL
        assert p[0, 0] == 0


def test_figure_of_merit(case):
    d = case
    D, N = d["diam"], d["N"]
    samp = d["pixel"] * N / D
    k = oracle.fsi_kernel(8, 2)
    secs = [oracle.central_section(d["spec"], m, D * samp, d["hi_res"] / 1.11, k) for m in d["mats"]]
    preps = [oracle.match_particle(img, D, float(d["file_avg"]), float(d["file_std"])) for img in d["images"]]
    for (i, v, ox, oy), (f, cv) in zip(d["hyps"], d["fom"]):
        x = oracle.phase_shift_2d(preps[int(i)], (ox * D / N, oy * D / N))
        row = d["ctf_rows"][int(i)]
        fo, cvo = oracle.recip_space_fom(x, secs[int(v)], d["n"] * d["pixel"], D * samp, samp, d["hi_res"],
                                         ctf=row[1:6] if row[6] > 0 else None)
        assert abs(fo - f) < 1e-6 and abs(cvo - cv) < 1e-6


def test_figure_of_merit_dpr(case):
    """The DPR form (brefine -fomtype dpr) of the same hypotheses against the
    reference's (tests/golden/match_dpr.npz, make_match_dpr_golden.py)."""
    import os
    from tests.helpers import GOLDEN
    d = case
    ref = np.load(os.path.join(GOLDEN, "match_dpr.npz"))[d["name"]]
    D, N = d["diam"], d["N"]
    samp = d["pixel"] * N / D
    k = oracle.fsi_kernel(8, 2)
    secs = [oracle.central_section(d["spec"], m, D * samp, d["hi_res"] / 1.11, k) for m in d["mats"]]
    preps = [oracle.match_particle(img, D, float(d["file_avg"]), float(d["file_std"])) for img in d["images"]]
    for (i, v, ox, oy), (f, cv) in zip(d["hyps"], ref):
        x = oracle.phase_shift_2d(preps[int(i)], (ox * D / N, oy * D / N))
        row = d["ctf_rows"][int(i)]
        fo, cvo = oracle.recip_space_fom(x, secs[int(v)], d["n"] * d["pixel"], D * samp, samp, d["hi_res"],
                                         fom_type=1, ctf=row[1:6] if row[6] > 0 else None)
        assert abs(fo - f) < 1e-6 and abs(cvo - cv) < 1e-6, (fo, f, cvo, cv)


def test_true_view_scores_best(case):
    """With the CTF applied to the reference, the generating view and origin
    score above the random views (without it the CTF-modulated images
    anticorrelate at low frequency, as in the reference)."""
    d = case
    nimg = len(d["images"])
    f = d["fom"][:, 0].reshape(nimg, -1)
    ctf = d["ctf_rows"][:, 6] > 0
    assert np.all(f[ctf, 0] > f[ctf, 3]) and np.all(f[ctf, 0] > f[ctf, 4])
    assert np.all(f[ctf, 0] > 0.15)


def test_asymmetric_unit_views():
    """The view grid restatement against asymmetric_unit_views of the
    reference (views_probe) for cyclic, dihedral, tetrahedral, octahedral and
    icosahedral groups: bit for bit, with the steps converted as the probe
    converts its degrees (deg * pi / 180)."""
    import math
    import os
    from bsoft_b200.geometry import asymmetric_unit_views, asymmetric_unit_views_c
    from tests.match_helpers import GOLDEN
    z = np.load(os.path.join(GOLDEN, "views.npz"))
    groups = set()
    for key in z.files:
        sym, t, p, f = key.split("_")
        groups.add(sym[0])
        v = asymmetric_unit_views(sym, float(t) * math.pi / 180, float(p) * math.pi / 180,
                                  full=bool(int(f) & 1), inplane=not (int(f) & 2))
        assert v.shape == z[key].shape, key
        assert np.array_equal(v, z[key]), (key, np.abs(v - z[key]).max())
        if sym[0] == "C":
            vc = asymmetric_unit_views_c(int(sym[1:]), float(t) * math.pi / 180, float(p) * math.pi / 180,
                                         full=bool(int(f) & 1), inplane=not (int(f) & 2))
            assert np.array_equal(vc, v)
    assert groups == {"C", "D", "T", "O", "I"}
    assert len(z["C1_3.0_3.0_1"]) == 4586


@pytest.mark.parametrize("sym", ["D3", "C5", "T", "O", "I"])
def test_random_symmetric_views_match_reference(sym):
    """breconstruct -mode 2's view per particle (random_symmetric_view after
    srandom(seed)): the group element random_view_indices picks, applied to
    the particle's matrix, equals the matrix of the view the reference
    returned (oracle/_ref/symview_probe, tests/golden/mode2.npz)."""
    import os
    from bsoft_b200.geometry import view_to_matrix
    from tests.match_helpers import GOLDEN
    from bsoft_b200.symmetry import operators, random_view_indices
    z = np.load(os.path.join(GOLDEN, "mode2.npz"))
    views, out = z[f"views_{sym}__in"], z[f"views_{sym}__out"]
    S = operators(sym)
    idx = random_view_indices(len(views), len(S), int(z[f"views_{sym}__seed"]))
    assert len(set(idx)) > 1
    for v, i, o in zip(views, idx, out):
        got = S[i] @ view_to_matrix(v)
        assert np.abs(got - view_to_matrix(o)).max() < 1e-12, (sym, i)
