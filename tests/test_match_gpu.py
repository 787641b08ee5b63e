"""The CUDA matching path (libbsgpu, bsg_match_*) against the reference's
own brefine steps (golden fixtures) and the FP64 oracle."""
import numpy as np
import pytest

import oracle
from tests.match_helpers import MATCH_CASES, ctf_records, hypotheses, load, rel_l2

pytestmark = pytest.mark.gpu

# float32 kernels vs float32 reference output
TOL_SPEC = 2e-6
TOL_SECTION = 2e-5      # 512-tap FP32 accumulation
TOL_FOM = 2e-5


@pytest.fixture(scope="module", params=MATCH_CASES)
def matcher(request):
    from bsoft_b200.match import Matcher
    d = load(request.param)
    m = Matcher(n=d["n"], map=d["N"], map_sampling=d["pixel"], pixel=d["pixel"], hi_res=d["hi_res"])
    m.set_reference(d["map"], d["map_origin"])
    m.set_images(d["images"], ctf_records(d), float(d["file_avg"]), float(d["file_std"]))
    yield m, d
    m.close()


def test_geometry(matcher):
    m, d = matcher
    assert m.diam == d["diam"]
    assert abs(m.info.section_res - m.info.hi_res / 1.11) < 1e-12


def test_reference_transform(matcher):
    m, d = matcher
    t = m.reference_transform()
    assert rel_l2(t, d["map_spec"]) < TOL_SPEC
    assert t[0, 0, 0] == 0


def test_sections(matcher):
    m, d = matcher
    s = m.sections(d["mats"])
    for a, b in zip(s, d["sections"]):
        assert rel_l2(a, b) < TOL_SECTION


def test_prepared_images(matcher):
    m, d = matcher
    p = m.prepared()
    for a, b in zip(p, d["prepared"]):
        assert rel_l2(a, b) < TOL_SPEC


def test_figure_of_merit_dpr(matcher):
    """The DPR figure of merit (brefine -fomtype dpr) of the fixture's
    hypotheses against the reference's own values (tests/golden/match_dpr.npz,
    made by make_match_dpr_golden.py): FP64 scoring to 1e-6, FP32 to 2e-5."""
    import os
    from tests.helpers import GOLDEN
    m, d = matcher
    ref = np.load(os.path.join(GOLDEN, "match_dpr.npz"))[d["name"]]
    f64, cv64 = m.score(hypotheses(d), fp64=True, dpr=True)
    f32, cv32 = m.score(hypotheses(d), dpr=True)
    assert np.abs(f64 - ref[:, 0]).max() < 1e-6 and np.abs(cv64 - ref[:, 1]).max() < 1e-6
    assert np.abs(f32 - ref[:, 0]).max() < TOL_FOM and np.abs(cv32 - ref[:, 1]).max() < TOL_FOM
    # a different figure from the FRC of the same hypotheses
    frc, _ = m.score(hypotheses(d), fp64=True)
    assert np.abs(frc - f64).max() > 1e-3


def test_figure_of_merit(matcher):
    m, d = matcher
    fom, cv = m.score(hypotheses(d))
    assert np.max(np.abs(fom - d["fom"][:, 0])) < TOL_FOM
    assert np.max(np.abs(cv - d["fom"][:, 1])) < TOL_FOM


def test_own_image_statistics(matcher):
    """file_std = 0 normalises each image by its own statistics; the figure
    of merit is scale-invariant, so it is unchanged."""
    m, d = matcher
    m.set_images(d["images"], ctf_records(d))
    fom, _ = m.score(hypotheses(d))
    assert np.max(np.abs(fom - d["fom"][:, 0])) < TOL_FOM
    p = m.prepared()
    o = oracle.match_particle(d["images"][0], d["diam"])
    assert rel_l2(p[0], o) < TOL_SPEC
    m.set_images(d["images"], ctf_records(d), float(d["file_avg"]), float(d["file_std"]))


def test_deterministic(matcher):
    m, d = matcher
    h = hypotheses(d)
    a, _ = m.score(h)
    b, _ = m.score(h[::-1].copy())
    assert np.array_equal(a, b[::-1])


def test_bad_arguments():
    from bsoft_b200.match import Matcher
    from bsoft_b200._lib import BsgError
    with pytest.raises(BsgError):
        Matcher(n=48, map=48, map_sampling=1.5, pixel=1.5, hi_res=3.75)   # not a power of two
    with pytest.raises(BsgError):
        Matcher(n=32, map=64, map_sampling=1.5, pixel=1.5, hi_res=3.0)    # cut edge above the box


def test_projections(matcher):
    """Bimage::project (Fourier projector with the FSI kernel) of the uncut map."""
    m, d = matcher
    p = m.project(d["mats"], resolution=float(d["proj_res"]))
    for a, b in zip(p, d["proj"]):
        assert rel_l2(a, b) < 1e-5


@pytest.mark.parametrize("fp64", [False, True])
def test_full_origin_groups(matcher, fp64):
    """Nine origins of one image and view share one gathered section (a full
    group): each scores as it does alone, in FP32 and in FP64."""
    m, d = matcher
    ox, oy = d["n"] / 2, d["n"] / 2
    hyps = np.array([[0, *d["mats"][0].reshape(9), ox + dx, oy + dy]
                     for dy in (-0.4, 0.0, 0.4) for dx in (-0.4, 0.0, 0.4)])
    f, cv = m.score(hyps, fp64=fp64)
    for i, h in enumerate(hyps):
        f1, cv1 = m.score(h[None], fp64=fp64)
        assert abs(f1[0] - f[i]) < 1e-12 and abs(cv1[0] - cv[i]) < 1e-12
    assert np.all(f != 0)


def test_fp64_scores_match_reference(matcher):
    m, d = matcher
    f, cv = m.score(hypotheses(d), fp64=True)
    f32, _ = m.score(hypotheses(d))
    assert np.abs(f - d["fom"][:, 0]).max() < 1e-6
    assert np.abs(f - f32).max() < 1e-5
