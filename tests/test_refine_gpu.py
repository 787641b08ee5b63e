"""bsg_match_refine (the reference's img_refine_grid on the GPU) against the
reference's own refinement (golden fixtures) and the grid-refinement oracle."""
import math

import numpy as np
import pytest

from tests.refine_helpers import REFINE_CASES, load

pytestmark = pytest.mark.gpu

TOL_FOM = 2e-5       # float32 gather and shell sums in the figure-of-merit kernel


@pytest.fixture(scope="module", params=REFINE_CASES)
def setup(request):
    from bsoft_b200.match import Matcher
    d = load(request.param)
    m = Matcher(n=d["n"], map=d["N"], map_sampling=d["pixel"], pixel=d["pixel"], hi_res=d["hi_res"])
    m.set_reference(d["map"], (d["N"] / 2,) * 3)
    rows = d["ctf_rows"]
    ctf = np.zeros((len(d["images"]), 8))
    ctf[:, :6] = rows[:, :6]
    ctf[:, 6] = rows[:, 6]               # 1: apply (the defocus search applies it anyway)
    m.set_images(d["images"], ctf, d["file_avg"], d["file_std"])
    d["start_rec"] = np.column_stack([np.arange(len(d["images"])), d["start"]])
    yield m, d
    m.close()


def _refine(m, d, start=None, **kw):
    args = dict(alpha_step=d["alpha"], accuracy=d["accuracy"], shift_step=d["shift_step"],
                shift_accuracy=d["shift_accuracy"], def_std=d["def_std"])
    args.update(kw)
    return m.refine(d["start_rec"] if start is None else start, **args)


def test_matches_reference(setup):
    m, d = setup
    out = _refine(m, d)
    ref = d["result"]
    assert np.array_equal(out[:, 8], ref[:, 8]), (out[:, 8], ref[:, 8])     # same hypotheses scored
    assert np.abs(out[:, :4] - ref[:, :4]).max() < 1e-12                     # same views chosen
    assert np.abs(out[:, 4:6] - ref[:, 4:6]).max() < 1e-9                    # same origins
    assert np.abs(out[:, 6] - ref[:, 6]).max() < TOL_FOM
    assert np.abs(out[:, 7] - ref[:, 7]).max() < TOL_FOM
    assert np.array_equal(out[:, 9], ref[:, 9]) or np.abs(out[:, 9] - ref[:, 9]).max() < 1e-9 * np.abs(ref[:, 9]).max()


def test_dpr_matches_reference(setup):
    """brefine -fomtype dpr: the same refinement scored with the DPR figure
    of merit against the reference's img_refine_grid with fom_type 1
    (tests/golden/refine_dpr.npz, make_refine_dpr_golden.py)."""
    import os
    from tests.refine_helpers import GOLDEN
    m, d = setup
    ref = np.load(os.path.join(GOLDEN, "refine_dpr.npz"))[d["case"]]
    out = _refine(m, d, dpr=True)
    assert np.array_equal(out[:, 8], ref[:, 8]), (out[:, 8], ref[:, 8])
    assert np.abs(out[:, :4] - ref[:, :4]).max() < 1e-12
    assert np.abs(out[:, 4:6] - ref[:, 4:6]).max() < 1e-9
    assert np.abs(out[:, 6] - ref[:, 6]).max() < TOL_FOM
    assert np.abs(out[:, 7] - ref[:, 7]).max() < TOL_FOM
    assert np.array_equal(out[:, 9], ref[:, 9]) or np.abs(out[:, 9] - ref[:, 9]).max() < 1e-9 * np.abs(ref[:, 9]).max()


@pytest.mark.parametrize("fom", ["frc", "dpr"])
def test_c_curve_weights_match_reference(setup, fom):
    """brefine weighs the figure of merit's shells with C_curve
    (project_refine_orientations, mg_refine.cpp:366-367): with those weights
    the refinement makes the reference's decisions (tests/golden/
    refine_ccurve.npz, the probe with the same curve), which differ from
    the unit-weight ones by up to a degree."""
    import os
    from tests.refine_helpers import GOLDEN
    m, d = setup
    ref = np.load(os.path.join(GOLDEN, "refine_ccurve.npz"))[f"{d['case']}_{fom}"]
    m.set_c_curve_weights()
    try:
        out = _refine(m, d, dpr=fom == "dpr")
    finally:
        m.set_shell_weights(None)
    assert np.array_equal(out[:, 8], ref[:, 8]), (out[:, 8], ref[:, 8])
    assert np.abs(out[:, :4] - ref[:, :4]).max() < 1e-12
    assert np.abs(out[:, 4:6] - ref[:, 4:6]).max() < 1e-9
    assert np.abs(out[:, 6] - ref[:, 6]).max() < TOL_FOM
    assert np.abs(out[:, 7] - ref[:, 7]).max() < TOL_FOM
    assert np.array_equal(out[:, 9], ref[:, 9]) or np.abs(out[:, 9] - ref[:, 9]).max() < 1e-9 * np.abs(ref[:, 9]).max()
    # unit weights again: the unit-weight fixture's results
    again = _refine(m, d)
    assert np.array_equal(again[:, 8], d["result"][:, 8])


def test_monte_carlo_matches_reference(setup):
    """brefine -monte: img_refine_monte with brefine's shell weights and the
    reference's random() stream for a seed (tests/golden/refine_monte.npz,
    the probe seeded the same way): the same hypotheses, views, origins,
    defoci and sampling (with the magnification steps)."""
    import math
    import os
    from tests.refine_helpers import GOLDEN
    m, d = setup
    z = np.load(os.path.join(GOLDEN, "refine_monte.npz"))
    ref = z[d["case"]]
    it, sh, vw, ang, mag, seed = z[d["case"] + "_params"]
    m.set_c_curve_weights()
    try:
        out = m.refine_monte(d["start_rec"], int(it), def_std=d["def_std"], shift_std=sh, view_std=vw,
                             max_angle=ang * math.pi / 180.0, max_mag=mag, seed=int(seed))
    finally:
        m.set_shell_weights(None)
    assert np.array_equal(out[:, 8], ref[:, 8])
    assert np.abs(out[:, :4] - ref[:, :4]).max() < 1e-9, np.abs(out[:, :4] - ref[:, :4]).max()
    assert np.abs(out[:, 4:6] - ref[:, 4:6]).max() < 1e-9
    assert np.abs(out[:, 6] - ref[:, 6]).max() < TOL_FOM
    assert np.abs(out[:, 7] - ref[:, 7]).max() < TOL_FOM
    if d["def_std"] > 0:
        assert np.abs(out[:, 9] - ref[:, 9]).max() < 1e-6 * np.abs(ref[:, 9]).max()
    if mag > 0:
        cut = float(np.float64(np.longdouble(m.diam) / np.longdouble(d["n"])))
        assert np.abs(out[:, 10:12] - ref[:, 10:12] * cut).max() < 1e-12 * d["pixel"]


def test_magnification_matches_reference(setup):
    """brefine -magnification: the angular rounds, then img_refine_grid's
    magnification stage over 21 x 21 per-axis sampling factors, against the
    reference's img_refine_grid with max_mag > 0 (tests/golden/
    refine_mag.npz, make_refine_mag_golden.py): same hypotheses, views,
    origins, defocus and refined sampling.  The probe prints the sampling of
    the cut transform; the result holds it times the cut scale."""
    import os
    from tests.refine_helpers import GOLDEN
    m, d = setup
    z = np.load(os.path.join(GOLDEN, "refine_mag.npz"))
    ref, max_mag = z[d["case"]], float(z[d["case"] + "_max_mag"])
    out = _refine(m, d, max_mag=max_mag)
    assert np.array_equal(out[:, 8], ref[:, 8]), (out[:, 8], ref[:, 8])
    assert np.abs(out[:, :4] - ref[:, :4]).max() < 1e-12
    assert np.abs(out[:, 4:6] - ref[:, 4:6]).max() < 1e-9
    assert np.abs(out[:, 6] - ref[:, 6]).max() < TOL_FOM
    assert np.abs(out[:, 7] - ref[:, 7]).max() < TOL_FOM
    assert np.array_equal(out[:, 9], ref[:, 9]) or np.abs(out[:, 9] - ref[:, 9]).max() < 1e-9 * np.abs(ref[:, 9]).max()
    cut = float(np.float64(np.longdouble(m.diam) / np.longdouble(d["n"])))
    assert np.abs(out[:, 10:12] - ref[:, 10:12] * cut).max() < 1e-12 * d["pixel"]
    # without the search the pixel size is the particle's own
    plain = _refine(m, d)
    assert np.abs(plain[:, 10:12] - d["pixel"]).max() < 1e-12 * d["pixel"]


def test_batch_invariant_and_repeated_images(setup):
    m, d = setup
    whole = _refine(m, d)
    for i in range(len(d["start_rec"])):
        one = _refine(m, d, start=d["start_rec"][i:i + 1])
        assert np.array_equal(one[0], whole[i])
    # an image may be refined from several starts (symmetry-related views)
    two = _refine(m, d, start=np.concatenate([d["start_rec"][:1], d["start_rec"][:1]]))
    assert np.array_equal(two[0], two[1]) and np.array_equal(two[0], whole[0])


def test_no_shift_levels_returns_start(setup):
    m, d = setup
    out = _refine(m, d, shift_step=0.05, shift_accuracy=0.1, def_std=0.0)
    assert np.all(out[:, 6] == -1) and np.all(out[:, 8] == 0) and np.all(out[:, 7] == 0)
    assert np.allclose(out[:, 4:6], d["start"][:, 4:6], atol=1e-12)
    v = d["start"][:, :3] / np.linalg.norm(d["start"][:, :3], axis=1, keepdims=True)
    assert np.allclose(out[:, :3], v, atol=1e-15)


def test_rejects_bad_steps(setup):
    from bsoft_b200._lib import BsgError
    m, d = setup
    with pytest.raises(BsgError):
        _refine(m, d, alpha_step=math.radians(0.1), accuracy=math.radians(0.5))
    with pytest.raises(BsgError):
        _refine(m, d, accuracy=0.0)
    with pytest.raises(BsgError):
        _refine(m, d, shift_accuracy=0.0)
    bad = d["start_rec"].copy()
    bad[0, 0] = len(d["images"])
    with pytest.raises(BsgError):
        _refine(m, d, start=bad)


def test_defocus_search_needs_a_defocus(setup):
    from bsoft_b200._lib import BsgError
    m, d = setup
    if d["def_std"] > 0:
        pytest.skip("this fixture's images have a defocus; the rejection applies to CTF-free images")
    with pytest.raises(BsgError):
        _refine(m, d, def_std=300.0)


def test_stats_count_refinement(setup):
    m, d = setup
    m.reset_stats()
    _refine(m, d)
    st = m.stats()
    assert st["refine_launches"] >= 3 and st["refine_ms"] > 0
