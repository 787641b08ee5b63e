"""The grid-refinement oracle (oracle/refine_oracle.py) against the
reference's own img_refine_grid (golden fixtures): refined views and origins
bit for bit, the hypothesis count exactly, the figure of merit to the
float32 precision of the reference's transforms."""
import math

import numpy as np
import pytest

import oracle
from oracle.refine_oracle import CtfSearch, Scorer, origin_grid, refine_grid, views_for_refinement
from tests.refine_helpers import REFINE_CASES, load


@pytest.mark.parametrize("case", REFINE_CASES)
def test_oracle_matches_reference(case):
    d = load(case)
    N, n = d["N"], d["n"]
    spec = oracle.match_map(d["map"], (N / 2,) * 3, d["pixel"], d["hi_res"])
    D = spec.shape[0]
    for i, img in enumerate(d["images"]):
        prep = oracle.match_particle(img, D, d["file_avg"], d["file_std"])
        score = Scorer(spec, prep, n, d["pixel"], N, d["hi_res"])
        st = d["start"][i]
        ctf = CtfSearch(d["volt"], d["ctf_rows"][i, 1:6], d["def_std"]) if d["def_std"] > 0 else None
        v, o, f, cv, num, dz = refine_grid(score, st[:4], (st[4] * (D / n), st[5] * (D / n)), d["alpha"],
                                           d["accuracy"], d["shift_step"], d["shift_accuracy"], ctf)
        ref = d["result"][i]
        assert np.array_equal(np.array(v), ref[:4]), (i, v, ref[:4])
        assert o[0] / (D / n) == ref[4] and o[1] / (D / n) == ref[5]
        assert num == ref[8]
        assert abs(f - ref[6]) < 1e-7 and abs(cv - ref[7]) < 1e-7
        assert dz == ref[9] or (ctf is None and ref[9] == 0)


def test_views_for_refinement_geometry():
    alpha = math.radians(2.0)
    for view in [(0.3, -0.5, 0.8, 1.0), (0.0, 0.0, 1.0, 0.2), (0.0, 0.0, -1.0, -3.0), (1.0, 0.0, 0.0, 3.1)]:
        vs = views_for_refinement(view, alpha)
        assert len(vs) == 27
        c = np.array(vs[13][:3])
        w = np.array(view[:3]) / np.linalg.norm(view[:3])
        assert np.allclose(c, w, atol=1e-15)                       # the centre view is the input
        for v in vs:
            ang = math.acos(min(1.0, float(np.dot(v[:3], w))))
            assert ang <= math.sqrt(2) * alpha * 1.0001             # within the 3 x 3 rotation grid


def test_origin_grid_loops():
    assert len(origin_grid(30.0, 30.0, 0.4)) == 9
    # the reference's floating loop: x - s + s + s can overshoot x + s
    counts = {len(origin_grid(o, 15.0, 0.3)) for o in np.linspace(10, 20, 101)}
    assert counts <= {6, 9}
