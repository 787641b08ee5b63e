"""The oracle's restatement of the reference's real-space weighted
back-projection (oracle/backproject_oracle.py: bbackproj's
project_back_projection over Bimage::back_project) against the reference's
own maps (tests/golden/backproject.npz, made by
tests/golden/make_backproject_golden.py with oracle/_ref/backproject_probe):
even images into an equal map and odd images into a larger one, the
untilted view included.  The reference transforms in float, the oracle in
double: relative L2 within 1e-6."""
import os

import numpy as np
import pytest

from oracle.backproject_oracle import back_projection, check_resolution
from tests.helpers import GOLDEN

Z = np.load(os.path.join(GOLDEN, "backproject.npz"))


@pytest.mark.parametrize("key", ["a", "b"])
def test_backprojection_matches_reference(key):
    pixel, res, N = Z[f"{key}_scalars"]
    ref = Z[f"{key}_map"]
    out = back_projection(Z[f"{key}_images"], Z[f"{key}_params"], int(N), float(res), float(pixel))
    assert np.linalg.norm(out.astype(np.float64) - ref) <= 1e-6 * np.linalg.norm(ref)


def test_resolution_limits():
    # at least 2 / sqrt(2 / u^2) = sqrt(2) u, at most the real size
    assert check_resolution(1.0, 16, 1.5) == pytest.approx(1.5 * 2 ** 0.5)
    assert check_resolution(100.0, 16, 1.5) == 24.0
    assert check_resolution(4.0, 16, 1.5) == 4.0
