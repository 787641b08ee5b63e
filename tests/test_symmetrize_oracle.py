"""The oracle's restatement of the reference's real-space point-group
symmetrization (oracle/symmetrize_oracle.py: Bimage::symmetrize(sym, 1),
breconstruct -symmetry with sym_mode 1) against the reference's own outputs
(tests/golden/symmetrize.npz, made by tests/golden/make_symmetrize_golden.py
with oracle/_ref/symmetrize_probe): cyclic, dihedral, tetrahedral,
octahedral and icosahedral groups on an even map about its centre and an
odd map about an off-centre origin."""
import os

import numpy as np
import pytest

from oracle.symmetrize_oracle import background, symmetrize
from tests.helpers import GOLDEN

Z = np.load(os.path.join(GOLDEN, "symmetrize.npz"))
GROUPS = [str(g) for g in Z["groups"]]


@pytest.mark.parametrize("key", ["a", "b"])
@pytest.mark.parametrize("group", GROUPS)
def test_symmetrize_matches_reference(key, group):
    m, origin, ref = Z[f"{key}_map"], tuple(Z[f"{key}_origin"]), Z[f"{key}_{group}"]
    out = symmetrize(m, origin, group)
    # float32 maps from the same float64 arithmetic: equal to rounding
    assert np.linalg.norm(out.astype(np.float64) - ref) <= 1e-6 * np.linalg.norm(ref)
    assert np.abs(out.astype(np.float64) - ref).max() <= 1e-6 * np.abs(ref).max()


def test_c1_is_identity_and_background_is_outside_mean():
    m, origin = Z["a_map"], tuple(Z["a_origin"])
    assert np.array_equal(symmetrize(m, origin, "C1"), m)
    n = m.shape[0]
    zz, yy, xx = np.mgrid[:n, :n, :n]
    r = ((xx - origin[0]) / (n // 2)) ** 2 + ((yy - origin[1]) / (n // 2)) ** 2 + \
        ((zz - origin[2]) / (n // 2)) ** 2 - 1
    assert background(m, origin) == pytest.approx(float(m[r > 0].astype(np.float64).mean()), rel=1e-12)
