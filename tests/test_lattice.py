"""The gridding kernel's phase lattice (bsoft_b200/csrc/lattice.h), chosen per
particle on the host: compiled here with g++ and checked by brute force
(tests/lattice_check.cpp) over random orientations, pixel steps 0.25-1.0 and
plane offsets.  The points of one phase must fall in distinct unit cells of
the map (the kernel's shared-memory updates rely on it), and no lattice may
have more phases than the orientation-independent one used before."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_phase_lattice_is_conflict_free(tmp_path):
    exe = str(tmp_path / "lattice_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe, os.path.join(HERE, "lattice_check.cpp")], check=True)
    r = subprocess.run([exe, "120"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " collisions 0 " in r.stdout and " more_phases_than_before 0 " in r.stdout, r.stdout
    # the Ewald sphere's curved surfaces, with the lattice's curvature margin
    assert " curved_collisions 0 " in r.stdout, r.stdout
