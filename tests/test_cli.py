"""The C++ drop-in `breconstruct` (bsoft_b200/host/breconstruct.cpp) over
libbsgpu: its planning against the Python host mirror (CPU) and its maps
against the compiled reference's breconstruct output (GPU)."""
import os
import shlex
import subprocess

import numpy as np
import pytest

from bsoft_b200.plan import PARTICLE_DOUBLES
from bsoft_b200.io import mrc
from tests.helpers import CASES, GOLDEN, load_case, materialize_dataset, rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "bsoft_b200", "_build", "breconstruct")


@pytest.fixture(scope="module")
def exe():
    if not os.path.exists(EXE):
        from bsoft_b200 import build
        build.build()
    return EXE


def _args(case):
    return shlex.split(str(np.load(os.path.join(GOLDEN, case + ".npz"))["options"]))


@pytest.mark.parametrize("case", CASES)
def test_plan_matches_host_mirror(case, exe, tmp_path):
    plan, _, _ = load_case(case, str(tmp_path))
    star = materialize_dataset(str(np.load(os.path.join(GOLDEN, case + ".npz"))["dataset"]), str(tmp_path))
    r = subprocess.run([exe, *_args(case), "-plan", star], capture_output=True, text=True, check=True)
    lines = r.stdout.strip().splitlines()
    head = lines[0].split()
    kv = {head[i]: head[i + 1] for i in range(0, len(head), 2)}
    assert int(kv["n"]) == plan.n and int(kv["ft"]) == plan.ft and int(kv["map"]) == plan.map
    assert float(kv["map_sampling"]) == plan.map_sampling and float(kv["hi_res"]) == plan.hi_res
    assert int(kv["nmaps"]) == plan.nmaps and float(kv["wiener"]) == plan.wiener
    rec = np.array([[float(t) for t in ln.split()] for ln in lines[1:]]).reshape(-1, PARTICLE_DOUBLES)
    assert rec.shape == plan.params.shape
    assert np.abs(rec - plan.params).max() <= 1e-12 * max(1.0, np.abs(plan.params).max())


def test_rejects_unknown_option(exe, tmp_path):
    r = subprocess.run([exe, "-nonsense", "x.star"], capture_output=True, text=True)
    assert r.returncode != 0 and "unknown option" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_maps_match_reference(case, exe, tmp_path):
    z = np.load(os.path.join(GOLDEN, case + ".npz"))
    star = materialize_dataset(str(z["dataset"]), str(tmp_path))
    out = os.path.join(str(tmp_path), "map.mrc")
    subprocess.run([exe, *_args(case), "-reconstruction", out, star], capture_output=True, text=True, check=True)
    keys = [k for k in z.files if k.startswith("map")]
    for k in keys:
        name = out if k == "map" else out.replace(".mrc", k[3:] + ".mrc")   # map_01 -> map_01.mrc
        h = mrc.read_header(name)
        assert (h.nx, h.ny, h.nz) == z[k].shape[::-1]
        m = np.fromfile(name, dtype="<f4", offset=1024 + h.nsymbt).reshape(z[k].shape)
        assert rel_l2(m, z[k]) < 1e-5, (k, rel_l2(m, z[k]))
