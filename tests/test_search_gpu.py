"""The exhaustive search (bsg_match_set_panel / bsg_match_search): the BF16
tensor-core correlation against an FP64 numpy evaluation of the same
shell-normalised correlation, the exact rescoring against bsg_match_score,
and the recovery of the generating views."""
import math

import numpy as np
import pytest

from bsoft_b200.geometry import random_views, views_to_matrices
from bsoft_b200.ctf import electron_wavelength
from tests.match_helpers import ctf_records, load

pytestmark = pytest.mark.gpu

N_RANDOM = 700


def wrapped(i, L):
    return i - L if i > (L - 1) // 2 else i


def coarse_scores(m, d, mats, origins, ctf):
    """The correlation the search computes, in FP64: per image and origin
    row X e^{i phi} c / (n_f sqrt(D_j C_j)), per section R / sqrt(M_j), over
    the half-plane pixels of shells 1 .. n_f - 1."""
    info = m.info
    D, n = m.diam, d["n"]
    us = d["pixel"] * d["N"] / D
    real_map = D * us
    nf = int(math.ceil(info.max_rad))
    maxs2 = 1.0 / info.section_res ** 2
    pix = []
    for yy in range(D):
        for xx in range(D):
            h, k = wrapped(xx, D), wrapped(yy, D)
            j = int(math.sqrt(h * h + k * k))
            if not (1 <= j < nf):
                continue
            if (h / real_map) ** 2 + (k / real_map) ** 2 > maxs2:
                continue
            if not (k > 0 or (k == 0 and h > 0)):
                continue
            pix.append((h, k, yy * D + xx, j))
    pix = np.array(pix)
    h, k, idx, sh = pix[:, 0], pix[:, 1], pix[:, 2], pix[:, 3]
    X = m.prepared().reshape(len(d["images"]), -1)[:, idx].astype(np.complex128)
    R = m.sections(mats).reshape(len(mats), -1)[:, idx].astype(np.complex128)
    fs = 1.0 / (n * d["pixel"])
    s2 = (fs * h) ** 2 + (fs * k) ** 2
    ang = np.arctan2(k, h)
    C = np.ones((len(X), len(idx)))
    for i, r in enumerate(ctf):
        t2 = -math.pi * electron_wavelength(r[0])
        if int(r[6]) & 1 and r[2] / t2 >= 1:
            chi = r[1] + s2 * (r[4] * np.sin(2 * ang) + r[2] + r[3] * np.cos(2 * ang)) + s2 * s2 * r[5]
            C[i] = np.sin(chi)
    Mj = np.zeros((len(R), nf))
    Dj = np.zeros((len(X), nf))
    Cj = np.zeros((len(X), nf))
    cnt = np.bincount(sh, minlength=nf)
    for j in range(1, nf):
        sel = sh == j
        Mj[:, j] = (np.abs(R[:, sel]) ** 2).sum(1)
        Dj[:, j] = (np.abs(X[:, sel]) ** 2).sum(1)
        Cj[:, j] = (C[:, sel] ** 2).sum(1) / cnt[j]
    B = R / np.sqrt(np.where(Mj[:, sh] > 0, Mj[:, sh], np.inf))
    g = 1.0 / (nf * np.sqrt(np.where(Dj * Cj > 0, Dj * Cj, np.inf)))
    out = np.zeros((len(X), len(origins), len(R)))
    for o, (ox, oy) in enumerate(origins):
        sx = (D / n) * ox / D * 2 * math.pi
        sy = (D / n) * oy / D * 2 * math.pi
        A = X * np.exp(1j * (h * sx + k * sy))[None] * C * g[:, sh]
        out[:, o, :] = (A @ B.conj().T).real
    return out


@pytest.fixture(scope="module")
def setup():
    from bsoft_b200.match import Matcher
    d = load("match64")
    rng = np.random.default_rng(7)
    views = np.concatenate([d["true_views"], random_views(rng, N_RANDOM)])
    mats = views_to_matrices(views)
    origins = np.array([(d["n"] // 2 + dx, d["n"] // 2 + dy) for dy in (-1, 0, 1) for dx in (-1, 0, 1)], float)
    ctf = ctf_records(d)
    m = Matcher(n=d["n"], map=d["N"], map_sampling=d["pixel"], pixel=d["pixel"], hi_res=d["hi_res"], batch=4)
    m.set_reference(d["map"], d["map_origin"])
    m.set_images(d["images"], ctf, float(d["file_avg"]), float(d["file_std"]))
    m.set_panel(mats)
    res = m.search(origins, topk=8)
    ref = coarse_scores(m, d, mats, origins, ctf)
    yield m, d, mats, origins, ctf, res, ref
    m.close()


def test_correlation_matches_fp64(setup):
    m, d, mats, origins, ctf, res, ref = setup
    scale = np.abs(ref).max()
    for i in range(len(d["images"])):
        for sec, org, score, fom, cv in res[i]:
            assert sec >= 0
            assert abs(score - ref[i, int(org), int(sec)]) < 1e-2 * scale
        # the best coarse candidate is the FP64 maximum up to BF16 rounding
        assert res[i][:, 2].max() > ref[i].max() - 1e-2 * scale


def test_top_candidates_are_the_fp64_top(setup):
    """Candidates are the 8 best by the BF16 score: every FP64 score clearly
    above the 8th best appears among them."""
    m, d, mats, origins, ctf, res, ref = setup
    scale = np.abs(ref).max()
    for i in range(len(d["images"])):
        flat = ref[i].reshape(-1)
        order = np.argsort(flat)[::-1]
        kth = flat[order[7]]
        got = {(int(s), int(o)) for s, o in res[i][:, :2]}
        for f in order[:8]:
            if flat[f] > kth + 2e-2 * scale:
                o, s = divmod(int(f), len(mats))
                assert (s, o) in got


def test_rescored_figure_of_merit(setup):
    m, d, mats, origins, ctf, res, ref = setup
    hyps = []
    for i in range(len(d["images"])):
        for sec, org, *_ in res[i]:
            hyps.append([i, *mats[int(sec)].reshape(9), *origins[int(org)]])
    fom, cv = m.score(np.array(hyps))
    got = res[:, :, 3].reshape(-1)
    assert np.max(np.abs(fom - got)) < 1e-12
    assert np.max(np.abs(cv - res[:, :, 4].reshape(-1))) < 1e-12
    assert np.all(np.diff(res[:, :, 3], axis=1) <= 0)     # best first


def test_rescoring_reads_the_panels_exact_sections(setup):
    """The panel keeps its FP32 sections at the figure-of-merit pixels and
    the rescoring reads them: the search gives the same records, to the
    bit, as with the sections gathered per candidate, and the local search
    too."""
    m, d, mats, origins, ctf, res, ref = setup
    assert m.stats()["panel_exact_bytes"] > 0
    m.set_panel(mats, exact_sections=False)
    try:
        gathered = m.search(origins, topk=8)
        props = np.zeros((len(d["images"]), 11), np.float32)
        props[:, :9] = mats[:len(d["images"])].reshape(-1, 9)
        props[:, 9:] = 0
        local_g = m.search_local(props, origins, 10.0, 1.5, 8)
    finally:
        m.set_panel(mats)
    assert np.array_equal(gathered, res)
    assert np.array_equal(m.search_local(props, origins, 10.0, 1.5, 8), local_g)


def test_generating_views_found(setup):
    """Images whose CTF is applied recover their own view and a trial
    origin within 1.5 pixels of the true one (the grid step is 1 pixel and
    the figure of merit of one noisy image is flat to a few tenths of a pixel)."""
    m, d, mats, origins, ctf, res, ref = setup
    for i in range(len(d["images"])):
        if not int(ctf[i, 6]) & 1:
            continue
        assert int(res[i, 0, 0]) == i
        assert np.abs(origins[int(res[i, 0, 1])] - d["true_origins"][i][:2]).max() < 1.5


def test_search_deterministic(setup):
    m, d, mats, origins, ctf, res, ref = setup
    again = m.search(origins, topk=8)
    assert np.array_equal(again, res)


def test_stats(setup):
    m, *_ = setup
    st = m.stats()
    assert st["gemm_flops"] > 0 and st["gemm_ms"] > 0 and st["gemm_launches"] >= 2
    assert st["kpad"] % 64 == 0 and st["coarse_k"] <= st["kpad"]


def _perturb(R, deg, rng):
    ax = rng.normal(size=3)
    ax /= np.linalg.norm(ax)
    a = math.radians(deg)
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    return (np.eye(3) + math.sin(a) * K + (1 - math.cos(a)) * K @ K) @ R


def test_local_search_around_proposals(setup):
    """Proposals a few degrees and ~0.5 pixel off the truth: the local
    search finds the generating view, and its correlation scores equal the
    exhaustive search's for the same (section, origin) pairs."""
    m, d, mats, origins, ctf, res, ref = setup
    rng = np.random.default_rng(11)
    nimg = len(d["images"])
    prop = np.zeros((nimg, 11), np.float32)
    for i in range(nimg):
        prop[i, :9] = _perturb(d["mats"][i], 4.0, rng).reshape(9)
        prop[i, 9:] = d["true_origins"][i][:2] - d["n"] // 2 + rng.uniform(-0.5, 0.5, 2)
    loc = m.search_local(prop, origins, radius_deg=10.0, origin_radius=1.5, topk=8)
    scale = np.abs(ref).max()
    for i in range(nimg):
        for sec, org, score, fom, cv in loc[i]:
            if sec < 0:
                continue
            assert abs(score - ref[i, int(org), int(sec)]) < 1e-2 * scale
        if int(ctf[i, 6]) & 1:
            assert int(loc[i, 0, 0]) == i
    # exact rescoring as in the exhaustive search
    hyps = [[i, *mats[int(s)].reshape(9), *origins[int(o)]] for i in range(nimg) for s, o, *_ in loc[i] if s >= 0]
    fom, _ = m.score(np.array(hyps))
    got = np.array([f for i in range(nimg) for s, o, sc, f, cv in loc[i] if s >= 0])
    assert np.max(np.abs(fom - got)) < 1e-12
