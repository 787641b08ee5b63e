"""The identity behind half-space gridding, in FP64 on the CPU.

A real image has a Hermitian transform, F(-q) = conj(F(q)), and trilinear
insertion of pixel q at m = h a + k b and of its mate -q at -m gives
mirrored corners of equal weights.  So the sums P of the pixels whose mate
is in the stored transform (q in [-ft/2, ft/2 - 1]^2) satisfy
P(-v) = conj(P(v)), P_w(-v) = P_w(v), and with U the sums of the unpaired
pixels (row k = -ft/2 and column h = -ft/2) the full map is
conj(P(-v)) + U(v) at every voxel, nothing subtracted.  The GPU kernels
(insert.cu walk_edges, finish.cu read_sums) rely on this; here it is
checked with an independent FP64 gridding of the reference's insertion
(bsoft/src/img/Bimage_reconstruct.cpp:25-88: trilinear, index wrap-around).
"""
import numpy as np


def _rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def _grid(N, ad, bd, pixels, values):
    """Trilinear scatter of values at m = h ad + k bd into an N^3 map."""
    M = np.zeros((N, N, N), complex)
    W = np.zeros((N, N, N))
    h, k = pixels[:, 0][:, None], pixels[:, 1][:, None]
    m = h * ad[None, :] + k * bd[None, :]
    fl = np.floor(m)
    r = m - fl
    i0 = fl.astype(int)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                w = ((r[:, 0] if dx else 1 - r[:, 0]) * (r[:, 1] if dy else 1 - r[:, 1]) *
                     (r[:, 2] if dz else 1 - r[:, 2]))
                x, y, z = (i0[:, 0] + dx) % N, (i0[:, 1] + dy) % N, (i0[:, 2] + dz) % N
                np.add.at(M, (z, y, x), values * w)
                np.add.at(W, (z, y, x), w)
    return M, W


def test_half_space_identity():
    rng = np.random.default_rng(3)
    N, ft = 32, 64
    hf = ft // 2
    F = np.fft.fft2(rng.standard_normal((ft, ft)))            # F[k mod ft, h mod ft]
    R = _rotation(rng)
    ad, bd = R[:, 0] * N / ft, R[:, 1] * N / ft
    hh, kk = np.meshgrid(np.arange(-hf, hf), np.arange(-hf, hf))
    q = np.stack([hh.ravel(), kk.ravel()], axis=1)
    val = F[q[:, 1] % ft, q[:, 0] % ft]
    unpaired = (q[:, 0] == -hf) | (q[:, 1] == -hf)
    full_m, full_w = _grid(N, ad, bd, q, val)
    P, Pw = _grid(N, ad, bd, q[~unpaired], val[~unpaired])
    U, Uw = _grid(N, ad, bd, q[unpaired], val[unpaired])
    mi = (N - np.arange(N)) % N
    mirror = np.ix_(mi, mi, mi)
    zsplit = (N // 2 // 8 + 1) * 8
    assert zsplit < N and ((N - np.arange(zsplit, N)) % N < zsplit).all()
    # above the split: conj(P(-v)) + U(v); below it: P(v) + U(v)
    m = P + U
    w = Pw + Uw
    m[zsplit:] = (np.conj(P[mirror]) + U)[zsplit:]
    w[zsplit:] = (Pw[mirror] + Uw)[zsplit:]
    scale = np.abs(full_m).max()
    assert np.abs(m - full_m).max() < 1e-12 * scale
    assert np.abs(w - full_w).max() < 1e-12 * np.abs(full_w).max()
    # voxels that nothing reaches stay exactly zero
    assert np.array_equal(w == 0, full_w == 0)
    # the unpaired pixels' own sums are needed: the mirror alone is off
    m0 = full_m.copy()
    m0[zsplit:] = np.conj(full_m[mirror])[zsplit:]
    assert np.abs(m0 - full_m).max() > 1e-2 * scale
