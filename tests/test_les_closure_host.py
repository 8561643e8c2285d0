"""Host-side measures of the closure study (les_closure.py): the spectral
interpolation of the filtered DNS onto the LES grid's positions, the
dataset normalisation, and the a-posteriori scores (spectrum error,
resolved dissipation, velocity correlation), against closed forms."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from distributednavierstokes_b200 import les_closure as L  # noqa: E402


def _mode_field(M, pos):
    """cos(2 pi (2 x + y)) + 0.5 sin(2 pi 3 z) on a unit box at the grid
    positions pos = (px, py, pz) in units of the spacing, array [z, y, x]."""
    idx = np.arange(M)
    x = (idx + pos[0]) / M
    y = (idx + pos[1]) / M
    z = (idx + pos[2]) / M
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return np.cos(2 * math.pi * (2 * X + Y)) + 0.5 * np.sin(2 * math.pi * 3 * Z)


def test_coarse_to_grid_identity_and_shift():
    """With the fine grid equal to the coarse one, a spectrum of the cell
    centres comes back at the cell centres, and at the faces (x shifted by
    half a cell; y and z likewise) equals the band-limited field there."""
    M = 8
    v = _mode_field(M, (0.5, 0.5, 0.5))
    a_hat = np.fft.rfftn(v, axes=(0, 1, 2)) / M ** 3
    assert np.allclose(L.coarse_to_grid(a_hat, M, M), v, atol=1e-12)
    for stag in ((1.0, 0.5, 0.5), (0.5, 1.0, 0.5), (0.5, 0.5, 1.0)):
        got = L.coarse_to_grid(a_hat, M, M, stag)
        assert np.allclose(got, _mode_field(M, stag), atol=1e-12), stag


def test_coarse_to_grid_from_a_finer_grid():
    """A spectrum taken on a finer grid's cell centres (truncated to the
    coarse wavenumbers, normalised by the fine count) lands on the coarse
    positions: the half-cell offset of the fine centres is removed."""
    M, n = 8, 16
    fine = _mode_field(n, (0.5, 0.5, 0.5))
    full = np.fft.rfftn(fine, axes=(0, 1, 2)) / n ** 3
    keep = np.r_[0:M // 2, n - M // 2:n]
    a_hat = full[np.ix_(keep, keep, np.arange(M // 2 + 1))]
    a_hat[:, :, M // 2] = 0.0  # the coarse Nyquist column is not a retained mode here
    got = L.coarse_to_grid(a_hat, M, n, (1.0, 0.5, 0.5))
    assert np.allclose(got, _mode_field(M, (1.0, 0.5, 0.5)), atol=1e-12)


def test_normalise_scales():
    rng = np.random.default_rng(3)
    pairs = []
    for _ in range(4):
        ub = rng.standard_normal((3, 4, 4, 4)) * np.array([1.0, 2.0, 4.0])[:, None, None, None]
        tau = rng.standard_normal((6, 4, 4, 4)) * 0.1
        pairs.append((None, ub, tau))
    data, insc, outsc = L.normalise(pairs)
    assert data.shape == (4, 9, 4, 4, 4) and data.dtype == np.float32
    assert np.allclose(data.std(axis=(0, 2, 3, 4)), 1.0, atol=1e-5)
    ub = np.stack([p[1] for p in pairs])
    assert np.allclose(insc, 1.0 / ub.std(axis=(0, 2, 3, 4)), rtol=1e-6)
    assert outsc.shape == (6,) and np.all(outsc > 0)


def test_spectrum_error_and_dissipation():
    mean, mx = L.spectrum_error([1.0, 2.0, 3.0], [1.0, 4.0, 2.0])
    assert math.isclose(mean, (0.0 + 0.5 + 0.5) / 3) and math.isclose(mx, 0.5)
    # 2 nu sum (2 pi k / l)^2 E(k): on l = 2 pi, k = 1 and 3 carry energy
    assert math.isclose(L.resolved_dissipation([1.0, 0.0, 2.0], 0.01), 2 * 0.01 * (1 + 9 * 2))
    assert math.isclose(L.resolved_dissipation([1.0], 0.5, l=1.0), 2 * 0.5 * (2 * math.pi) ** 2)


def test_correlation():
    """sum_c <u_c, ref_c> / |u| |ref| over the interiors: 1 for equal
    fields, -1 for opposite ones, the cosine for mixed ones."""
    rng = np.random.default_rng(5)
    M = 6
    ref = {c: rng.standard_normal((M, M, M)) for c in "xyz"}

    def ghosted(vals):
        out = {}
        for c in "xyz":
            g = torch.zeros((M + 2, M + 2, M + 2), dtype=torch.float64)
            g[1:-1, 1:-1, 1:-1] = torch.from_numpy(vals[c])
            out[c] = g
        return out

    assert math.isclose(L.correlation(ghosted(ref), ref), 1.0, rel_tol=1e-12)
    assert math.isclose(L.correlation(ghosted({c: -ref[c] for c in "xyz"}), ref), -1.0, rel_tol=1e-12)
    other = {c: rng.standard_normal((M, M, M)) for c in "xyz"}
    a = np.concatenate([ref[c].ravel() for c in "xyz"])
    b = np.concatenate([other[c].ravel() for c in "xyz"])
    cos = float(a @ b / math.sqrt((a @ a) * (b @ b)))
    assert math.isclose(L.correlation(ghosted(other), ref), cos, rel_tol=1e-12)
