"""Numerics of the chunked wall-normal Thomas solve (k_ythomas), on CPU.

The CUDA kernel splits every y-line of thomas_kernel! (src/poisson.jl:14-41)
into 32 chunks of MR rows.  The c' entering each chunk is taken from a
per-context table filled once by the reference's sequential recurrence (it
depends on the line's wavenumbers only); the forward and backward sweeps are
carried across chunks as affine maps.  This test restates that formulation
in numpy (vectorised over lines) and compares it, and the sequential Thomas
algorithm, with an extended-precision Thomas solve on the production channel
grid (ny = 256, tanh(1.5) stretching, the modified wavenumbers of a
384 x 384 x-z plane, the pinned mean mode included).
"""
import math

import numpy as np

CHUNKS = 32


def tanh_grid(ny, beta=1.5):
    t = np.arange(ny + 1) / ny
    y = -1 + 2 * (np.tanh(beta * (2 * t - 1)) / math.tanh(beta) + 1) / 2
    dy = np.diff(y)
    yc = 0.5 * (y[1:] + y[:-1])
    dyu = np.diff(yc)
    return dy, dyu


def poisson_rows(ny):
    """Wall-bounded y operator rows (plan_poisson, src/poisson.jl:56-120)."""
    dy, dyu = tanh_grid(ny)
    a = np.zeros(ny)
    c = np.zeros(ny)
    for j in range(ny):
        if j > 0:
            a[j] = 1 / (dy[j] * dyu[j - 1])
        if j < ny - 1:
            c[j] = 1 / (dy[j] * dyu[j])
    return a, -(a + c), c


def modlam(n, L):
    d = L / n
    k = np.arange(n)
    return 2 * (np.cos(2 * np.pi * k / n) - 1) / d ** 2


def thomas_seq(a, b, c, lam, d):
    """Sequential Thomas with the pinned mean mode (lines along axis 0)."""
    ny = len(a)
    pin = lam == 0.0
    x = d.copy()
    cp = np.zeros((ny,) + lam.shape)
    beta = np.where(pin, 1.0, b[0] + lam)
    cp[0] = np.where(pin, 0.0, c[0]) / beta
    x[0] = np.where(pin, 0.0, d[0]) / beta
    for j in range(1, ny):
        beta = (b[j] + lam) - a[j] * cp[j - 1]
        cp[j] = c[j] / beta
        x[j] = (d[j] - a[j] * x[j - 1]) / beta
    for j in range(ny - 2, -1, -1):
        x[j] = x[j] - cp[j] * x[j + 1]
    return x


def thomas_chunked(a, b, c, lam, d, chunks=CHUNKS):
    ny = len(a)
    mr = -(-ny // chunks)
    pin = lam == 0.0

    def row(j):
        if j == 0:
            return (np.zeros_like(lam), np.where(pin, 1.0, b[0] + lam), np.where(pin, 0.0, c[0]))
        return a[j] + 0 * lam, b[j] + lam, c[j] + 0 * lam

    d = d.copy()
    d[0] = np.where(pin, 0.0, d[0])
    rows = [range(k * mr, min(ny, (k + 1) * mr)) for k in range(chunks)]
    # per-context table: c' entering each chunk, by the sequential recurrence
    cin = []
    cprev = np.zeros_like(lam)
    for k, rk in enumerate(rows):
        cin.append(cprev)
        for j in rk:
            aj, bj, cj = row(j)
            cprev = cj / (bj - aj * cprev)
    # forward: local maps (zero carry), carries, rerun from the true carry
    cp = np.zeros_like(d)
    ib = np.zeros_like(d)
    Z, G = [], []
    for k, rk in enumerate(rows):
        cprev = cin[k]
        z = np.zeros_like(d[0])
        g = np.ones_like(lam)
        for j in rk:
            aj, bj, cj = row(j)
            ib[j] = 1.0 / (bj - aj * cprev)
            cprev = cj * ib[j]
            cp[j] = cprev
            z = (d[j] - aj * z) * ib[j]
            g = g * (-aj * ib[j])
        Z.append(z)
        G.append(g)
    carry = np.zeros_like(d[0])  # true d' entering chunk k, composed from the maps
    for k, rk in enumerate(rows):
        dp = carry
        for j in rk:
            d[j] = (d[j] - row(j)[0] * dp) * ib[j]
            dp = d[j]
        carry = Z[k] + G[k] * carry
    # backward: local maps, carries, rerun
    Y, H = [], []
    for rk in rows:
        y = np.zeros_like(d[0])
        h = np.ones_like(lam)
        for j in reversed(rk):
            y = d[j] - cp[j] * y
            h = h * (-cp[j])
        Y.append(y)
        H.append(h)
    x = np.zeros_like(d)
    carry = np.zeros_like(d[0])  # true x after chunk k, composed from the maps
    for k in range(chunks - 1, -1, -1):
        xn = carry
        for j in reversed(rows[k]):
            xn = d[j] - cp[j] * xn
            x[j] = xn
        carry = Y[k] + H[k] * carry
    return x


def test_chunked_matches_sequential_thomas():
    ny, nx, nz = 256, 384, 384
    a, b, c = poisson_rows(ny)
    l1 = modlam(nx, 4 * math.pi)[: nx // 2 + 1]
    l3 = modlam(nz, 4 * math.pi / 3)
    # every kz of a spread of kx planes, the mean mode included
    lam = (l1[[0, 1, 2, 7, 50, 192]][:, None] + l3[None, :]).ravel()
    lam[0] = 0.0
    rng = np.random.default_rng(7)
    d = rng.standard_normal((ny, lam.size))
    xs = thomas_seq(a, b, c, lam, d)
    xc = thomas_chunked(a, b, c, lam, d)
    L = np.longdouble
    xl = thomas_seq(a.astype(L), b.astype(L), c.astype(L), lam.astype(L), d.astype(L))
    scale = np.max(np.abs(xl), axis=0)
    es = np.max(np.abs(xs - xl), axis=0) / scale
    ec = np.max(np.abs(xc - xl), axis=0) / scale
    assert np.all(np.isfinite(xc))
    # as accurate as the sequential algorithm, up to a small factor, on every line
    assert np.all(ec <= np.maximum(4 * es, 1e-13)), np.max(ec / np.maximum(es, 1e-16))
    assert ec.max() <= 5e-12
