"""Fixture helpers restated from the reference's own test suite.

These mirror test/serialtests.jl:4-41 (tanhstretch, channelsetup,
randomfield!, weighted_dot) and test/mpitests.jl:20-28,86-106 (casesetup,
expectedvalue).  They are written against a generic "setup" object so the
same helpers drive both the oracle (oracle.Setup) and the CUDA library's
host mirror (distributednavierstokes_b200.setup); fields are numpy arrays
of shape (nz+2, ny+2, nx+2).
"""
import math

import numpy as np


def tanhstretch(beta):
    """test/serialtests.jl:4"""
    return lambda t: (math.tanh(beta * (2 * t - 1)) / math.tanh(beta) + 1) / 2


CHANNEL = dict(lims=((0.0, 2 * math.pi), (-1.0, 1.0), (0.0, math.pi)),
               bc=("periodic", "wall", "periodic"))


def channel_kwargs(**kw):
    """channelsetup (test/serialtests.jl:6-13): n = (16, 12, 8), tanh(1.5)."""
    d = dict(n=(16, 12, 8), stretch=tanhstretch(1.5), **CHANNEL)
    d.update(kw)
    return d


def case_kwargs(bcy, **kw):
    """casesetup (test/mpitests.jl:22-28): n = (12, 10, 8)."""
    d = dict(n=(12, 10, 8),
             lims=((0.0, 2 * math.pi), (-1.0, 1.0) if bcy == "wall" else (0.0, 2 * math.pi),
                   (0.0, math.pi)),
             bc=("periodic", bcy, "periodic"),
             stretch=tanhstretch(1.3) if bcy == "wall" else None)
    d.update(kw)
    return d


def active_shape(s, c):
    return tuple(x.stop - x.start for x in s.active(c))


def random_values(s, seed=42):
    """Seeded normal values on all active DOFs (randomfield!,
    test/serialtests.jl:16-23; Julia's MersenneTwister stream cannot be
    reproduced, so numpy's is used)."""
    rng = np.random.default_rng(seed)
    return {c: rng.standard_normal(active_shape(s, c)) for c in "xyz"}


def weighted_dot(u, q, s):
    """test/serialtests.jl:26-41"""
    d = 0.0
    n2 = 0.0
    for c in "xyz":
        sl = s.active(c)
        D2 = s.dyu if c == "y" else s.dy
        vol = s.dx * D2[sl[1]][None, :, None] * s.dz
        d += float(np.sum(vol * u[c][sl] * q[c][sl]))
        n2 += float(np.sum(vol * u[c][sl] ** 2))
    return d, n2


def expectedvalue(stag, g, gi, gj, gk, n, wall):
    """test/mpitests.jl:92-106"""
    ny = n[1]
    if wall:
        if stag == "y":
            if gj == 0 or gj == ny:
                return 0.0
            if gj < 0:
                return -expectedvalue(stag, g, gi, -gj, gk, n, wall)
            if gj > ny:
                return -expectedvalue(stag, g, gi, 2 * ny - gj, gk, n, wall)
        else:
            sgn = 1.0 if stag == "p" else -1.0
            if gj < 1:
                return sgn * expectedvalue(stag, g, gi, 1 - gj, gk, n, wall)
            if gj > ny:
                return sgn * expectedvalue(stag, g, gi, 2 * ny + 1 - gj, gk, n, wall)
    mod1 = lambda a, m: (a - 1) % m + 1
    return g(mod1(gi, n[0]), mod1(gj, n[1]), mod1(gk, n[2]))


def halo_case(s, stag, wall):
    """Field for the halo test (test/mpitests.jl:108-129): returns (phi,
    expected) with phi filled on the active DOFs only."""
    nx, ny, nz = s.n
    g = lambda i, j, k: math.sin(0.7 * i) + math.cos(0.3 * j) * math.sin(0.2 * k)
    phi = np.zeros((nz + 2, ny + 2, nx + 2))
    sl = s.active("p" if stag == "p" else stag)
    for K in range(sl[0].start, sl[0].stop):
        for J in range(sl[1].start, sl[1].stop):
            for I in range(sl[2].start, sl[2].stop):
                phi[K, J, I] = g(I, J, K)
    exp = np.zeros_like(phi)
    for K in range(nz + 2):
        for J in range(ny + 2):
            for I in range(nx + 2):
                exp[K, J, I] = expectedvalue(stag, g, I, J, K, s.n, wall)
    return phi, exp


def poisson_pex(s):
    """Exact pressure of the Poisson test (test/mpitests.jl:137-142)."""
    nx, ny, nz = s.n
    pex = np.zeros((nz + 2, ny + 2, nx + 2))
    for K in range(1, nz + 1):
        for J in range(1, ny + 1):
            for I in range(1, nx + 1):
                pex[K, J, I] = math.sin(0.5 * I) + math.cos(0.3 * J) * math.sin(0.2 * K)
    return pex


RUNCASE_IC = dict(
    x=lambda x, y, z: math.sin(x) * math.cos(y) * math.cos(z) + 0.2 * math.cos(2 * z),
    y=lambda x, y, z: (1 - y ** 2) * math.sin(2 * x),
    z=lambda x, y, z: math.cos(x) * math.sin(z) + 0.1 * math.sin(2 * y),
)
"""Initial field of runcase (test/mpitests.jl:158-172)."""

TG_IC = dict(x=lambda x, y, z: math.sin(x) * math.cos(y),
             y=lambda x, y, z: -math.cos(x) * math.sin(y))
"""Taylor-Green field (test/serialtests.jl:85-90)."""


def _rel(a, b):
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


def pressure_sensitivity(so, u0, p0, dt, seed=1):
    """Relative change of the oracle's one-step pressure when its initial
    velocity u0 (with lagged pressure p0) is perturbed by Gaussian relative
    noise of 4e-16 (about 4 ulp)."""
    rng = np.random.default_rng(seed)

    def run(u):
        u = {c: np.array(u[c]) for c in "xyz"}
        so.exchange_halo(u)
        p = p0.copy()
        q = so.vectorfield()
        d = so.scalarfield() if so.imexy else p
        so.step(u, p, q, d, dt)
        return p

    pa = run(u0)
    pb = run({c: u0[c] * (1 + 4e-16 * rng.standard_normal(u0[c].shape)) for c in "xyz"})
    return _rel(pb, pa)


def check_pressure(err, so, u0, p0, dt):
    """The one-step pressure error err (relative, max-norm) is <= 1e-12, or
    <= 2x the oracle's own sensitivity where that is larger: the pressure
    solves a Poisson problem whose right-hand side, the divergence of the
    intermediate velocity, is a difference of nearly equal fluxes, so the
    round-off of u is amplified in p by the grid's conditioning."""
    if err <= 1e-12:
        return
    sens = pressure_sensitivity(so, u0, p0, dt)
    assert err <= 2 * sens, f"pressure error {err:.3e} > 1e-12 and > 2 x oracle sensitivity {sens:.3e}"
