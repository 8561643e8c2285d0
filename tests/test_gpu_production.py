"""The production channel at full size against the oracle, and the bounded
device-side wait of the opt-in TMA z-transform.

The 384 x 256 x 384 semi-implicit channel (domain 4pi x 2 x 4pi/3,
tanh(1.5) stretching, nu = 1/395, body force 1, CFL 0.8) starts from the
benchmark's own initial condition (a Reichardt mean profile at
Re_tau = 395 plus splitmix64 noise of amplitude 0.2), is projected, and
takes one CFL step through the C ABI (dnsb_step) and through the CPU
oracle (all host threads).  Tolerances: u <= 1e-12 relative (max-norm over
the field's max), as every one-step test; p as refcases.check_pressure
(1e-12, or twice the oracle's own sensitivity); the divergence is bounded by the
oracle's own (at this grid 1/dy near the walls and |u| ~ 20 lift the
round-off of the discrete divergence above 1e-12 in absolute terms).
"""
import ctypes
import math
import os

import numpy as np
import pytest

import refcases as R

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def D():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import distributednavierstokes_b200 as dns
    from distributednavierstokes_b200 import _lib

    _lib.load()
    return dns


def rel(a, b):
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


def test_production_channel_one_step_full_size(oracle_mod, D):
    import sys

    sys.path.insert(0, ROOT)
    import bench

    O = oracle_mod
    O.set_threads(os.cpu_count() or 1)
    wl = bench.WORKLOADS["channel384_implicit"]
    kw = dict(n=wl["n"], stretch=bench.tanhstretch(1.5), visc=wl["visc"],
              ydiffusion=wl["ydiffusion"], **bench.COMMON)
    so = O.Setup(**kw)
    sd = D.setup(**kw)
    prof = bench.mean_profile(wl)
    # oracle initial field: profile on the u.x faces, then the noise
    u = so.vectorfield()
    nx, ny, nz = so.n
    so.interior(u["x"])[:] = np.broadcast_to(
        prof(so.xf[None, None, :], so.yc[None, :, None], so.zc[:, None, None]), (nz, ny, nx))
    for c in "xyz":
        so.noise(u[c], c, 0, wl["amp"])
    so.exchange_halo(u)
    # device initial field through the mirror (the benchmark's path)
    ud = D.vectorfield(sd)
    D.velocityfield(ud, sd, x=prof)
    for c in "xyz":
        D.noise(ud[c], c, sd, 0, wl["amp"])
    D.exchange_halo(ud, sd)
    for c in "xyz":
        assert rel(ud[c].cpu().numpy(), u[c]) <= 1e-15, c
    p, q, delta = so.scalarfield(), so.vectorfield(), so.scalarfield()
    pd, qd, deltad = D.scalarfield(sd), D.vectorfield(sd), D.scalarfield(sd)
    so.project(u, delta)
    D.project(ud, deltad, sd)
    for c in "xyz":
        assert rel(ud[c].cpu().numpy(), u[c]) <= 1e-12, c
    dt = so.cfl_timestep(u, wl["cfl"])
    dtd = D.cfl_timestep(ud, sd, wl["cfl"])
    assert math.isclose(dt, dtd, rel_tol=1e-13)
    u0, p0 = {c: u[c].copy() for c in "xyz"}, p.copy()
    so.step(u, p, q, delta, dt)
    D.step(ud, pd, qd, deltad, sd, dt)
    for c in "xyz":
        assert rel(ud[c].cpu().numpy(), u[c]) <= 1e-12, c
    R.check_pressure(rel(pd.cpu().numpy(), p), so, u0, p0, dt)
    md_o = so.maxdiv(u)
    md_d = D.maxdiv(ud, sd)
    assert md_d <= max(1e-12, 2 * md_o), (md_d, md_o)
    sd.close()


def test_tma_zfft_wait_runs_out(oracle_mod, D, monkeypatch):
    """DNSB_TMA=1 with a poll limit of 0: every wait of the persistent TMA
    z-transform gives up at once, its CTAs drain their copies and return, and
    the next dnsb_sync reports DNSB_ECUDA; with the limit restored the same
    context solves the Poisson equation to 1e-12 of the oracle."""
    from distributednavierstokes_b200 import _lib

    monkeypatch.setenv("DNSB_TMA", "1")
    kw = dict(n=(16, 12, 40), visc=0.01)   # periodic; nz = 40 (no four-step split)
    so = oracle_mod.Setup(**kw)
    sd = D.setup(**kw)
    lib = _lib.load()
    rng = np.random.default_rng(3)
    r = rng.standard_normal((40, 12, 16))
    r -= r.mean()
    sd.poisson["r"].copy_(torch.from_numpy(r).cuda())
    assert lib.dnsb_set_wait_limit(sd.ctx, 0) == 0
    pd = D.scalarfield(sd)
    D.poisson(pd, sd)
    rc = lib.dnsb_sync(sd.ctx)
    assert rc == 2
    assert b"iteration limit" in lib.dnsb_last_error(sd.ctx)
    assert lib.dnsb_sync(sd.ctx) == 0          # reported once, then cleared
    assert lib.dnsb_set_wait_limit(sd.ctx, 1 << 26) == 0
    D.poisson(pd, sd)
    assert lib.dnsb_sync(sd.ctx) == 0
    po = so.scalarfield()
    so.poisson(r, po)
    assert rel(D.interior(pd).cpu().numpy(), po[1:-1, 1:-1, 1:-1]) <= 1e-12
    sd.close()
