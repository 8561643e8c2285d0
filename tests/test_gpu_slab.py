"""The z-slab decomposition (slab.py, the reference's (P,1) process grid):
P ranks emulated in one process on one GPU (every exchange a device copy,
no kernel waits on another) against the 1-rank step — the reference's
decomposition-invariance check (test/mpitests.jl:158-198, 1e-11)."""
import math

import numpy as np
import pytest

import refcases as R

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CASES = {
    "periodic": dict(n=(16, 12, 16), visc=0.01, bodyforce=(0.3, 0.1, -0.2)),
    "channel": dict(n=(16, 12, 16), lims=((0, 2.0), (-1, 1), (0, 1.5)), bc=("periodic", "wall", "periodic"),
                    stretch=R.tanhstretch(1.3), visc=0.02, bodyforce=(1.0, 0.0, 0.0)),
    "channel_implicit": dict(n=(16, 24, 16), lims=((0, 2.0), (-1, 1), (0, 1.5)),
                             bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5),
                             visc=0.02, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"),
}


@pytest.fixture(scope="module")
def D():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import distributednavierstokes_b200 as dns
    from distributednavierstokes_b200 import slab

    return dns, slab


def rel(a, b):
    return float((a - b).abs().max()) / max(float(b.abs().max()), 1e-300)


@pytest.mark.parametrize("P", [2, 4])
@pytest.mark.parametrize("case", list(CASES))
def test_slab_step_equals_one_rank(D, case, P):
    dns, slab = D
    kw = CASES[case]
    s = dns.setup(**kw)
    u = dns.vectorfield(s)
    for i, c in enumerate("xyz"):
        dns.noise(u[c], c, s, 3 + i, 0.5)
    dns.exchange_halo(u, s)
    p = dns.scalarfield(s)
    dns.project(u, p, s)
    dt = 0.5 * dns.cfl_timestep(u, s, 0.5)
    comm = slab.LocalComm(P)
    parts, sg = slab.make_parts(comm, kw)
    us = {c: slab.scatter(parts, u[c]) for c in "xyz"}
    implicit = s.imexy
    if implicit:
        p.zero_()           # the lagged pressure starts at zero (solve!); delta holds the projection
    ps = slab.scatter(parts, p)
    st = {r: (dns.VectorField(x=us["x"][r], y=us["y"][r], z=us["z"][r]), ps[r], dns.vectorfield(parts[r].s))
          + ((dns.scalarfield(parts[r].s),) if implicit else ()) for r in parts}
    # the slab pieces of the projection alone: divergence-free to 1e-12
    assert slab.maxdiv(parts, comm, lambda p_: st[p_.rank][0]) < 1e-12
    assert math.isclose(slab.cfl_timestep(parts, comm, lambda p_: st[p_.rank][0], 0.5), 2 * dt,
                        rel_tol=1e-13)
    q = dns.vectorfield(s)
    delta = dns.scalarfield(s) if implicit else None
    for _ in range(3):
        dns.step(u, p, q, delta, s, dt)
        slab.step(parts, comm, lambda p_: st[p_.rank], dt)
    nz = kw["n"][2]
    for c in "xyz":
        got = slab.gather_interior(parts, {r: st[r][0][c] for r in parts}, nz)
        assert rel(got[:, 1:-1, 1:-1], u[c][1:-1, 1:-1, 1:-1]) <= 1e-11, c
    gp = slab.gather_interior(parts, {r: st[r][1] for r in parts}, nz)
    assert rel(gp[:, 1:-1, 1:-1], p[1:-1, 1:-1, 1:-1]) <= 1e-11
    assert slab.maxdiv(parts, comm, lambda p_: st[p_.rank][0]) < 1e-12
    for part in parts.values():
        part.close()
    sg.close()
    s.close()
