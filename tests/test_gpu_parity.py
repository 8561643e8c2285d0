"""GPU parity: libdnsb.so (through its C ABI, via the host mirror) against
the CPU oracle on the same seeded inputs, plus the reference's own identity
and known-answer tests run on the GPU path.

Tolerances (FP64): operators and one RK3 step agree with the oracle to
<= 1e-12 relative (max-norm, relative to the field's max); 100 steps of the
64^3 channel to <= 1e-9; halo fills are exact; divergence after projection
< 1e-12 as in the reference.  The pressure after one step is held to
1e-12 too, or to twice the oracle's own change under a 4-ulp perturbation
of its initial velocity where that is larger (check_pressure): the step's
pressure solves a Poisson problem whose right-hand side is the divergence
of the intermediate velocity, a difference of nearly equal fluxes, so
round-off of u is amplified in p by the grid's conditioning (on the 256-row
tanh(1.5) channel both the device-vs-oracle difference and the oracle's own
sensitivity are about 1.0e-12 to 1.7e-12; everywhere else <= 2.6e-13).
"""
import ctypes
import math
import os

import numpy as np
import pytest

import refcases as R

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL_STEP = 1e-12


@pytest.fixture(scope="module")
def D():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import distributednavierstokes_b200 as dns
    from distributednavierstokes_b200 import _lib

    _lib.load()
    return dns


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def N(t):
    return t.detach().cpu().numpy()


def both(O, D, **kw):
    return O.Setup(**kw), D.setup(**kw)


def rel(a, b):
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale


def rand_fields(so, seed=42):
    u = so.vectorfield()
    vals = R.random_values(so, seed)
    for c in "xyz":
        u[c][so.active(c)] = vals[c]
    so.exchange_halo(u)
    return u


def to_dev(D, u):
    return D.VectorField(x=T(u["x"]), y=T(u["y"]), z=T(u["z"]))


check_pressure = R.check_pressure



GRID_CASES = {
    "periodic": dict(n=(16, 12, 8), visc=0.01, bodyforce=(0.3, 0.1, -0.2)),
    "channel": R.channel_kwargs(visc=0.05, bodyforce=(1.0, 0.0, 0.0)),
    "channel_implicit": R.channel_kwargs(visc=0.05, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"),
    "ragged": dict(n=(12, 10, 6), lims=((0.0, 2.0), (-1.0, 1.0), (0.0, 3.0)),
                   bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.3), visc=0.02),
    "c1_shape": dict(n=(24, 20, 12), lims=((0, 4 * math.pi), (-1, 1), (0, 4 * math.pi / 3)),
                     bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5),
                     visc=1 / 180, bodyforce=(1.0, 0.0, 0.0)),
}


# --------------------------------------------------------------- halo fill

@pytest.mark.parametrize("bcy", ["periodic", "wall"])
@pytest.mark.parametrize("stag", ["x", "y", "z", "p"])
def test_halo_exact(oracle_mod, D, bcy, stag):
    """test/mpitests.jl:108-129 on the GPU: exact equality."""
    s = D.setup(**R.case_kwargs(bcy))
    phi, exp = R.halo_case(s, stag, bcy == "wall")
    t = T(phi)
    D.exchange_halo(t, stag, s)
    assert np.array_equal(N(t), exp)


# --------------------------------------------------------------- operators

@pytest.mark.parametrize("cfg", list(GRID_CASES))
def test_divergence_momentum_gradient(oracle_mod, D, cfg):
    so, sd = both(oracle_mod, D, **GRID_CASES[cfg])
    u = rand_fields(so)
    ud = to_dev(D, u)
    r = so.divergence(u)
    rd = sd.poisson["r"]
    D.divergence(rd, ud, sd)
    assert rel(N(rd), r) <= 1e-13
    for A, dt in ((0.0, 1.0), (-5 / 9, 0.01)):
        q = so.vectorfield()
        qvals = R.random_values(so, 7)
        for c in "xyz":
            q[c][so.active(c)] = qvals[c]
        qd = to_dev(D, q)
        so.momentum(q, u, A, dt)
        D.momentum(qd, ud, A, dt, sd)
        for c in "xyz":
            assert rel(N(qd[c]), q[c]) <= 1e-13, (c, A)
    p = so.scalarfield()
    p[so.active("p")] = np.random.default_rng(3).standard_normal(R.active_shape(so, "p"))
    so.fill_halo(p, "p")
    pd = T(p)
    for c in "xyz":
        so.pressuregrad_component(u[c], p, c, 0.7)
        D.pressuregrad_component(ud[c], pd, c, 0.7, sd)
        assert rel(N(ud[c]), u[c]) <= 1e-13


@pytest.mark.parametrize("cfg", ["periodic", "channel", "ragged"])
def test_poisson_and_project(oracle_mod, D, cfg):
    so, sd = both(oracle_mod, D, **GRID_CASES[cfg])
    u = rand_fields(so)
    ud = to_dev(D, u)
    r = so.divergence(u)
    p = so.scalarfield()
    so.poisson(r, p)
    sd.poisson["r"].copy_(T(r))
    pd = D.scalarfield(sd)
    D.poisson(pd, sd)
    assert rel(N(pd), p) <= 1e-12
    psi = so.scalarfield()
    so.project(u, psi)
    psid = D.scalarfield(sd)
    D.project(ud, psid, sd)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= 1e-12
    assert rel(N(psid), psi) <= 1e-12
    assert D.maxdiv(ud, sd) < 1e-12


@pytest.mark.parametrize("bcy", ["periodic", "wall"])
def test_poisson_recovers_pressure(oracle_mod, D, bcy):
    """test/mpitests.jl:133-154 on the GPU."""
    s = D.setup(**R.case_kwargs(bcy))
    pex = T(R.poisson_pex(s))
    D.exchange_halo(pex, "p", s)
    u = D.vectorfield(s)
    D.pressuregrad_update(u, pex, s)
    D.exchange_halo(u, s)
    D.divergence(s.poisson["r"], u, s)
    p2 = D.scalarfield(s)
    D.poisson(p2, s)
    d = N(D.interior(p2)) + N(D.interior(pex))
    assert np.max(np.abs(d - d.mean())) < 1e-8


def test_imex_update(oracle_mod, D):
    so, sd = both(oracle_mod, D, **GRID_CASES["channel_implicit"])
    u = rand_fields(so)
    q = rand_fields(so, 5)
    p = so.scalarfield()
    p[so.active("p")] = np.random.default_rng(9).standard_normal(R.active_shape(so, "p"))
    so.fill_halo(p, "p")
    ud, qd, pd = to_dev(D, u), to_dev(D, q), T(p)
    so.imex_update(u, q, p, 15 / 16, 5 / 12, 0.01)
    D.imex_update(ud, qd, pd, 15 / 16, 5 / 12, 0.01, sd)
    for c in "xyz":
        sl = so.active(c)
        assert rel(N(ud[c])[1:-1, 1:-1, 1:-1], u[c][1:-1, 1:-1, 1:-1]) <= 1e-13, c


# ----------------------------------------------------------------- stepping

@pytest.mark.parametrize("cfg", list(GRID_CASES))
def test_one_step(oracle_mod, D, cfg):
    """One RK3 step from the same projected random field: <= 1e-12 relative."""
    so, sd = both(oracle_mod, D, **GRID_CASES[cfg])
    u = rand_fields(so)
    p = so.scalarfield()
    so.project(u, p)
    ud, pd = to_dev(D, u), T(p)
    q, qd = so.vectorfield(), D.vectorfield(sd)
    delta = so.scalarfield() if so.imexy else p
    deltad = D.scalarfield(sd) if sd.imexy else pd
    dt = 0.5 * so.cfl_timestep(u, 0.5)
    u0, p0 = {c: u[c].copy() for c in "xyz"}, p.copy()
    so.step(u, p, q, delta, dt)
    D.step(ud, pd, qd, deltad, sd, dt)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= TOL_STEP, c
        assert rel(N(qd[c]), q[c]) <= 1e-11, c
    check_pressure(rel(N(pd), p), so, u0, p0, dt)
    assert D.maxdiv(ud, sd) < 1e-12


# Production lengths in one direction at a time (the other two small, so the
# oracle stays fast): ny = 256 takes the 16-row Crank-Nicolson chunks and the
# 8-row chunked Poisson y-solve; nx = nz = 384 take the four-step 16 x 12
# x-transforms and 16 x 24 z-transforms of the 384 x 256 x 384 benchmark.
PRODUCTION = {
    "ny256": dict(n=(16, 256, 8), lims=((0, 4 * math.pi), (-1, 1), (0, 4 * math.pi / 3)),
                  bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5),
                  visc=1 / 395, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"),
    "nx384_nz384": dict(n=(384, 8, 384), lims=((0, 4 * math.pi), (-1, 1), (0, 4 * math.pi / 3)),
                        bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5),
                        visc=1 / 395, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"),
    # two x tiles with two wrap columns, several y tiles with both walls
    "nx64_ny40": dict(n=(64, 40, 24), lims=((0, 4 * math.pi), (-1, 1), (0, 4 * math.pi / 3)),
                      bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5),
                      visc=1 / 395, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"),
    # the fused z-FFT / y-solve / inverse z-FFT (one cluster of ny/32 CTAs per
    # kx plane): 8, 1 and 2 chunks, nz = 384 and 256
    "zyz_ny256_nz384": dict(n=(8, 256, 384), lims=((0, 4 * math.pi), (-1, 1), (0, 4 * math.pi / 3)),
                            bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5),
                            visc=1 / 395, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"),
    "zyz_ny32_nz384": dict(n=(12, 32, 384), lims=((0, 4 * math.pi), (-1, 1), (0, 4 * math.pi / 3)),
                           bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5),
                           visc=1 / 395, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"),
    "zyz_ny64_nz256": dict(n=(16, 64, 256), lims=((0, 4 * math.pi), (-1, 1), (0, 4 * math.pi / 3)),
                           bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.2),
                           visc=1 / 180, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"),
}

ZYZ = {
    "zyz_ny96_nz256_explicit": dict(n=(8, 96, 256), lims=((0, 2.0), (-1, 1), (0, 3.0)),
                                    bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.3),
                                    visc=0.02),
    "zyz_ny256_nz384": PRODUCTION["zyz_ny256_nz384"],
}


@pytest.mark.parametrize("mode", ["1", "2"])
@pytest.mark.parametrize("cfg", list(ZYZ))
def test_fused_poisson_kernel(oracle_mod, D, cfg, mode, monkeypatch):
    """With DNSB_ZYZ=1 (32-row chunks, one CTA per SM) or 2 (16-row chunks,
    two CTAs per SM, clusters up to 16) the fused kernel runs (and the
    three-kernel path does not) where it applies; the Poisson solve, the
    projection and one RK3 step agree with the oracle."""
    from distributednavierstokes_b200 import _lib

    monkeypatch.setenv("DNSB_ZYZ", mode)
    so, sd = both(oracle_mod, D, **ZYZ[cfg])
    lib = _lib.load()
    lib.dnsb_profile(sd.ctx, 1)
    u = rand_fields(so)
    ud = to_dev(D, u)
    r = so.divergence(u)
    p = so.scalarfield()
    so.poisson(r, p)
    sd.poisson["r"].copy_(T(r))
    pdv = D.scalarfield(sd)
    D.poisson(pdv, sd)
    assert rel(N(pdv), p) <= 1e-12
    psi, psid = so.scalarfield(), D.scalarfield(sd)
    so.project(u, psi)
    D.project(ud, psid, sd)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= 1e-12, c
    # 256 tanh(1.5) rows: 1/dy near the walls lifts the oracle's own maxdiv
    # to 4.5e-12, so the bound is relative to it
    assert D.maxdiv(ud, sd) <= max(1e-12, 2 * so.maxdiv(u))
    counts = {}
    for k, name in enumerate(_lib.KINDS):
        t, n = ctypes.c_double(), ctypes.c_long()
        lib.dnsb_profile_read(sd.ctx, k, ctypes.byref(t), ctypes.byref(n))
        counts[name] = n.value
    lib.dnsb_profile(sd.ctx, 0)
    assert counts["fft_z_y_solve"] == 2 and counts["fft_z"] == 0 and counts["y_solve"] == 0
    p, pd = psi, psid
    q, qd = so.vectorfield(), D.vectorfield(sd)
    delta = so.scalarfield() if so.imexy else p
    deltad = D.scalarfield(sd) if sd.imexy else pd
    dt = 0.5 * so.cfl_timestep(u, 0.5)
    so.step(u, p, q, delta, dt)
    D.step(ud, pd, qd, deltad, sd, dt)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= TOL_STEP, c


@pytest.mark.parametrize("cfg", list(PRODUCTION))
def test_one_step_production_lengths(oracle_mod, D, cfg):
    """One semi-implicit RK3 step at the benchmark's line lengths: <= 1e-12."""
    so, sd = both(oracle_mod, D, **PRODUCTION[cfg])
    u = rand_fields(so)
    p = so.scalarfield()
    so.project(u, p)
    ud, pd = to_dev(D, u), T(p)
    q, qd = so.vectorfield(), D.vectorfield(sd)
    delta, deltad = so.scalarfield(), D.scalarfield(sd)
    dt = 0.5 * so.cfl_timestep(u, 0.5)
    u0, p0 = {c: u[c].copy() for c in "xyz"}, p.copy()
    so.step(u, p, q, delta, dt)
    D.step(ud, pd, qd, deltad, sd, dt)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= TOL_STEP, c
        assert rel(N(qd[c]), q[c]) <= 1e-11, c
    check_pressure(rel(N(pd), p), so, u0, p0, dt)
    assert D.maxdiv(ud, sd) < 1e-12


@pytest.mark.parametrize("planes,pipe", [("5", "0"), ("40", "0"), ("5", "1"), ("7", "1"),
                                         ("32", "1"), ("5", "2"), ("7", "2"), ("32", "2"),
                                         ("5", "3"), ("7", "3"), ("32", "3")])
@pytest.mark.parametrize("cfg", ["channel_implicit", "nx384_nz384", "nx64_ny40"])
def test_fused_projection_momentum_planes(oracle_mod, D, cfg, planes, pipe, monkeypatch):
    """The fused projection + momentum kernel with other z-planes per CTA
    (DNSB_GMZ; 5, 7 and 40 leave a shorter last column, 7 a single-plane one
    at nz = 8), its one-barrier pipelined variant (DNSB_GMPIPE=1), the
    variant that stages two planes ahead (DNSB_GMPIPE=2) and the one staged
    by TMA boxes (DNSB_GMPIPE=3; the 16-wide channel falls back to 1): one
    semi-implicit step agrees with the oracle."""
    monkeypatch.setenv("DNSB_GMZ", planes)
    monkeypatch.setenv("DNSB_GMPIPE", pipe)
    kw = GRID_CASES.get(cfg) or PRODUCTION[cfg]
    so, sd = both(oracle_mod, D, **kw)
    u = rand_fields(so)
    p = so.scalarfield()
    so.project(u, p)
    ud, pd = to_dev(D, u), T(p)
    q, qd = so.vectorfield(), D.vectorfield(sd)
    delta, deltad = so.scalarfield(), D.scalarfield(sd)
    dt = 0.5 * so.cfl_timestep(u, 0.5)
    u0, p0 = {c: u[c].copy() for c in "xyz"}, p.copy()
    so.step(u, p, q, delta, dt)
    D.step(ud, pd, qd, deltad, sd, dt)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= TOL_STEP, c
        assert rel(N(qd[c]), q[c]) <= 1e-11, c
    check_pressure(rel(N(pd), p), so, u0, p0, dt)


@pytest.mark.parametrize("planes", ["1", "3"])
@pytest.mark.parametrize("cfg", ["channel", "channel_implicit", "nx64_ny40"])
def test_momentum_march_planes(oracle_mod, D, cfg, planes, monkeypatch):
    """The z-marching momentum with 1 and 3 planes per CTA (DNSB_MOMZ: a
    one-plane column, and columns of 3 that leave a shorter last one at
    nz = 8): one RK3 step agrees with the oracle (the production grids use
    16 planes, small boxes 2 to 8)."""
    monkeypatch.setenv("DNSB_MOMZ", planes)
    kw = GRID_CASES.get(cfg) or PRODUCTION[cfg]
    so, sd = both(oracle_mod, D, **kw)
    u = rand_fields(so)
    p = so.scalarfield()
    so.project(u, p)
    ud, pd = to_dev(D, u), T(p)
    q, qd = so.vectorfield(), D.vectorfield(sd)
    delta = so.scalarfield() if so.imexy else p
    deltad = D.scalarfield(sd) if sd.imexy else pd
    dt = 0.5 * so.cfl_timestep(u, 0.5)
    so.step(u, p, q, delta, dt)
    D.step(ud, pd, qd, deltad, sd, dt)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= TOL_STEP, c
        assert rel(N(qd[c]), q[c]) <= 1e-11, c


@pytest.mark.parametrize("post,pairs", [("1", "0"), ("0", "0"), ("1", "1")])
@pytest.mark.parametrize("nx", [64, 384])
def test_rfftx_output_pass_in_registers(oracle_mod, D, nx, post, pairs, monkeypatch):
    """The divergence x-FFT with its output pass in registers (the default)
    and with the separate shared-memory pass (DNSB_RXPOST=0), and the
    inverse x-FFT with its pair pre-processing inside the first FFT pass
    (DNSB_IXPAIRS=1), at the splits 8 x 4 and 16 x 12; nz = 12 leaves a
    short last group of lines: Poisson solve, projection and one step agree
    with the oracle."""
    monkeypatch.setenv("DNSB_RXPOST", post)
    monkeypatch.setenv("DNSB_IXPAIRS", pairs)
    kw = dict(n=(nx, 8, 12), lims=((0, 4 * math.pi), (-1, 1), (0, 4 * math.pi / 3)),
              bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5),
              visc=1 / 395, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit")
    so, sd = both(oracle_mod, D, **kw)
    u = rand_fields(so)
    ud = to_dev(D, u)
    psi, psid = so.scalarfield(), D.scalarfield(sd)
    so.project(u, psi)
    D.project(ud, psid, sd)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= 1e-12, c
    assert rel(N(psid), psi) <= 1e-12
    assert D.maxdiv(ud, sd) < 1e-12
    p, pd = psi, psid
    q, qd = so.vectorfield(), D.vectorfield(sd)
    delta, deltad = so.scalarfield(), D.scalarfield(sd)
    dt = 0.5 * so.cfl_timestep(u, 0.5)
    so.step(u, p, q, delta, dt)
    D.step(ud, pd, qd, deltad, sd, dt)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= TOL_STEP, c


def T_offset(a):
    """Device copy of a whose data starts 8 bytes past a 16-byte boundary."""
    a = np.ascontiguousarray(a)
    buf = torch.zeros(a.size + 1, dtype=torch.float64, device="cuda")
    t = buf[1:].view(a.shape)
    t.copy_(torch.from_numpy(a))
    assert t.data_ptr() % 16 == 8
    return t


@pytest.mark.parametrize("cfg", ["periodic", "channel", "channel_implicit"])
def test_one_step_unaligned_fields(oracle_mod, D, cfg):
    """Velocity fields that are not 16-byte aligned take the per-cell momentum
    kernel (the z-marching one copies 16-byte chunks): one RK3 step <= 1e-12."""
    so, sd = both(oracle_mod, D, **GRID_CASES[cfg])
    u = rand_fields(so)
    p = so.scalarfield()
    so.project(u, p)
    ud = D.VectorField(x=T_offset(u["x"]), y=T_offset(u["y"]), z=T_offset(u["z"]))
    pd = T(p)
    q, qd = so.vectorfield(), D.vectorfield(sd)
    delta = so.scalarfield() if so.imexy else p
    deltad = D.scalarfield(sd) if sd.imexy else pd
    dt = 0.5 * so.cfl_timestep(u, 0.5)
    u0, p0 = {c: u[c].copy() for c in "xyz"}, p.copy()
    so.step(u, p, q, delta, dt)
    D.step(ud, pd, qd, deltad, sd, dt)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= TOL_STEP, c
        assert rel(N(qd[c]), q[c]) <= 1e-11, c
    check_pressure(rel(N(pd), p), so, u0, p0, dt)


def _c1_ic(O, D, n, ydiff="explicit", amp=0.1, visc=1 / 180):
    kw = dict(n=n, lims=((0, 4 * math.pi), (-1, 1), (0, 4 * math.pi / 3)),
              bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5), visc=visc,
              bodyforce=(1.0, 0.0, 0.0), ydiffusion=ydiff)
    so, sd = both(O, D, **kw)
    u = so.vectorfield()
    so.velocityfield(u, x=lambda x, y, z: 1.5 * (1 - y ** 2))
    ud = D.vectorfield(sd)
    D.velocityfield(ud, sd, x=lambda x, y, z: 1.5 * (1 - y ** 2))
    for c in "xyz":
        so.noise(u[c], c, 0, amp)
        D.noise(ud[c], c, sd, 0, amp)
    so.exchange_halo(u)
    D.exchange_halo(ud, sd)
    for c in "xyz":
        assert np.array_equal(N(ud[c]), u[c])  # same initial condition, bit for bit
    return so, sd, u, ud


@pytest.mark.parametrize("ydiff", ["explicit", "implicit"])
def test_channel_64_one_step_and_100_steps(oracle_mod, D, ydiff):
    """The 64^3 channel case: one RK3 step <= 1e-12, 100 CFL steps <= 1e-9."""
    so, sd, u, ud = _c1_ic(oracle_mod, D, (64, 64, 64), ydiff)
    po, _, _ = so.solve(u, (0.0, 100.0), cfl=0.5, max_steps=1)
    D.solve(u=ud, setup=sd, tlims=(0.0, 100.0), cfl=0.5, max_steps=1)
    for c in "xyz":
        assert rel(N(ud[c]), u[c]) <= TOL_STEP, c
    so2, sd2, u2, ud2 = _c1_ic(oracle_mod, D, (64, 64, 64), ydiff)
    so2.solve(u2, (0.0, 100.0), cfl=0.5, max_steps=100)
    D.solve(u=ud2, setup=sd2, tlims=(0.0, 100.0), cfl=0.5, max_steps=100)
    for c in "xyz":
        assert rel(N(ud2[c]), u2[c]) <= 1e-9, c
    assert D.maxdiv(ud2, sd2) < 1e-12


# --------------------------------------------------- golden fixtures (oracle)

@pytest.mark.parametrize("name", ["runcase_periodic_explicit", "runcase_wall_explicit",
                                  "runcase_wall_implicit", "channel_noise_cfl"])
def test_golden(D, name):
    import golden_cases as G

    spec = G.SPECS[name]
    ref = np.load(os.path.join(GOLDEN, name + ".npz"))
    s = D.setup(**spec["setup"])
    u = D.vectorfield(s)
    if spec["ic"] == "runcase":
        D.velocityfield(u, s, **R.RUNCASE_IC)
    else:
        D.velocityfield(u, s, x=lambda x, y, z: 1.5 * (1 - y ** 2))
        for c in "xyz":
            D.noise(u[c], c, s, 0, 0.1)
        D.exchange_halo(u, s)
    procs = {}
    acc = None
    if spec.get("stats") == "channel":
        acc = D.channelstats(s, nupdate=spec["nupdate"])
        procs["stats"] = acc["sample"]
    elif spec.get("stats") == "spectrum":
        acc = D.spectrumstats(s, nupdate=spec["nupdate"])
        procs["stats"] = acc["sample"]
    D.solve(u=u, setup=s, tlims=spec["tlims"], dt=spec["dt"], cfl=spec["cfl"] or 0.5,
            processors=procs, max_steps=spec.get("max_steps"))
    for k, c in (("ux", "x"), ("uy", "y"), ("uz", "z")):
        assert rel(N(u[c]), ref[k]) <= 1e-11, (name, k)
    if spec.get("stats") == "channel":
        prof = D.channelprofiles(acc, s)
        for k in ("U", "V", "W", "uu", "vv", "ww", "uv"):
            assert np.max(np.abs(prof[k] - ref["prof_" + k])) <= 1e-11, k
    elif spec.get("stats") == "spectrum":
        E = D.energyspectrum(acc, s)["E"]
        assert np.max(np.abs(E - ref["E"])) <= 1e-11 * max(1.0, ref["E"].max())


# ----------------------------------------- the reference's identity tests

@pytest.mark.parametrize("case", ["periodic", "channel"])
def test_projection_and_skew_symmetry(oracle_mod, D, case):
    """test/serialtests.jl:43-58 on the GPU."""
    kw = dict(n=(16, 12, 8), visc=0.0) if case == "periodic" else R.channel_kwargs(visc=0.0)
    so, s = both(oracle_mod, D, **kw)
    u = to_dev(D, rand_fields(so))
    p = D.scalarfield(s)
    D.project(u, p, s)
    assert D.maxdiv(u, s) < 1e-12
    q = D.vectorfield(s)
    D.momentum(q, u, 0.0, 1.0, s)
    d, n2 = R.weighted_dot({c: N(u[c]) for c in "xyz"}, {c: N(q[c]) for c in "xyz"}, s)
    assert abs(d) < 1e-12 * n2


def test_inviscid_energy_conservation(oracle_mod, D):
    """test/serialtests.jl:61-72 on the GPU."""
    so, s = both(oracle_mod, D, n=(16, 16, 16), visc=0.0)
    u = to_dev(D, rand_fields(so))
    p = D.scalarfield(s)
    D.project(u, p, s)
    e0 = D.kinetic_energy(u, s)
    D.solve(u=u, setup=s, tlims=(0.0, 0.1), dt=0.002)
    e1 = D.kinetic_energy(u, s)
    assert abs(e1 - e0) / e0 < 1e-7
    assert D.maxdiv(u, s) < 1e-12


def test_taylor_green_order(D):
    """test/serialtests.jl:74-101 on the GPU."""
    nu, tend = 0.01, 0.5
    err = []
    for n in (16, 32):
        s = D.setup(n=(n, n, 4), visc=nu)
        u = D.vectorfield(s)
        D.velocityfield(u, s, **R.TG_IC)
        D.solve(u=u, setup=s, tlims=(0.0, tend), dt=1e-3)
        decay = math.exp(-2 * nu * tend)
        ex = np.sin(s.xf)[None, None, :] * np.cos(s.yc)[None, :, None] * decay
        err.append(np.max(np.abs(N(u["x"])[s.active("x")] - ex)))
    assert err[1] < 1e-3
    assert 3 < err[0] / err[1] < 5


def test_energy_spectrum(oracle_mod, D):
    """test/serialtests.jl:103-125 on the GPU."""
    so, s = both(oracle_mod, D, n=(16, 16, 16), visc=0.0)
    u = to_dev(D, rand_fields(so))
    p = D.scalarfield(s)
    D.project(u, p, s)
    sp = D.spectrumstats(s)
    sp["sample"](D.State(u, p, 0.0, 0), s)
    E = D.energyspectrum(sp, s)["E"]
    V = (2 * math.pi) ** 3
    assert math.isclose(E.sum(), D.kinetic_energy(u, s) / V, rel_tol=1e-12)
    utg = D.vectorfield(s)
    D.velocityfield(utg, s, **R.TG_IC)
    sptg = D.spectrumstats(s)
    sptg["sample"](D.State(utg, p, 0.0, 0), s)
    Etg = D.energyspectrum(sptg, s)["E"]
    assert math.isclose(Etg[1] / Etg.sum(), 1.0, rel_tol=1e-12)


def test_channel_statistics_laminar(D):
    """test/serialtests.jl:127-139 on the GPU."""
    s = D.setup(**R.channel_kwargs())
    u = D.vectorfield(s)
    D.velocityfield(u, s, x=lambda x, y, z: 1 - y ** 2)
    cs = D.channelstats(s)
    cs["sample"](D.State(u, None, 0.0, 0), s)
    prof = D.channelprofiles(cs, s)
    assert np.max(np.abs(prof["U"] - (1 - prof["y"] ** 2))) <= 1e-13
    assert np.max(np.abs(prof["uu"])) < 1e-13
    assert np.max(np.abs(prof["uv"])) < 1e-13
    assert len(prof["U"]) == s.n[1]
    assert len(prof["uv"]) == s.n[1] - 1


def _runwith(D, yd, dt):
    s = D.setup(**R.channel_kwargs(visc=0.05, bodyforce=(1.0, 0.0, 0.0), ydiffusion=yd))
    u = D.vectorfield(s)
    D.velocityfield(u, s, x=lambda x, y, z: (1 - y ** 2) * (1 + 0.1 * np.sin(2 * x) * np.cos(z)))
    D.solve(u=u, setup=s, tlims=(0.0, 0.2), dt=dt)
    return u, s


def test_implicit_ydiffusion(D):
    """test/serialtests.jl:141-173 on the GPU."""
    d = []
    for dt in (0.004, 0.002):
        ue, _ = _runwith(D, "explicit", dt)
        ui, si = _runwith(D, "implicit", dt)
        assert D.maxdiv(ui, si) < 1e-12
        d.append(max(float(torch.max(torch.abs(ue[c] - ui[c]))) for c in "xyz"))
    assert d[0] < 1e-6
    assert 3 < d[0] / d[1] < 5
    s = D.setup(**R.channel_kwargs(n=(8, 48, 8), stretch=R.tanhstretch(2.5), visc=0.2,
                                   bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"))
    u = D.vectorfield(s)
    D.velocityfield(u, s, x=lambda x, y, z: (1 - y ** 2) * (1 + 0.1 * np.sin(2 * x)))
    D.solve(u=u, setup=s, tlims=(0.0, 1.0), dt=5e-3)
    assert all(bool(torch.isfinite(u[c]).all()) for c in "xyz")
    assert D.kinetic_energy(u, s) < 100
    assert D.maxdiv(u, s) < 1e-12


def test_channel_flow_sanity(D):
    """test/serialtests.jl:176-189 on the GPU."""
    s = D.setup(**R.channel_kwargs(visc=0.05, bodyforce=(1.0, 0.0, 0.0)))
    u = D.vectorfield(s)
    st = D.solve(u=u, setup=s, tlims=(0.0, 1.0))
    assert math.isclose(st.t, 1.0)
    assert D.maxdiv(u, s) < 1e-12
    assert 0 < D.kinetic_energy(u, s) < 100
    prof = N(u["x"])[s.active("x")].sum(axis=(0, 2))
    assert np.all(prof > 0)
    assert np.allclose(prof, prof[::-1], rtol=1e-8, atol=0)


# ------------------------------------------------------------ reductions

@pytest.mark.parametrize("cfg", ["periodic", "channel", "channel_implicit"])
def test_reductions(oracle_mod, D, cfg):
    so, sd = both(oracle_mod, D, **GRID_CASES[cfg])
    u = rand_fields(so)
    ud = to_dev(D, u)
    assert D.cfl_timestep(ud, sd, 0.7) == so.cfl_timestep(u, 0.7)
    assert math.isclose(D.maxdiv(ud, sd), so.maxdiv(u), rel_tol=1e-13)
    assert math.isclose(D.kinetic_energy(ud, sd), so.kinetic_energy(u), rel_tol=1e-13)


def test_solve_host_matches_device(oracle_mod, D):
    """dnsb_solve_host (host buffers through the C ABI) == device solve."""
    import ctypes
    from distributednavierstokes_b200 import _lib

    so, sd, u, ud = _c1_ic(oracle_mod, D, (32, 24, 16))
    hu = {c: np.ascontiguousarray(u[c].copy()) for c in "xyz"}
    hp = np.zeros_like(hu["x"])
    t_out, n_out = ctypes.c_double(), ctypes.c_long()
    lib = _lib.load()
    rc = lib.dnsb_solve_host(sd.ctx, *(h.ctypes.data_as(ctypes.c_void_p) for h in
                                        (hu["x"], hu["y"], hu["z"], hp)),
                             0.0, 10.0, 0.0, 0.5, 5, ctypes.byref(t_out), ctypes.byref(n_out))
    assert rc == 0
    assert n_out.value == 5
    D.solve(u=ud, setup=sd, tlims=(0.0, 10.0), cfl=0.5, max_steps=5)
    for c in "xyz":
        assert rel(hu[c], N(ud[c])) <= 1e-13


# ----------------------------------------------------------- error paths

def test_errors(D):
    from distributednavierstokes_b200._lib import DNSBError

    with pytest.raises(ValueError):
        D.setup(n=(8, 8, 8), bc=("wall", "periodic", "periodic"))
    with pytest.raises(ValueError):
        D.setup(n=(8, 8, 8), ydiffusion="implicit")
    with pytest.raises(DNSBError):
        D.setup(n=(8, 8, 14))  # FFT length with a factor 7
    with pytest.raises(DNSBError):
        D.setup(n=(7, 8, 8))   # odd nx
    s = D.setup(n=(8, 8, 8))
    u = D.vectorfield(s)
    with pytest.raises(DNSBError):
        D.step(u, D.scalarfield(s), D.vectorfield(s), None, s, -1.0)
