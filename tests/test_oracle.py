"""Pins the CPU oracle (oracle/dns_oracle.c) to the reference.

The reference ships no golden vectors and its Julia toolchain is not
available, so the oracle is pinned by re-running every single-rank
known-answer / identity test of test/serialtests.jl and test/mpitests.jl
against it, with the reference's tolerances, plus its FFTs against
numpy.fft.  The committed golden fixtures (tests/golden/) are then checked
to be what the oracle produces.
"""
import math
import os

import numpy as np
import pytest

import refcases as R

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def mk(O, **kw):
    return O.Setup(**kw)


def rand_u(O, s, seed=42):
    u = s.vectorfield()
    vals = R.random_values(s, seed)
    for c in "xyz":
        u[c][s.active(c)] = vals[c]
    s.exchange_halo(u)
    return u


@pytest.mark.parametrize("n", [4, 6, 8, 10, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 7, 11, 52])
def test_fft_vs_numpy(oracle_mod, n):
    O = oracle_mod
    rng = np.random.default_rng(n)
    x = rng.standard_normal((5, n)) + 1j * rng.standard_normal((5, n))
    ref = np.fft.fft(x)
    assert np.max(np.abs(O.cfft(x) - ref)) <= 1e-14 * np.max(np.abs(ref))
    assert np.max(np.abs(O.cfft(x, True) - np.fft.ifft(x))) <= 1e-14 * np.max(np.abs(x))
    if n % 2 == 0:
        xr = rng.standard_normal((5, n))
        Xr = np.fft.rfft(xr)
        assert np.max(np.abs(O.rfft(xr) - Xr)) <= 1e-14 * np.max(np.abs(Xr))
        assert np.max(np.abs(O.irfft(Xr, n) - xr)) <= 1e-14 * np.max(np.abs(xr))


@pytest.mark.parametrize("case", ["periodic", "channel"])
def test_projection_and_skew_symmetry(oracle_mod, case):
    """test/serialtests.jl:43-58"""
    O = oracle_mod
    if case == "periodic":
        s = O.Setup((16, 12, 8), visc=0.0)
    else:
        s = O.Setup(**R.channel_kwargs(visc=0.0))
    u = rand_u(O, s)
    p = s.scalarfield()
    s.project(u, p)
    assert s.maxdiv(u) < 1e-12
    q = s.vectorfield()
    s.momentum(q, u, 0.0, 1.0)
    d, n2 = R.weighted_dot(u, q, s)
    assert abs(d) < 1e-12 * n2


def test_inviscid_energy_conservation(oracle_mod):
    """test/serialtests.jl:61-72"""
    O = oracle_mod
    s = O.Setup((16, 16, 16), visc=0.0)
    u = rand_u(O, s)
    p = s.scalarfield()
    s.project(u, p)
    e0 = s.kinetic_energy(u)
    s.solve(u, (0.0, 0.1), dt=0.002)
    e1 = s.kinetic_energy(u)
    assert abs(e1 - e0) / e0 < 1e-7
    assert s.maxdiv(u) < 1e-12


def test_taylor_green_order(oracle_mod):
    """test/serialtests.jl:74-101"""
    O = oracle_mod
    nu, tend = 0.01, 0.5
    err = []
    for n in (16, 32):
        s = O.Setup((n, n, 4), visc=nu)
        u = s.vectorfield()
        s.velocityfield(u, **R.TG_IC)
        s.solve(u, (0.0, tend), dt=1e-3)
        decay = math.exp(-2 * nu * tend)
        sl = s.active("x")
        ex = np.sin(s.xf)[None, None, :] * np.cos(s.yc)[None, :, None] * decay
        err.append(np.max(np.abs(u["x"][sl] - ex)))
    assert err[1] < 1e-3
    assert 3 < err[0] / err[1] < 5


def test_energy_spectrum(oracle_mod):
    """test/serialtests.jl:103-125"""
    O = oracle_mod
    s = O.Setup((16, 16, 16), visc=0.0)
    u = rand_u(O, s)
    p = s.scalarfield()
    s.project(u, p)
    sp = s.spectrumstats()
    sp["sample"](u, p, 0.0, 0)
    _, E = s.energyspectrum(sp)
    V = (2 * math.pi) ** 3
    assert math.isclose(E.sum(), s.kinetic_energy(u) / V, rel_tol=1e-12)
    utg = s.vectorfield()
    s.velocityfield(utg, **R.TG_IC)
    sptg = s.spectrumstats()
    sptg["sample"](utg, p, 0.0, 0)
    _, Etg = s.energyspectrum(sptg)
    assert math.isclose(Etg[1] / Etg.sum(), 1.0, rel_tol=1e-12)


def test_channel_statistics_laminar(oracle_mod):
    """test/serialtests.jl:127-139"""
    O = oracle_mod
    s = O.Setup(**R.channel_kwargs())
    u = s.vectorfield()
    s.velocityfield(u, x=lambda x, y, z: 1 - y ** 2)
    cs = s.channelstats()
    cs["sample"](u, None, 0.0, 0)
    prof = s.channelprofiles(cs)
    assert np.max(np.abs(prof["U"] - (1 - prof["y"] ** 2))) <= 1e-13
    assert np.max(np.abs(prof["uu"])) < 1e-13
    assert np.max(np.abs(prof["uv"])) < 1e-13
    assert len(prof["U"]) == s.n[1]
    assert len(prof["uv"]) == s.n[1] - 1


def _runwith(O, yd, dt):
    s = O.Setup(**R.channel_kwargs(visc=0.05, bodyforce=(1.0, 0.0, 0.0), ydiffusion=yd))
    u = s.vectorfield()
    s.velocityfield(u, x=lambda x, y, z: (1 - y ** 2) * (1 + 0.1 * math.sin(2 * x) * math.cos(z)))
    s.solve(u, (0.0, 0.2), dt=dt)
    return u, s


def test_implicit_ydiffusion_second_order(oracle_mod):
    """test/serialtests.jl:141-157"""
    O = oracle_mod
    d = []
    for dt in (0.004, 0.002):
        ue, _ = _runwith(O, "explicit", dt)
        ui, si = _runwith(O, "implicit", dt)
        assert si.maxdiv(ui) < 1e-12
        d.append(max(np.max(np.abs(ue[c] - ui[c])) for c in "xyz"))
    assert d[0] < 1e-6
    assert 3 < d[0] / d[1] < 5


def test_implicit_ydiffusion_stable(oracle_mod):
    """test/serialtests.jl:159-173"""
    O = oracle_mod
    s = O.Setup(**R.channel_kwargs(n=(8, 48, 8), stretch=R.tanhstretch(2.5), visc=0.2,
                                   bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"))
    u = s.vectorfield()
    s.velocityfield(u, x=lambda x, y, z: (1 - y ** 2) * (1 + 0.1 * math.sin(2 * x)))
    s.solve(u, (0.0, 1.0), dt=5e-3)
    assert all(np.all(np.isfinite(u[c])) for c in "xyz")
    assert s.kinetic_energy(u) < 100
    assert s.maxdiv(u) < 1e-12


def test_channel_flow_sanity(oracle_mod):
    """test/serialtests.jl:176-189"""
    O = oracle_mod
    s = O.Setup(**R.channel_kwargs(visc=0.05, bodyforce=(1.0, 0.0, 0.0)))
    u = s.vectorfield()
    _, t, n = s.solve(u, (0.0, 1.0))
    assert math.isclose(t, 1.0)
    assert s.maxdiv(u) < 1e-12
    assert 0 < s.kinetic_energy(u) < 100
    sl = s.active("x")
    prof = u["x"][sl].sum(axis=(0, 2))
    assert np.all(prof > 0)
    assert np.allclose(prof, prof[::-1], rtol=1e-8, atol=0)


@pytest.mark.parametrize("bcy", ["periodic", "wall"])
@pytest.mark.parametrize("stag", ["x", "y", "z", "p"])
def test_halo(oracle_mod, bcy, stag):
    """test/mpitests.jl:108-129 (single rank): exact equality."""
    O = oracle_mod
    s = O.Setup(**R.case_kwargs(bcy))
    phi, exp = R.halo_case(s, stag, bcy == "wall")
    s.fill_halo(phi, stag)
    assert np.array_equal(phi, exp)


@pytest.mark.parametrize("bcy", ["periodic", "wall"])
def test_poisson_recovers_pressure(oracle_mod, bcy):
    """test/mpitests.jl:133-154 (single rank)."""
    O = oracle_mod
    s = O.Setup(**R.case_kwargs(bcy))
    pex = R.poisson_pex(s)
    s.fill_halo(pex, "p")
    u = s.vectorfield()
    s.pressuregrad_update(u, pex)
    s.exchange_halo(u)
    r = s.divergence(u)
    p2 = s.scalarfield()
    s.poisson(r, p2)
    d = s.interior(p2) + s.interior(pex)
    dev = np.max(np.abs(d - d.mean()))
    assert dev < 1e-8


def test_golden_fixtures_match_oracle(oracle_mod):
    """The committed fixtures are what the oracle computes (regenerate with
    tests/golden/make_golden.py)."""
    import golden_cases as G

    for name, fn in G.CASES.items():
        path = os.path.join(GOLDEN, name + ".npz")
        assert os.path.exists(path), path
        ref = np.load(path)
        out = fn(oracle_mod)
        for k in ref.files:
            a, b = ref[k], out[k]
            scale = max(1.0, float(np.max(np.abs(a))))
            assert np.max(np.abs(a - b)) <= 1e-13 * scale, (name, k)
