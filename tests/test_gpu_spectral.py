"""GPU parity of the pseudo-spectral solver (dnsb_spectral_*,
distributednavierstokes_b200/spectral.py) against the numpy oracle
(oracle/spectral_oracle.py): transforms, right-hand side, projection, one
and five IF-RK3 steps, diagnostics, and the exact viscous decay of a shear
wave.  Tolerances (FP64): 1e-12 relative for transforms, right-hand side
and steps; diagnostics 1e-12.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def SP():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from distributednavierstokes_b200 import _lib, spectral

    _lib.load()
    return spectral


def rel(a, b):
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n,kcut", [(12, None), (16, None), (24, 7), (32, None)])
def test_transforms_rhs_project(SP, n, kcut):
    import spectral_oracle as SO

    O = SO.Spectral(n, visc=2e-3, kcut=kcut)
    s = SP.spectral_setup(n=n, visc=2e-3, kcut=kcut)
    uh = O.random(n, amp=0.7)
    v = O.to_phys(uh)
    vd = SP.spec_to_phys(SP.physvelocity(s), dev(uh), s)
    assert rel(vd.cpu().numpy(), v) < 1e-12
    back = SP.phys_to_spec(SP.specvelocity(s), dev(v), s)
    assert rel(back.cpu().numpy(), O.from_phys(v)) < 1e-12
    du, _ = O.rhs(uh)
    dud = SP.spectral_rhs(SP.specvelocity(s), dev(uh), s)
    assert rel(dud.cpu().numpy(), du) < 1e-12
    raw = O.from_phys(np.random.default_rng(1).standard_normal((3, n, n, n)))
    pd = SP.spectral_project(dev(raw), s)
    assert rel(pd.cpu().numpy(), O.project(raw)) < 1e-13
    for f, g in ((SP.spectral_energy, O.energy), (SP.spectral_dissipation, O.dissipation)):
        assert math.isclose(f(dev(uh), s), g(uh), rel_tol=1e-12)
    assert SP.spectral_maxdiv(dev(uh), s) < 1e-12 * float(np.max(np.abs(uh))) * n
    s.close()


@pytest.mark.parametrize("n", [16, 24])
def test_steps_match_oracle(SP, n):
    import spectral_oracle as SO

    O = SO.Spectral(n, visc=5e-3)
    s = SP.spectral_setup(n=n, visc=5e-3)
    uh = O.random(7, amp=1.0)
    ud = dev(uh)
    for k in range(5):
        uh, vmax = O.step(uh, 0.01)
        vd = SP.spectral_step(ud, s, 0.01)
        assert math.isclose(vd, vmax, rel_tol=1e-12)
        assert rel(ud.cpu().numpy(), uh) < 1e-12 * (k + 1)
    assert SP.spectral_maxdiv(ud, s) < 1e-12
    s.close()


def test_shear_wave_exact_decay_and_solve(SP):
    s = SP.spectral_setup(n=16, visc=0.05)
    uh = SP.specvelocity(s)
    SP.spectral_velocityfield(uh, s, x=lambda x, y, z: 0.7 * math.sin(2 * y), y=None, z=None)
    e0 = SP.spectral_energy(uh, s)
    st = SP.spectral_solve(uh=uh, setup=s, tlims=(0.0, 0.3), dt=0.03)
    assert st.n == 10
    assert abs(SP.spectral_energy(uh, s) / e0 - math.exp(-8 * 0.05 * 0.3)) < 1e-13
    # CFL-adaptive solve of a Taylor-Green vortex: stays solenoidal, energy decays
    tg = SP.taylorgreen(SP.specvelocity(s), s)
    e1 = SP.spectral_energy(tg, s)
    st = SP.spectral_solve(uh=tg, setup=s, tlims=(0.0, 0.2), cfl=0.5)
    assert st.n > 1 and SP.spectral_energy(tg, s) < e1
    assert SP.spectral_maxdiv(tg, s) < 1e-12
    s.close()


def test_bad_setups(SP):
    from distributednavierstokes_b200._lib import DNSBError

    with pytest.raises(ValueError):
        SP.spectral_setup(n=15)
    with pytest.raises(ValueError):
        SP.spectral_setup(n=16, kcut=6)
    with pytest.raises(DNSBError):
        SP.spectral_setup(n=14)  # FFT length with a factor 7


def test_random_field_and_forcing_match_oracle(SP):
    """spectral_randomfield! and shellforcing on the GPU against the oracle,
    with the reference's own checks (test/spectralmpitests.jl:128-161:
    n = 18, totalenergy 0.4, kpeak 2, seed 7)."""
    import spectral_oracle as SO

    O = SO.Spectral(18, visc=5e-3)
    s = SP.spectral_setup(n=18, visc=5e-3)
    assert SP.shell_count(s) == int(math.floor(math.sqrt(3) * s.kcut)) + 1
    uo = O.randomfield(totalenergy=0.4, kpeak=2, seed=7)
    uh = SP.spectral_randomfield(SP.specvelocity(s), s, totalenergy=0.4, kpeak=2, seed=7)
    assert rel(uh.cpu().numpy(), uo) < 1e-12
    again = SP.spectral_randomfield(SP.specvelocity(s), s, totalenergy=0.4, kpeak=2, seed=7)
    assert torch.equal(again, uh)
    assert abs(SP.spectral_energy(uh, s) - 0.4) < 1e-13
    assert SP.spectral_maxdiv(uh, s) < 1e-13
    nb = SP.shell_count(s)
    k = np.arange(nb)
    prof = k ** 4 * np.exp(-2 * (k / 2) ** 2)
    E = SP.shell_energies(uh, s, range(nb))
    assert np.max(np.abs(E[:s.kcut + 1] - (0.4 * prof / prof.sum())[:s.kcut + 1])) < 1e-13
    fo = O.shellforcing(uo, shells=(1, 2))
    f = SP.shellforcing(uh, s, shells=(1, 2))
    assert np.allclose(f.eref, fo.eref, rtol=1e-12, atol=0)
    for _ in range(4):
        uo, _ = O.step(uo, 0.02)
        uo = fo(uo)
    st = SP.spectral_solve(uh=uh, setup=s, tlims=(0.0, 0.08), dt=0.02, forcing=f)
    assert st.n == 4
    assert rel(uh.cpu().numpy(), uo) < 1e-11
    assert np.allclose(SP.shell_energies(uh, s, (1, 2)), f.eref, rtol=1e-13, atol=0)
    s.close()


def test_spectral_sfs_sample_matches_oracle(SP):
    """sfs_sample! on the spectral state: the GPU cube against the oracle's,
    then the bank through the host half against the loop restatement."""
    import les_oracle as LO
    import spectral_oracle as SO

    O = SO.Spectral(24, visc=5e-3)
    s = SP.spectral_setup(n=24, visc=5e-3)
    uo = O.randomfield(totalenergy=0.4, kpeak=3, seed=5)
    uh = SP.spectral_randomfield(SP.specvelocity(s), s, totalenergy=0.4, kpeak=3, seed=5)
    cube = SP.les_cube(uh, s, 12)
    ref = O.les_cube(uo, 12)
    for f in range(9):
        assert rel(cube[f], ref[f]) < 1e-12, f
    cells = [dict(M=12, kernel="gaussian", dfac=2.0), dict(M=8, kernel="helmholtz", dfac=1.5)]
    sam = SP.lessampler(s, cells=cells)
    got = SP.sfs_sample(sam, uh, s)
    want = LO.sfs(sam["cells"], 12, 2, s.l, 5e-3, ref)
    for g, r in zip(got, want):
        for i, k in enumerate("xyz"):
            assert rel(g["ubar"][k], r["ubar"][i]) < 1e-11
        for i, name in enumerate(("xx", "yy", "zz", "xy", "yz", "zx")):
            assert rel(g["tau"][name], r["tau"][i]) < 1e-11
        assert math.isclose(g["redelta"], r["redelta"], rel_tol=1e-11)
    with pytest.raises(ValueError):
        SP.lessampler(s, nles=20, filters=[2.0])  # M/2 > kcut
    s.close()


def test_spectral_stats_and_spectrum(SP, tmp_path):
    import spectral_oracle as SO

    O = SO.Spectral(18, visc=5e-3)
    s = SP.spectral_setup(n=18, visc=5e-3)
    uh = SP.spectral_randomfield(SP.specvelocity(s), s, totalenergy=0.4, kpeak=2, seed=7)
    uo = O.randomfield(totalenergy=0.4, kpeak=2, seed=7)
    st = SP.spectral_stats(uh, s)
    e, d = O.energy(uo), O.dissipation(uo)
    assert math.isclose(st["e"], e, rel_tol=1e-12) and math.isclose(st["diss"], d, rel_tol=1e-12)
    assert math.isclose(st["l_kol"], (5e-3 ** 3 / d) ** 0.25, rel_tol=1e-12)
    assert math.isclose(st["kmax_eta"], math.pi * 18 / s.l * st["l_kol"], rel_tol=1e-14)
    sp = SP.spectral_spectrum(uh, s)
    assert np.allclose(sp["E"], O.shell_energies(uo, s.kcut + 1), rtol=1e-12, atol=1e-18)
    f = str(tmp_path / "stats.csv")
    SP.spectral_solve(uh=uh, setup=s, tlims=(0.0, 0.04), dt=0.01,
                      processors={"stats": SP.statswriter(f, nupdate=2)})
    rows = open(f).read().strip().splitlines()
    assert rows[0].startswith("t,step,e,uavg,diss") and len(rows) == 4  # n = 0, 2, 4
    s.close()


def test_phaserandomize_and_offline_bank(SP, tmp_path):
    """spectral_phaserandomize! against the oracle (|u_hat| and the
    divergence kept, the result still a real field), and sfs_offline over
    saved snapshots = sfs_sample of the phase-randomised states."""
    import os

    import spectral_oracle as SO
    from distributednavierstokes_b200 import spectral_io as SIO

    O = SO.Spectral(12, visc=5e-3)
    s = SP.spectral_setup(n=12, visc=5e-3)
    uo = O.randomfield(totalenergy=0.4, kpeak=2, seed=3)
    uh = dev(uo)
    SP.spectral_phaserandomize(uh, s, seed=9)
    ref = O.phaserandomize(uo, seed=9)
    got = uh.cpu().numpy()
    assert rel(got, ref) < 1e-14
    assert np.max(np.abs(np.abs(got) - np.abs(uo))) < 1e-15
    assert SP.spectral_maxdiv(uh, s) < 1e-13
    assert rel(O.from_phys(O.to_phys(got)), got) < 1e-13  # Hermitian-consistent
    pre = [os.path.join(tmp_path, f"raw_{i}") for i in (1, 2)]
    u1 = dev(uo)
    SIO.spectral_save(pre[0], u1, s, time=0.5, step=5)
    SP.spectral_step(u1, s, 0.01)
    SIO.spectral_save(pre[1], u1, s, time=0.51, step=6)
    cells = [dict(M=8, kernel="gaussian", dfac=2.0)]
    SIO.sfs_offline(pre, s, str(tmp_path / "bank"), cells=cells, phaseseed=4)
    f = np.load(tmp_path / "bank" / "delta=2.0" / "fields.npz")
    assert f["inputs"].shape == (2, 3, 8, 8, 5) and f["outputs"].shape == (2, 6, 8, 8, 5)
    m = np.load(tmp_path / "bank" / "dns_meta.npz")
    assert list(m["times"]) == [0.5, 0.51] and m["spectra_dns"].shape == (2, s.kcut)
    u2 = SP.specvelocity(s)
    SIO.spectral_load(u2, pre[1], s)
    SP.spectral_phaserandomize(u2, s, seed=4)
    direct = SP.sfs_sample(SP.lessampler(s, cells=cells), u2, s)[0]
    assert np.array_equal(f["inputs"][1][0], direct["ubar"]["x"])
    assert np.array_equal(f["outputs"][1][5], direct["tau"]["zx"])
    s.close()
