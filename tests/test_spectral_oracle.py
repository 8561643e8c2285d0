"""The pseudo-spectral oracle (oracle/spectral_oracle.py) against known
answers, on CPU: the exact viscous decay of a shear wave (the nonlinear term
vanishes and the integrating factor is exact, as the reference's step.jl
header states), inviscid energy conservation of the truncated Galerkin
system to the RK3 truncation error, solenoidality after a step, and the
transform round trip of a band-limited field.
"""
import math

import numpy as np

import spectral_oracle as SO


def test_shear_wave_decays_exactly():
    S = SO.Spectral(12, visc=0.05)
    uh = S.velocityfield(lambda x, y, z: 0.7 * math.sin(2 * y), None, None)
    e0 = S.energy(uh)
    t = 0.0
    for _ in range(10):
        uh, _ = S.step(uh, 0.03)
        t += 0.03
    # u = 0.7 sin(2y) exp(-4 nu t): energy exp(-8 nu t)
    assert abs(S.energy(uh) / e0 - math.exp(-8 * 0.05 * t)) < 1e-13
    v = S.to_phys(uh)
    c = S.l / S.n * (np.arange(S.n) + 0.5)
    ref = 0.7 * np.sin(2 * c) * math.exp(-4 * 0.05 * t)
    assert np.max(np.abs(v[0] - ref[None, :, None])) < 1e-13
    assert np.max(np.abs(v[1:])) < 1e-14


def test_inviscid_energy_conservation():
    S = SO.Spectral(16, visc=0.0)
    uh = S.random(3, amp=0.5)
    e0 = S.energy(uh)
    for _ in range(5):
        uh, vmax = S.step(uh, 2e-3)
    assert abs(S.energy(uh) - e0) / e0 < 1e-8
    assert S.maxdiv(uh) < 1e-13 * max(1.0, float(np.max(np.abs(uh))))
    assert vmax > 0


def test_transform_round_trip():
    S = SO.Spectral(12)
    uh = S.random(1)
    assert np.max(np.abs(S.from_phys(S.to_phys(uh)) - uh)) < 1e-15


def test_dissipation_matches_energy_decay_rate():
    S = SO.Spectral(16, visc=0.02)
    uh = S.random(5, amp=0.1)
    e0, d0 = S.energy(uh), S.dissipation(uh)
    dt = 1e-4
    uh1, _ = S.step(uh, dt)
    # dE/dt = -nu sum k^2 |u_hat|^2 = -dissipation (the nonlinear transfer
    # conserves E)
    rate = (S.energy(uh1) - e0) / dt
    assert abs(rate + d0) < 1e-3 * d0


def test_random_field_reference_checks():
    """The reference's own checks of spectral_randomfield! and shellforcing
    (test/spectralmpitests.jl:128-161: n = 18, totalenergy 0.4, kpeak 2,
    seed 7): energy 0.4, divergence-free, spectrum = profile over the
    shells 0..kcut to 1e-13, forced shells held through a run."""
    S = SO.Spectral(18, visc=5e-3)
    uh = S.randomfield(totalenergy=0.4, kpeak=2, seed=7)
    assert abs(S.energy(uh) - 0.4) < 1e-14
    assert S.maxdiv(uh) < 1e-14
    kdiag = int(math.floor(math.sqrt(3) * S.kcut))
    k = np.arange(kdiag + 1)
    prof = k ** 4 * np.exp(-2 * (k / 2) ** 2)
    target = 0.4 * prof / prof.sum()
    E = S.shell_energies(uh, kdiag + 1)
    assert np.max(np.abs(E[:S.kcut + 1] - target[:S.kcut + 1])) < 1e-13
    f = S.shellforcing(uh, shells=(1, 2))
    for _ in range(4):
        uh, _ = S.step(uh, 0.02)
        uh = f(uh)
    assert np.allclose(S.shell_energies(uh, 3)[1:], f.eref, rtol=1e-13, atol=0)
