"""Oracle restatement of the random-phase initial condition and the
shell-clamp forcing on a periodic FV box (CPU only).

The reference defines both on its pseudo-spectral state
(src/spectral/ic.jl:37-84, src/spectral/forcing.jl:1-56); its own test
(test/spectralmpitests.jl:128-161) checks, for totalenergy = 0.4, kpeak = 2,
seed = 7: the energy equals totalenergy, the field is divergence-free, the
shell spectrum equals totalenergy * profile / sum(profile), and the forced
shells keep their reference energy through a run.  The same properties are
checked here on the oracle's FV counterpart, plus the published SplitMix64
known answers for the counter hash.
"""
import math

import numpy as np
import pytest

import oracle as O


def test_splitmix64_known_answers():
    # SplitMix64 seeded with 0: the published first outputs; splitmix64(x)
    # of src/spectral/ic.jl:31-36 is one step from state x
    g = np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        states = np.array([0, 1, 2], dtype=np.uint64) * g
    out = O._splitmix64(states)
    assert [int(v) for v in out] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_uniform_hash_matches_c_noise():
    s = O.Setup((12, 10, 8))
    phi = s.scalarfield()
    s.noise(phi, "y", 99, 1.0)
    nx, ny, nz = s.n
    K, J, I = np.meshgrid(*(np.arange(v, dtype=np.uint64) for v in (nz, ny, nx)), indexing="ij")
    key = ((np.uint64(1) * np.uint64(nz) + K) * np.uint64(ny) + J) * np.uint64(nx) + I
    U = ((O._splitmix64(np.uint64(99) + key) >> np.uint64(11)).astype(float) + 0.5) * 2.0 ** -53
    assert np.array_equal(s.interior(phi), 2 * U - 1)


def test_gaussian_noise_statistics():
    s = O.Setup((32, 32, 32))
    phi = s.scalarfield()
    s.gauss_noise(phi, "x", 3)
    v = s.interior(phi).ravel()
    assert abs(v.mean()) < 0.02 and abs(v.std() - 1) < 0.02


@pytest.mark.parametrize("n", [(18, 18, 18), (16, 12, 20)])
def test_random_field_properties(n):
    s = O.Setup(n)
    u = s.vectorfield()
    s.random_field(u, totalenergy=0.4, kpeak=2, seed=7)
    nb = s.shell_count()
    E = s.shell_energies(u, nb)
    k = np.arange(nb, dtype=np.float64)
    prof = k ** 4 * np.exp(-2 * (k / 2) ** 2)
    assert np.abs(E - 0.4 * prof / prof.sum()).max() < 1e-13
    assert abs(E.sum() - 0.4) < 1e-13
    # kinetic_energy integrates over the (2 pi)^3 box
    assert abs(s.kinetic_energy(u) / (2 * math.pi) ** 3 - 0.4) < 1e-12
    assert s.maxdiv(u) < 1e-13


def test_custom_profile_and_mean_removed():
    s = O.Setup((16, 16, 16))
    u = s.vectorfield()
    s.random_field(u, totalenergy=2.0, seed=1, profile=lambda k: 1.0 if 3 <= k <= 5 else 0.0)
    E = s.shell_energies(u, s.shell_count())
    assert np.allclose(E[3:6], 2.0 / 3, rtol=0, atol=1e-13)
    assert np.abs(np.delete(E, [3, 4, 5])).max() < 1e-14
    for c in "xyz":
        assert abs(s.interior(u[c]).mean()) < 1e-14


def test_shellforcing_restores_reference_energy():
    s = O.Setup((16, 16, 16), visc=5e-3)
    u = s.vectorfield()
    s.random_field(u, totalenergy=0.4, kpeak=2, seed=7)
    f = s.shellforcing(u, shells=(1, 2))
    eref = f.eref.copy()
    s.solve(u, (0.0, 0.05), cfl=0.4, forcing=f)
    assert np.allclose(s.shell_energies(u, 3)[1:3], eref, rtol=1e-13, atol=0)
    assert s.maxdiv(u) < 1e-12
