"""GPU parity of the wavenumber-shell entry points (dnsb_random_field,
dnsb_shell_energies, dnsb_shell_rescale, dnsb_shell_clamp) against the
oracle's numpy restatement, plus the reference's own checks of its random
initial condition and shell forcing (test/spectralmpitests.jl:128-161):
energy = totalenergy, divergence-free, spectrum = profile, forced shells
held through a run.

Tolerances (FP64): fields and energies within 1e-12 relative of the oracle;
a forced 5-step run within 1e-11.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

BOXES = [(18, 18, 18), (16, 12, 20), (32, 32, 32)]


@pytest.fixture(scope="module")
def D():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import distributednavierstokes_b200 as dns
    from distributednavierstokes_b200 import _lib

    _lib.load()
    return dns


def host(u):
    return {c: u[c].detach().cpu().numpy() for c in "xyz"}


def rel(a, b):
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


@pytest.mark.parametrize("n", BOXES)
def test_random_field_matches_oracle(oracle_mod, D, n):
    so, s = oracle_mod.Setup(n, visc=5e-3), D.setup(n=n, visc=5e-3)
    assert D.shell_count(s) == so.shell_count()
    uo = so.random_field(so.vectorfield(), totalenergy=0.4, kpeak=2, seed=7)
    u = D.random_field(D.vectorfield(s), s, totalenergy=0.4, kpeak=2, seed=7)
    ud = host(u)
    for c in "xyz":
        assert rel(ud[c], uo[c]) < 1e-12, c
    nb = D.shell_count(s)
    E = D.shell_energies(u, s, range(nb))
    k = np.arange(nb, dtype=np.float64)
    prof = k ** 4 * np.exp(-2 * (k / 2) ** 2)
    assert np.abs(E - 0.4 * prof / prof.sum()).max() < 1e-13
    assert abs(D.kinetic_energy(u, s) / (2 * math.pi) ** 3 - 0.4) < 1e-12
    assert D.maxdiv(u, s) < 1e-13


def test_random_field_custom_profile(oracle_mod, D):
    n = (16, 16, 16)
    prof = lambda k: 1.0 if 3 <= k <= 5 else 0.0  # noqa: E731
    so, s = oracle_mod.Setup(n), D.setup(n=n)
    uo = so.random_field(so.vectorfield(), totalenergy=2.0, seed=1, profile=prof)
    u = D.random_field(D.vectorfield(s), s, totalenergy=2.0, seed=1, profile=prof)
    ud = host(u)
    for c in "xyz":
        assert rel(ud[c], uo[c]) < 1e-12


@pytest.mark.parametrize("n", BOXES[:2])
def test_shell_energies_and_rescale(oracle_mod, D, n):
    so, s = oracle_mod.Setup(n), D.setup(n=n)
    rng = np.random.default_rng(3)
    uo = so.vectorfield()
    for c in "xyz":
        uo[c][1:-1, 1:-1, 1:-1] = rng.standard_normal(uo[c][1:-1, 1:-1, 1:-1].shape)
    so.exchange_halo(uo)
    u = D.VectorField(**{c: torch.from_numpy(uo[c].copy()).cuda() for c in "xyz"})
    nb = so.shell_count()
    Eo = so.shell_energies(uo, nb)
    E = D.shell_energies(u, s, range(nb))
    assert np.max(np.abs(E - Eo)) <= 1e-12 * Eo.max()
    f = 0.5 + rng.random(nb)
    so.rescale_shells(uo, f)
    D.rescale_shell(u, s, 3, f[3])
    for sh in range(nb):
        if sh != 3:
            D.rescale_shell(u, s, sh, f[sh])
    ud = host(u)
    for c in "xyz":
        assert rel(ud[c], uo[c]) < 1e-12
        # ghost images are rewritten too
        assert np.array_equal(ud[c][0], ud[c][-2]) and np.array_equal(ud[c][:, :, -1], ud[c][:, :, 1])


# shells below 4 take the direct partial-sum clamp, (1, 3, 4) the transform one
@pytest.mark.parametrize("shells", [(1, 2), (2, 3), (1, 3, 4)])
def test_forced_run_matches_oracle(oracle_mod, D, shells):
    n = (18, 18, 18)
    so, s = oracle_mod.Setup(n, visc=5e-3), D.setup(n=n, visc=5e-3)
    uo = so.random_field(so.vectorfield(), totalenergy=0.4, kpeak=2, seed=7)
    u = D.random_field(D.vectorfield(s), s, totalenergy=0.4, kpeak=2, seed=7)
    fo = so.shellforcing(uo, shells=shells)
    f = D.shellforcing(u, s, shells=shells)
    assert np.allclose(f.eref, fo.eref, rtol=1e-12, atol=0)
    so.solve(uo, (0.0, 0.05), dt=0.01, forcing=fo)
    st = D.solve(u=u, setup=s, tlims=(0.0, 0.05), dt=0.01, forcing=f)
    assert st.n == 5
    ud = host(u)
    for c in "xyz":
        assert rel(ud[c], uo[c]) < 1e-11
    assert np.allclose(D.shell_energies(u, s, shells), f.eref, rtol=1e-13, atol=0)
    assert D.maxdiv(u, s) < 1e-12
    ud = host(u)
    for c in "xyz":  # ghost images rewritten by the clamp
        assert np.array_equal(ud[c][0], ud[c][-2]) and np.array_equal(ud[c][:, :, -1], ud[c][:, :, 1])


def test_shells_need_periodic_box(D):
    from distributednavierstokes_b200._lib import DNSBError

    s = D.setup(n=(8, 8, 8), bc=("periodic", "wall", "periodic"))
    with pytest.raises(DNSBError):
        D.shell_energies(D.vectorfield(s), s, (1, 2))


def test_random_field_and_clamp_bit_reproducible(D):
    """Shell energies are summed in a fixed order: the same seed gives the
    same field bit for bit, and so does a clamp of the same state."""
    s = D.setup(n=(32, 32, 32))
    a = D.random_field(D.vectorfield(s), s, totalenergy=0.4, kpeak=4, seed=11)
    b = D.random_field(D.vectorfield(s), s, totalenergy=0.4, kpeak=4, seed=11)
    for c in "xyz":
        assert torch.equal(a[c], b[c])
    f = D.shellforcing(a, s, shells=(1, 2))
    for c in "xyz":
        a[c].mul_(1.1)
        b[c].mul_(1.1)
    f(a, s)
    f(b, s)
    for c in "xyz":
        assert torch.equal(a[c], b[c])
