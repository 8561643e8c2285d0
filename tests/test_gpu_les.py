"""GPU parity of the filtered-field sampler: dnsb_les_cube (cell-centred
velocity, its six products, 3-D transforms and the LES-cube extraction on
the GPU) against the oracle's numpy restatement, the whole sfs_sample
bank against the oracle's loop restatement of src/spectral/les.jl, and the
snapshot IO round trip on device fields.

Tolerances (FP64): cubes and sampler outputs within 1e-12 relative;
snapshots bit-exact.
"""
import math
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


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


def dev(u):
    import distributednavierstokes_b200 as dns

    return dns.VectorField(**{c: torch.from_numpy(u[c].copy()).cuda() for c in "xyz"})


@pytest.mark.parametrize("n,M", [((16, 16, 16), 8), ((16, 16, 16), 16), ((16, 12, 20), 8)])
def test_les_cube_matches_oracle(oracle_mod, D, n, M):
    import les_oracle as LO

    so, s = oracle_mod.Setup(n), D.setup(n=n)
    rng = np.random.default_rng(9)
    u = so.vectorfield()
    for c in "xyz":
        u[c][1:-1, 1:-1, 1:-1] = rng.standard_normal(u[c][1:-1, 1:-1, 1:-1].shape)
    so.exchange_halo(u)
    ref = LO.cube(so, u, M)
    got = D.les_cube(dev(u), s, M)
    assert got.shape == ref.shape
    for f in range(9):
        assert rel(got[f], ref[f]) < 1e-12, f


def test_sfs_sample_matches_oracle(oracle_mod, D):
    import les_oracle as LO

    n = (24, 24, 24)
    so, s = oracle_mod.Setup(n, visc=5e-3), D.setup(n=n, visc=5e-3)
    u = D.random_field(D.vectorfield(s), s, totalenergy=0.4, kpeak=3, seed=5)
    uo = so.random_field(so.vectorfield(), totalenergy=0.4, kpeak=3, seed=5)
    cells = [dict(M=12, kernel="gaussian", dfac=2.0), dict(M=8, kernel="tophat", dfac=1.5)]
    sam = D.lessampler(s, cells=cells)
    got = D.sfs_sample(sam, u, s)
    ref = LO.sfs(sam["cells"], 12, 2, 2 * math.pi, 5e-3, LO.cube(so, uo, 12))
    for g, r in zip(got, ref):
        for i, k in enumerate("xyz"):
            assert rel(g["ubar"][k], r["ubar"][i]) < 1e-11
        for i, name in enumerate(("xx", "yy", "zz", "xy", "yz", "zx")):
            assert rel(g["tau"][name], r["tau"][i]) < 1e-11
        assert math.isclose(g["redelta"], r["redelta"], rel_tol=1e-11)
        assert rel(g["spectrum"], r["spectrum"]) < 1e-11


def test_snapshot_roundtrip_device(D, tmp_path):
    s = D.setup(n=(16, 16, 16))
    u = D.random_field(D.vectorfield(s), s, totalenergy=1.0, seed=3)
    p = torch.randn(s.shape, dtype=torch.float64, device="cuda")
    prefix = os.path.join(tmp_path, "state")
    D.save_snapshot(prefix, u, s, p=p, time=0.25, step=12, meta=dict(eref=[0.5]))
    u2, p2 = D.vectorfield(s), D.scalarfield(s)
    md = D.load_snapshot(u2, prefix, s, p=p2)
    assert md == dict(time=0.25, step=12, meta=dict(eref=[0.5]))
    for c in "xyz":
        assert torch.equal(u2[c], u[c])
    assert torch.equal(p2, p)
