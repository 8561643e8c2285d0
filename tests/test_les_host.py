"""The host half of the filtered-field sampler (distributednavierstokes_b200
/les.py) against the oracle's per-mode loop restatement of
src/spectral/les.jl, on CPU; snapshot IO round trips on host arrays.

The coarse cubes come from the oracle's own FV state (a random solenoidal
field of a periodic 16^3 box), so the whole rank-0 pipeline is checked on
physically shaped input: u_bar, tau (6 components), Re_Delta and the shell
spectrum of every bank cell agree to 1e-12 relative.
"""
import math
import os

import numpy as np
import pytest

import les_oracle as LO
import oracle as O

les = pytest.importorskip("distributednavierstokes_b200.les")


def rel(a, b):
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


@pytest.fixture(scope="module")
def state():
    so = O.Setup((16, 16, 16), visc=5e-3)
    u = so.random_field(so.vectorfield(), totalenergy=0.4, kpeak=3, seed=5)
    return so, u


def test_cube_shape_and_hermitian_mean(state):
    so, u = state
    cb = LO.cube(so, u, 8)
    assert cb.shape == (9, 8, 8, 5)
    # the velocity is mean-free after the random initial condition
    assert np.max(np.abs(cb[:3, 0, 0, 0])) < 1e-15
    # mean of sigma_ii = twice the kinetic energy density of the cell-centred
    # field, which face averaging damps below the staggered field's (0.4)
    ke = so.kinetic_energy(u) / (2 * math.pi) ** 3
    tr = (cb[3, 0, 0, 0] + cb[4, 0, 0, 0] + cb[5, 0, 0, 0]).real
    assert 0.5 * 2 * ke < tr < 2 * ke


@pytest.mark.parametrize("kernel", ["gaussian", "cutoff", "tophat", "helmholtz"])
def test_coarse_kernels_match_loops(state, kernel):
    so, u = state
    cb = LO.cube(so, u, 12)
    n, l, delta = 12, 2 * math.pi, 2.0 * 2 * math.pi / 12
    a = cb[0]
    assert np.array_equal(les.les_twothirds(a.copy(), n), LO.twothirds(a, n))
    assert rel(les.les_filterkernel(a.copy(), n, l, delta, 2, kernel),
               LO.filterkernel(a, n, l, delta, 2, kernel)) < 1e-15
    ub = [LO.twothirds(cb[c], n) for c in range(3)]
    s_prod, s_or = les.les_nonlinearity(ub, n), LO.nonlinearity(ub, n)
    for c in range(6):
        assert rel(s_prod[c], s_or[c]) < 1e-13
    assert math.isclose(les.les_filter_reynolds(ub, n, l, 5e-3, delta),
                        LO.filter_reynolds(ub, n, l, 5e-3, delta), rel_tol=1e-13)
    assert rel(les.les_spectrum(ub, n), LO.spectrum(ub, n)) < 1e-14
    tp = les.les_tracefree([cb[3 + c].copy() for c in range(6)])
    to = LO.tracefree([cb[3 + c] for c in range(6)])
    for c in range(6):
        assert rel(tp[c], to[c]) < 1e-15
    assert np.max(np.abs(tp[0] + tp[1] + tp[2])) < 1e-15


def test_extract_matches_loops(state):
    so, u = state
    cb = LO.cube(so, u, 12)
    assert np.array_equal(les.les_extract(cb[2], 8, 12), LO.extract(cb[2], 8, 12))
    assert np.array_equal(les.les_extract(cb[2], 12, 12), cb[2])
    # extracting the 8-cube from the 12-cube = taking the 8-cube directly
    assert np.array_equal(les.les_extract(cb[4], 8, 12), LO.cube(so, u, 8)[4])


def test_sfs_bank_matches_oracle(state):
    so, u = state
    cells = [dict(M=12, kernel="gaussian", dfac=2.0), dict(M=8, kernel="tophat", dfac=1.5),
             dict(M=12, kernel="helmholtz", dfac=3.0), dict(M=8, kernel="cutoff", dfac=2.0)]
    cb = LO.cube(so, u, 12)
    l = 2 * math.pi
    sam = dict(cells=les.lescells(cells=cells), nles=12, protectshells=2,
               outtype=lambda M: np.float64, l=l)
    got = les.sfs_from_cube(sam, cb, so.visc)
    ref = LO.sfs(sam["cells"], 12, 2, l, so.visc, cb)
    for g, r in zip(got, ref):
        for i, k in enumerate("xyz"):
            assert rel(g["ubar"][k], r["ubar"][i]) < 1e-12
        for i, (name, _, _) in enumerate(les.SIGMA):
            assert rel(g["tau"][name], r["tau"][i]) < 1e-12
        assert math.isclose(g["redelta"], r["redelta"], rel_tol=1e-12)
        assert rel(g["spectrum"], r["spectrum"]) < 1e-12
        # tau is trace-free and dealiased
        tr = g["tau"]["xx"] + g["tau"]["yy"] + g["tau"]["zz"]
        assert np.max(np.abs(tr)) < 1e-15


def test_lescells_and_validation():
    cells = les.lescells(nles=64, filters=[2.0, 4.0])
    assert cells == [dict(M=64, kernel="gaussian", dfac=2.0, deta=None),
                     dict(M=64, kernel="gaussian", dfac=4.0, deta=None)]
    with pytest.raises(ValueError):
        les.lescells(nles=64)

    class Box:
        bc = ("periodic",) * 3
        n = (16, 16, 16)
        lims = ((0.0, 1.0),) * 3

    with pytest.raises(ValueError):
        les.lessampler(Box(), cells=[dict(M=7, kernel="gaussian", dfac=2.0)])
    with pytest.raises(ValueError):
        les.lessampler(Box(), cells=[dict(M=8, kernel="box", dfac=2.0)])
    with pytest.raises(ValueError):
        les.lessampler(Box(), cells=[dict(M=32, kernel="gaussian", dfac=2.0)])
    Box.bc = ("periodic", "wall", "periodic")
    with pytest.raises(ValueError):
        les.lessampler(Box(), nles=8, filters=[2.0])


def test_snapshot_roundtrip_host(tmp_path, state):
    so, u = state

    class S:
        n = so.n
        bc = so.bc
        lims = so.lims
        visc = so.visc
        shape = so.shape

    p = np.arange(np.prod(so.shape), dtype=np.float64).reshape(so.shape)
    prefix = os.path.join(tmp_path, "snap_7")
    les.save_snapshot(prefix, u, S, p=p, time=1.5, step=7, meta=dict(eref=[0.1, 0.2]))
    assert sorted(os.listdir(tmp_path)) == ["snap_7.bin", "snap_7.json"]
    u2 = {c: np.zeros(so.shape) for c in "xyz"}
    p2 = np.zeros(so.shape)
    md = les.load_snapshot(u2, prefix, S, p=p2)
    assert md["time"] == 1.5 and md["step"] == 7 and md["meta"]["eref"] == [0.1, 0.2]
    for c in "xyz":
        assert np.array_equal(u2[c], u[c])
    assert np.array_equal(p2, p)

    class T(S):
        n = (8, 8, 8)

    with pytest.raises(ValueError):
        les.load_snapshot(u2, prefix, T)
