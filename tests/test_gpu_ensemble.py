"""The batched ensemble (dnsb_ensemble_*, api.Ensemble): members of uneven
sizes and viscosities advanced through one CUDA graph must equal, bit for
bit, each member stepped alone with dnsb_step (a batched periodic-box
ensemble; the reference has no ensemble path)."""
import math

import pytest

import refcases as R

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MEMBERS = [
    dict(n=(16, 16, 16), visc=1e-2),
    dict(n=(24, 20, 16), visc=3e-3),
    dict(n=(32, 32, 32), visc=1e-3),
    R.channel_kwargs(visc=0.05, bodyforce=(1.0, 0.0, 0.0), ydiffusion="implicit"),
]


@pytest.fixture(scope="module")
def D():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import distributednavierstokes_b200 as dns

    return dns


def _state(D, s, seed):
    u = D.vectorfield(s)
    for i, c in enumerate("xyz"):
        D.noise(u[c], c, s, seed + i, 0.5)
    D.exchange_halo(u, s)
    p = D.scalarfield(s)
    D.project(u, p, s)
    q = D.vectorfield(s)
    delta = D.scalarfield(s) if s.imexy else None
    return u, p, q, delta


def _clone(st):
    u, p, q, delta = st
    return ({c: u[c].clone() for c in "xyz"}, p.clone(), {c: q[c].clone() for c in "xyz"},
            None if delta is None else delta.clone())


def _as_fields(D, st):
    u, p, q, delta = st
    return (D.VectorField(x=u["x"], y=u["y"], z=u["z"]), p,
            D.VectorField(x=q["x"], y=q["y"], z=q["z"]), delta)


def test_ensemble_equals_members_stepped_alone(D):
    setups = [D.setup(**kw) for kw in MEMBERS]
    ref = [_state(D, s, 10 * i) for i, s in enumerate(setups)]
    ens_states = [_as_fields(D, _clone(st)) for st in ref]
    ref = [_as_fields(D, st) for st in ref]
    dts = [0.5 * D.cfl_timestep(st[0], s, 0.5) for st, s in zip(ref, setups)]
    E = D.Ensemble(setups)
    for nsteps in (3, 2):  # the second call replays the captured graph
        E.run(ens_states, dts, nsteps)
        for st, s, dt in zip(ref, setups, dts):
            for _ in range(nsteps):
                D.step(st[0], st[1], st[2], st[3] if st[3] is not None else st[1], s, dt)
        torch.cuda.synchronize()
        for i, (a, b) in enumerate(zip(ens_states, ref)):
            for c in "xyz":
                assert torch.equal(a[0][c], b[0][c]), (i, c)
                assert torch.equal(a[2][c], b[2][c]), (i, c)
            assert torch.equal(a[1], b[1]), i
    # new steps: the graph is captured again
    dts2 = [0.8 * dt for dt in dts]
    E.run(ens_states, dts2, 2)
    for st, s, dt in zip(ref, setups, dts2):
        for _ in range(2):
            D.step(st[0], st[1], st[2], st[3] if st[3] is not None else st[1], s, dt)
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(ens_states, ref)):
        for c in "xyz":
            assert torch.equal(a[0][c], b[0][c]), (i, c)
    for (u, _, _, _), s in zip(ens_states, setups):
        assert D.maxdiv(u, s) < 1e-12
    E.close()


def test_ensemble_rejects_bad_arguments(D):
    s = D.setup(**MEMBERS[0])
    E = D.Ensemble([s])
    st = _as_fields(D, _state(D, s, 1))
    with pytest.raises(Exception):
        E.run([st], [0.0], 1)  # non-positive step
    with pytest.raises(ValueError):
        E.run([st, st], [0.1], 1)
    E.close()


def test_forced_ensemble_equals_members_alone(D):
    """Random-phase initial fields and shell-clamp forcing inside the graph
    (the ensemble configuration's IC and forcing) equal stepping and forcing
    each member alone."""
    kws = [dict(n=(16, 16, 16), visc=1e-2), dict(n=(24, 24, 24), visc=3e-3),
           dict(n=(32, 32, 32), visc=1e-3)]
    setups = [D.setup(**kw) for kw in kws]
    ref, ens_states, forcings, dts = [], [], [], []
    for i, s in enumerate(setups):
        u = D.random_field(D.vectorfield(s), s, totalenergy=0.5, kpeak=4, seed=i)
        st = (u, D.scalarfield(s), D.vectorfield(s), None)
        forcings.append(D.shellforcing(u, s, shells=(1, 2)))
        dts.append(0.5 * D.cfl_timestep(u, s, 0.5))
        ens_states.append(_as_fields(D, _clone(st)))
        ref.append(_as_fields(D, st))
    E = D.Ensemble(setups)
    for i, f in enumerate(forcings):
        E.set_forcing(i, f)
    E.run(ens_states, dts, 3)
    for st, s, dt, f in zip(ref, setups, dts, forcings):
        for _ in range(3):
            D.step(st[0], st[1], st[2], st[1], s, dt)
            f(st[0], s)
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(ens_states, ref)):
        for c in "xyz":
            assert torch.equal(a[0][c], b[0][c]), (i, c)
        e = D.shell_energies(a[0], setups[i], (1, 2))
        assert all(math.isclose(x, y, rel_tol=1e-13) for x, y in zip(e, forcings[i].eref))
    # forcing removed: plain steps again (graph re-captured)
    E.set_forcing(0, None)
    E.run(ens_states, dts, 1)
    D.step(ref[0][0], ref[0][1], ref[0][2], ref[0][1], setups[0], dts[0])
    torch.cuda.synchronize()
    for c in "xyz":
        assert torch.equal(ens_states[0][0][c], ref[0][0][c])
    E.close()


def test_launch_shapes_do_not_change_results(D):
    """A setup created with other launch shapes (dnsb_create_tuned) steps to
    the same bits as the default one; the shapes in effect read back."""
    kw = dict(n=(24, 16, 32), visc=3e-3)
    s0 = D.setup(**kw)
    tun = dict(lines_x=2, lines_y=2, lines_z=1, lines_z4=2, cell_bx=32, cell_by=8)
    s1 = D.setup(**kw, tuning=tun)
    t = s1.tuning()
    assert t["cell_bx"] == 32 and t["cell_by"] == 8 and t["lines_z4"] == 2
    u0 = D.random_field(D.vectorfield(s0), s0, totalenergy=0.5, kpeak=3, seed=4)
    u1 = D.vectorfield(s1)
    for c in "xyz":
        u1[c].copy_(u0[c])
    dt = 0.5 * D.cfl_timestep(u0, s0, 0.5)
    for s, u in ((s0, u0), (s1, u1)):
        p, q = D.scalarfield(s), D.vectorfield(s)
        for _ in range(3):
            D.step(u, p, q, None, s, dt)
    torch.cuda.synchronize()
    for c in "xyz":
        assert torch.equal(u0[c], u1[c]), c
    with pytest.raises(Exception):
        D.setup(**kw, tuning=dict(cell_bx=48, cell_by=2))   # not a multiple of 32
    s0.close()
    s1.close()


def test_autotuner_picks_valid_shapes(D, tmp_path):
    """The coordinate-descent autotuner on a small box returns shapes that
    the library accepts, caches them, and reads the cache back."""
    from distributednavierstokes_b200 import autotune

    cache = str(tmp_path / "tuning.json")
    out, rep = autotune.tune_sizes([16], cache=cache)
    assert 16 in out and not rep[16]["cached"] and rep[16]["ms_per_step"] > 0
    s = D.setup(n=(16, 16, 16), visc=1e-2, tuning=out[16])
    s.close()
    out2, rep2 = autotune.tune_sizes([16], cache=cache)
    assert rep2[16]["cached"] and out2[16] == out[16]


def test_tuned_ensemble_one_launch_many_steps(D):
    """Members with their own launch shapes in the ensemble; 7 steps in one
    graph launch equal 7 steps of each member alone (bit for bit)."""
    kws = [dict(n=(16, 16, 16), visc=1e-2), dict(n=(32, 32, 32), visc=2e-3)]
    tuns = [dict(lines_z4=4, lines_y=4), dict(cell_bx=32, cell_by=4, lines_x=4)]
    setups = [D.setup(**kw, tuning=t) for kw, t in zip(kws, tuns)]
    alone = [D.setup(**kw) for kw in kws]
    ens_states, ref, dts = [], [], []
    for i, (s, sa) in enumerate(zip(setups, alone)):
        u = D.random_field(D.vectorfield(s), s, totalenergy=0.5, kpeak=3, seed=20 + i)
        ua = D.vectorfield(sa)
        for c in "xyz":
            ua[c].copy_(u[c])
        ens_states.append(_as_fields(D, (u, D.scalarfield(s), D.vectorfield(s), None)))
        ref.append(_as_fields(D, (ua, D.scalarfield(sa), D.vectorfield(sa), None)))
        dts.append(0.5 * D.cfl_timestep(u, s, 0.5))
    E = D.Ensemble(setups)
    E.run(ens_states, dts, 7)
    for st, s, dt in zip(ref, alone, dts):
        for _ in range(7):
            D.step(st[0], st[1], st[2], st[1], s, dt)
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(ens_states, ref)):
        for c in "xyz":
            assert torch.equal(a[0][c], b[0][c]), (i, c)
    E.close()
