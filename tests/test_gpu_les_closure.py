"""The closure in the loop: the SFS stage update (dnsb_sfs_stage) against a
numpy restatement of its discrete -div(tau), the plain stage sequence
against the library's fused step, the CNN-closed LES step, and a small
end-to-end study (DNS -> filtered pairs -> training -> LES) in which the
trained closure must beat the method without it on unseen snapshots.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import distributednavierstokes_b200 as dns
    from distributednavierstokes_b200 import les_closure

    return dns, les_closure


def rel(a, b):
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


def sfs_force_numpy(tau, dx, dy, dz):
    """-div(tau) on the staggered faces of a uniform periodic box; tau
    [6, nz, ny, nx] (xx, yy, zz, xy, yz, zx), returns f[c] [nz, ny, nx] at
    the faces (i+1/2, j, k), (i, j+1/2, k), (i, j, k+1/2)."""
    xx, yy, zz, xy, yz, zx = tau
    sh = lambda a, ax, d: np.roll(a, -d, axis=ax)     # a[i + d] along ax
    X, Y, Z = 2, 1, 0
    edge = lambda a, a1, a2, d1, d2: 0.25 * (a + sh(a, a1, d1) + sh(a, a2, d2) + sh(sh(a, a1, d1), a2, d2))
    fx = -((sh(xx, X, 1) - xx) / dx + (edge(xy, X, Y, 1, 1) - edge(xy, X, Y, 1, -1)) / dy
           + (edge(zx, X, Z, 1, 1) - edge(zx, X, Z, 1, -1)) / dz)
    fy = -((edge(xy, Y, X, 1, 1) - edge(xy, Y, X, 1, -1)) / dx + (sh(yy, Y, 1) - yy) / dy
           + (edge(yz, Y, Z, 1, 1) - edge(yz, Y, Z, 1, -1)) / dz)
    fz = -((edge(zx, Z, X, 1, 1) - edge(zx, Z, X, 1, -1)) / dx + (edge(yz, Z, Y, 1, 1) - edge(yz, Z, Y, 1, -1)) / dy
           + (sh(zz, Z, 1) - zz) / dz)
    return fx, fy, fz


def test_sfs_force_matches_numpy(M):
    dns, L = M
    n = (12, 10, 8)
    s = dns.setup(n=n, lims=((0, 2.0), (0, 3.0), (0, 1.5)), visc=0.01)
    rng = np.random.default_rng(1)
    tau = rng.standard_normal((6, n[2], n[1], n[0]))
    q, u = dns.vectorfield(s), dns.vectorfield(s)
    L.sfs_stage(torch.from_numpy(tau).cuda(), q, u, 1.0, 0.0, s)
    ref = sfs_force_numpy(tau, s.dx, 3.0 / 10, s.dz)
    for c, f in zip("xyz", ref):
        assert rel(dns.interior(q[c]).cpu().numpy(), f) <= 1e-13, c
    s.close()


def test_plain_stages_match_fused_step(M):
    """momentum! -> stage update -> projection per stage (the closure's
    sequence without a closure) equals dnsb_step on a periodic box."""
    dns, L = M
    s = dns.setup(n=(16, 16, 16), visc=0.01)
    u = dns.random_field(dns.vectorfield(s), s, totalenergy=0.5, kpeak=3.0, seed=2)
    u2 = dns.vectorfield(s)
    for c in "xyz":
        u2[c].copy_(u[c])
    dt = dns.cfl_timestep(u, s, 0.5)
    p, q = dns.scalarfield(s), dns.vectorfield(s)
    dns.step(u, p, q, None, s, dt)
    p2, q2 = dns.scalarfield(s), dns.vectorfield(s)
    L.les_step(u2, p2, q2, s, dt)
    for c in "xyz":
        assert rel(u2[c].cpu().numpy(), u[c].cpu().numpy()) <= 1e-13, c
    s.close()


def test_closed_les_step(M):
    """With a closure each stage adds -div(tau(u)): the step stays
    divergence-free, differs from the unclosed one, and its first stage's
    q matches momentum + dt * f(tau) of the closure's own output."""
    dns, L = M
    from distributednavierstokes_b200.closure import Closure

    n = 16
    s = dns.setup(n=(n,) * 3, visc=0.01)
    cl = Closure(batch=0, crop=0, nfield=n, seed=4)
    cl.set_scales([2.0, 2.0, 2.0], [0.2] * 6)
    u = dns.random_field(dns.vectorfield(s), s, totalenergy=0.5, kpeak=3.0, seed=3)
    u_pl = dns.vectorfield(s)
    for c in "xyz":
        u_pl[c].copy_(u[c])
    dt = dns.cfl_timestep(u, s, 0.5)
    tau = torch.zeros((6, n, n, n), dtype=torch.float64, device="cuda")
    # first stage by hand: tau(u), q = dt F(u) + dt f(tau)
    t0 = cl.infer(u).cpu().numpy()
    q0 = dns.vectorfield(s)
    dns.momentum(q0, u, 0.0, dt, s)
    fref = sfs_force_numpy(t0, s.dx, s.dy[1], s.dz)
    p, q = dns.scalarfield(s), dns.vectorfield(s)
    L.les_step(u, p, q, s, dt, cl, tau)
    assert dns.maxdiv(u, s) < 1e-12
    p2, q2 = dns.scalarfield(s), dns.vectorfield(s)
    L.les_step(u_pl, p2, q2, s, dt)
    diff = max(float((u[c] - u_pl[c]).abs().max()) for c in "xyz")
    assert diff > 1e-6
    # the stage update alone on a copy of the first stage reproduces q
    qa = dns.vectorfield(s)
    for c in "xyz":
        qa[c].copy_(q0[c])
    ua = dns.vectorfield(s)
    L.sfs_stage(torch.from_numpy(t0).cuda(), qa, ua, dt, 0.0, s)
    for c, f in zip("xyz", fref):
        got = dns.interior(qa[c]).cpu().numpy() - dns.interior(q0[c]).cpu().numpy()
        assert rel(got, dt * f) <= 1e-12, c
    cl.close()
    s.close()


def test_small_study_closure_beats_unclosed(M):
    """64^3 DNS (nu = 5e-3) -> 24 filtered pairs on 16^3 -> 600 Adam steps
    -> on snapshots the network never saw, its stress error (relative MSE)
    is below the unclosed model's (tau = 0, relative MSE 1); the closed and
    unclosed 16^3 LES both run and stay finite."""
    dns, L = M
    res = L.pipeline(n_dns=64, M=16, visc=5e-3, energy=0.5, kpeak=3.0, t_train=2.0, nsnap=24,
                     t_les=0.4, nsample=2, cfl=0.5, train_steps=600, lr=2e-3, batch=4, crop=8)
    tr, les = res["training"], res["les"]
    print({k: les[k] for k in ("apriori_rel_mse", "spectrum_err_cnn", "spectrum_err_plain",
                               "corr_cnn_final", "corr_plain_final", "speedup_cnn_vs_dns")})
    assert tr["loss_last"] < tr["loss_first"]
    assert les["apriori_rel_mse"] < 0.9
    assert math.isfinite(les["spectrum_err_cnn"]) and math.isfinite(les["spectrum_err_plain"])
    assert les["steps"]["les_cnn"] > 0 and les["steps"]["dns"] > 0


@pytest.mark.parametrize("graph", ["1", "0"])
def test_les_advance_matches_step_loop(M, graph, monkeypatch):
    """dnsb_les_advance (CFL steps, closure every stage, shell clamp after
    each step, the last step shortened onto t1) equals the same loop driven
    step by step from Python bit for bit; without a closure it runs
    dnsb_step.  graph "1": the whole run as one CUDA-graph launch with the
    step size computed on the device (the default); "0": the host loop."""
    monkeypatch.setenv("DNSB_LESGRAPH", graph)
    dns, L = M
    from distributednavierstokes_b200.closure import Closure

    n = 16
    s = dns.setup(n=(n,) * 3, visc=0.01)
    cl = Closure(batch=0, crop=0, nfield=n, seed=5)
    cl.set_scales([2.0, 2.0, 2.0], [0.2] * 6)
    u = dns.random_field(dns.vectorfield(s), s, totalenergy=0.5, kpeak=3.0, seed=7)
    forcing = dns.shellforcing(u, s, shells=(1, 2))
    fields = []
    for _ in range(4):
        v = dns.vectorfield(s)
        for c in "xyz":
            v[c].copy_(u[c])
        fields.append(v)
    tau = torch.zeros((6, n, n, n), dtype=torch.float64, device="cuda")
    t1 = 0.4
    for closed, (ua, ub) in ((True, fields[:2]), (False, fields[2:])):
        p, q = dns.scalarfield(s), dns.vectorfield(s)
        t_end, steps = L.advance(ua, p, q, s, 0.0, t1, 0.5, forcing, cl if closed else None,
                                 tau if closed else None)
        assert t_end == t1 and steps >= 2
        p2, q2 = dns.scalarfield(s), dns.vectorfield(s)
        t, k = 0.0, 0
        while t < t1 - 1e-12 * (abs(t1) + 1):
            dt = min(dns.cfl_timestep(ub, s, 0.5), t1 - t)
            if closed:
                L.les_step(ub, p2, q2, s, dt, cl, tau)
            else:
                dns.step(ub, p2, q2, None, s, dt)
            forcing(ub, s)
            t += dt
            k += 1
        assert k == steps
        for c in "xyz":
            assert torch.equal(ua[c], ub[c]), (closed, c)
    cl.close()
    s.close()


def test_les_advance_graph_reuse(M):
    """The advance graph is captured once per argument set and relaunched
    for later intervals: closed and unclosed runs alternating on one
    context over six intervals, a wait-limit change between two of them
    (a new capture), the closure's per-launch timing on (the host loop) and
    off again (the earlier graph relaunched), and a closure created after
    the first one was closed (a new capture even where the new closure
    reuses the old one's address) each equal the step-by-step loop bit for
    bit."""
    dns, L = M
    from distributednavierstokes_b200 import _lib
    from distributednavierstokes_b200.closure import Closure

    n = 16
    s = dns.setup(n=(n,) * 3, visc=0.01)
    u = dns.random_field(dns.vectorfield(s), s, totalenergy=0.5, kpeak=3.0, seed=11)
    forcing = dns.shellforcing(u, s, shells=(1, 2))
    copies = []
    for _ in range(4):
        v = dns.vectorfield(s)
        for c in "xyz":
            v[c].copy_(u[c])
        copies.append((v, dns.scalarfield(s), dns.vectorfield(s)))
    tau = torch.zeros((6, n, n, n), dtype=torch.float64, device="cuda")

    def loop(ub, p, q, t, t1, cl):
        k = 0
        while t < t1 - 1e-12 * (abs(t1) + 1):
            dt = min(dns.cfl_timestep(ub, s, 0.5), t1 - t)
            if cl is not None:
                L.les_step(ub, p, q, s, dt, cl, tau)
            else:
                dns.step(ub, p, q, None, s, dt)
            forcing(ub, s)
            t += dt
            k += 1
        return k

    cl = Closure(batch=0, crop=0, nfield=n, seed=5)
    cl.set_scales([2.0, 2.0, 2.0], [0.2] * 6)
    times = (0.0, 0.15, 0.3, 0.45, 0.6, 0.75, 0.9)
    for i in range(6):
        t0, t1 = times[i], times[i + 1]
        if i == 2:
            assert _lib.load().dnsb_set_wait_limit(s.ctx, 1 << 26) == 0
        if i == 3:  # the closure's per-launch timing on: the host loop
            cl.profile(True)
        if i == 4:  # off again: the graph captured at i == 2 is relaunched
            cl.profile_read()
            cl.profile(False)
        if i == 5:
            cl.close()
            cl = Closure(batch=0, crop=0, nfield=n, seed=6)
            cl.set_scales([2.0, 2.0, 2.0], [0.2] * 6)
        for closed, (ga, ref) in ((True, (copies[0], copies[1])), (False, (copies[2], copies[3]))):
            c = cl if closed else None
            t_end, steps = L.advance(*ga, s, t0, t1, 0.5, forcing, c, tau if closed else None)
            assert t_end == t1 and steps >= 1
            assert loop(*ref, t0, t1, c) == steps, (i, closed)
            for comp in "xyz":
                assert torch.equal(ga[0][comp], ref[0][comp]), (i, closed, comp)
    cl.close()
    s.close()


def test_les_advance_edges(M):
    """dnsb_les_advance: an interval shorter than the time tolerance takes no
    step and leaves u alone; a closure without its tau buffer and the closed
    step on a semi-implicit (channel) context are refused with an error."""
    dns, L = M
    from distributednavierstokes_b200 import _lib
    from distributednavierstokes_b200.closure import Closure

    n = 16
    s = dns.setup(n=(n,) * 3, visc=0.01)
    u = dns.random_field(dns.vectorfield(s), s, totalenergy=0.5, kpeak=3.0, seed=9)
    u0 = {c: u[c].clone() for c in "xyz"}
    p, q = dns.scalarfield(s), dns.vectorfield(s)
    t_end, steps = L.advance(u, p, q, s, 0.3, 0.3, 0.5)
    assert (t_end, steps) == (0.3, 0)
    for c in "xyz":
        assert torch.equal(u[c], u0[c]), c
    cl = Closure(batch=0, crop=0, nfield=n, seed=1)
    with pytest.raises(ValueError):
        L.les_step(u, p, q, s, 0.01, cl, None)
    ch = dns.setup(n=(16, 12, 16), lims=((0, 1.0), (-1, 1), (0, 1.0)),
                   bc=("periodic", "wall", "periodic"), visc=0.01, ydiffusion="implicit")
    uc = dns.vectorfield(ch)
    pc, qc = dns.scalarfield(ch), dns.vectorfield(ch)
    tau = torch.zeros((6, n, n, n), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.DNSBError):
        L.les_step(uc, pc, qc, ch, 0.01, cl, tau)
    cl.close()
    ch.close()
    s.close()
