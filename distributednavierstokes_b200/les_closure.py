"""A-posteriori LES of a periodic box with the CNN closure, and the pipeline
that trains the closure on the library's own DNS.

No counterpart in the reference: DistributedNavierStokes samples filtered
fields and sub-filter stresses (src/spectral/les.jl:302-370) but has no
closure model.  This module chains:

* DNS of a periodic box (FV, explicit RK3, src/timestep.jl:41-63) from the
  random-phase E(k) ~ k^4 exp(-2 (k/k0)^2) field with shell-clamp forcing
  (src/spectral/ic.jl:53-84, src/spectral/forcing.jl:37-56);
* the filtered pair of a snapshot: les.sfs_sample (Gaussian filter of width
  dfac * l / M, exp(-Delta^2 k^2 / 24), les.jl:77; trace-free tau, :370)
  evaluated on the cell centres of the coarse M^3 grid;
* the normalised dataset and the closure's training (closure.Closure);
* the LES step: per RK3 stage the closure's tau(u) (dnsb_cnn_infer), then
  momentum!, the stage update with -div(tau) (dnsb_sfs_stage) and the
  projection; the same step without tau is the unclosed fallback;
* diagnostics against the filtered DNS: shell spectra (floor shells
  1..M/3, as les_spectrum, les.jl:119-131), resolved dissipation and the
  correlation of the LES velocity with the filtered DNS velocity.
"""
import concurrent.futures as cf
import ctypes
import math
import time

import numpy as np

from . import _lib
from . import api
from . import les
from ._lib import check


def sfs_stage(tau, q, u, dt, B, s):
    """dnsb_sfs_stage: q += dt (-div tau) (tau None: nothing), u += B q."""
    lib = _lib.load()
    tp = ctypes.c_void_p(tau.data_ptr()) if tau is not None else None
    check(lib.dnsb_sfs_stage(s.ctx, tp, *(api._ptr(q[c]) for c in "xyz"),
                             *(api._ptr(u[c]) for c in "xyz"), float(dt), float(B)), s._ctx)


def les_step(u, p, q, s, dt, closure=None, tau=None):
    """One explicit RK3 step of step! (src/timestep.jl:41-63) whose stages
    add the closure's -div(tau(u)) (dnsb_les_step: tau(u), momentum!, the
    stage update, the projection, per stage); closure None: the same stages
    without tau."""
    if closure is not None and tau is None:
        raise ValueError("a closure needs the tau buffer")
    h = closure.handle if closure is not None else None
    tp = ctypes.c_void_p(tau.data_ptr()) if closure is not None else None
    check(_lib.load().dnsb_les_step(s.ctx, h, *api._u3(u), api._ptr(p), *api._u3(q), tp, float(dt)),
          s._ctx)
    return u


def advance(u, p, q, s, t, t_end, cfl, forcing=None, closure=None, tau=None, plain=False):
    """CFL-adaptive steps from t to exactly t_end; returns (t_end, steps).
    With a closure: dnsb_les_step; without (or plain): the library's fused
    step (dnsb_step), the unclosed fallback.  A shell forcing from
    api.shellforcing is applied after every step; the whole loop runs in
    dnsb_les_advance: on explicit boxes one launch of a CUDA graph (the
    step size computed on the device; captured on the first call with these
    fields, closure and CFL number, relaunched by later ones), else a host
    loop with one synchronisation per step for the CFL maximum."""
    if closure is not None and plain:
        raise ValueError("plain excludes a closure")
    table = getattr(forcing, "_table", None) if forcing is not None else None
    if forcing is not None and table is None:
        raise ValueError("advance takes the forcing of api.shellforcing")
    h = closure.handle if closure is not None else None
    tp = ctypes.c_void_p(tau.data_ptr()) if closure is not None else None
    eref = table.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if table is not None else None
    t_out, n_out = ctypes.c_double(), ctypes.c_long()
    check(_lib.load().dnsb_les_advance(s.ctx, h, *api._u3(u), api._ptr(p), *api._u3(q), tp, float(t),
                                       float(t_end), float(cfl), eref, len(table) if table is not None else 0,
                                       ctypes.byref(t_out), ctypes.byref(n_out)), s._ctx)
    return t_out.value, n_out.value


# ------------------------------------------------------------ the pairs

def _phase(M, shifts):
    """exp(2 pi i (kx sx + ky sy + kz sz)) on a coarse rfft array [kz, ky, kx]
    (integer wavenumbers; shifts in units of the box length)."""
    kw = np.fft.fftfreq(M, 1.0 / M)
    kx = np.arange(M // 2 + 1)
    sx, sy, sz = shifts
    return (np.exp(2j * math.pi * sz * kw)[:, None, None] * np.exp(2j * math.pi * sy * kw)[None, :, None]
            * np.exp(2j * math.pi * sx * kx)[None, None, :])


def coarse_to_grid(a_hat, M, n_fine, stag=(0.5, 0.5, 0.5)):
    """Values of a coarse spectrum (u_hat = F[u]/N of the fine grid's cell
    centres, dnsb_les_cube) at coarse positions (i + stag) l / M."""
    # the fine transform's sample i sits at (i + 1/2) l / n: shift by the
    # difference to the coarse positions
    sh = [st / M - 0.5 / n_fine for st in stag]
    return np.fft.irfftn(a_hat * _phase(M, sh), s=(M, M, M), axes=(0, 1, 2)) * M ** 3


def sampler(s, M, dfac=1.0, protectshells=2):
    """The one-cell bank of the pipeline: Gaussian filter of width
    dfac * l / M onto the M^3 grid."""
    return les.lessampler(s, cells=[dict(M=M, kernel="gaussian", dfac=dfac)],
                          protectshells=protectshells)


def filtered_pair(u, s, sam, pool=None):
    """(sample, ubar [3, M, M, M], tau [6, M, M, M]) at the coarse cell
    centres.  With a thread pool the host half runs there and a future of
    the same triple is returned."""
    cube = les.les_cube(u, s, sam["nles"])

    def host():
        out = les.sfs_from_cube(sam, cube, s.visc)[0]
        M, n = sam["nles"], s.n[0]
        ub = np.stack([coarse_to_grid(out["ubar"][c], M, n) for c in "xyz"])
        tau = np.stack([coarse_to_grid(out["tau"][k], M, n) for k, _, _ in les.SIGMA])
        return out, ub, tau

    return pool.submit(host) if pool is not None else host()


def normalise(pairs):
    """The dataset [S, 9, M, M, M] float32 of normalised (ubar, tau) and the
    scales: in_scale = 1 / std(ubar_c), out_scale = std(tau_k)."""
    ub = np.stack([p[1] for p in pairs])
    tau = np.stack([p[2] for p in pairs])
    su = ub.std(axis=(0, 2, 3, 4))
    st = tau.std(axis=(0, 2, 3, 4))
    data = np.concatenate([ub / su[None, :, None, None, None], tau / st[None, :, None, None, None]],
                          axis=1).astype(np.float32)
    return data, (1.0 / su).astype(np.float32), st.astype(np.float32)


# -------------------------------------------------------- the LES state

def les_initial_state(ubar_hat, s_les, n_fine):
    """The staggered FV velocity of the M^3 LES box from the filtered DNS
    spectrum (u.x on the x-faces (i+1) l/M, cell centres across), projected
    onto discretely divergence-free fields."""
    import torch

    M = s_les.n[0]
    u = api.vectorfield(s_les)
    for c, st in zip("xyz", ((1.0, 0.5, 0.5), (0.5, 1.0, 0.5), (0.5, 0.5, 1.0))):
        v = coarse_to_grid(ubar_hat[c], M, n_fine, st)
        api.interior(u[c])[:] = torch.from_numpy(np.ascontiguousarray(v)).to(u[c].device)
    api.exchange_halo(u, s_les)
    psi = api.scalarfield(s_les)
    api.project(u, psi, s_les)
    return u


def face_values(ubar_hat, M, n_fine):
    """The filtered DNS velocity on the LES grid's staggered positions."""
    return {c: coarse_to_grid(ubar_hat[c], M, n_fine, st)
            for c, st in zip("xyz", ((1.0, 0.5, 0.5), (0.5, 1.0, 0.5), (0.5, 0.5, 1.0)))}


def spectrum(u, s, kmax):
    """Shell energies 1..kmax (floor shells, each component on its own
    staggered grid) of the FV state."""
    return api.shell_energies(u, s, list(range(1, kmax + 1)))


def correlation(u, ref):
    """sum_c <u_c, ref_c> / sqrt(sum |u|^2 sum |ref|^2) over the interior."""
    num = den_a = den_b = 0.0
    for c in "xyz":
        a = api.interior(u[c]).double().cpu().numpy()
        b = ref[c]
        num += float(np.sum(a * b))
        den_a += float(np.sum(a * a))
        den_b += float(np.sum(b * b))
    return num / math.sqrt(den_a * den_b)


def spectrum_error(E, Eref):
    """Mean and max over the shells of |E / Eref - 1|."""
    r = np.abs(np.asarray(E) / np.asarray(Eref) - 1.0)
    return float(r.mean()), float(r.max())


def resolved_dissipation(E, visc, l=2 * math.pi):
    """2 nu sum_k (2 pi k / l)^2 E(k) over the given shells 1..len(E)."""
    k = 2 * math.pi * np.arange(1, len(E) + 1) / l
    return float(2 * visc * np.sum(k ** 2 * np.asarray(E)))


# ------------------------------------------------------------ the runs

def make_dns(n, visc, energy, kpeak, seed, shells, device):
    s = api.setup(n=(n,) * 3, visc=visc, device=device)
    u = api.random_field(api.vectorfield(s), s, totalenergy=energy, kpeak=kpeak, seed=seed)
    forcing = api.shellforcing(u, s, shells=shells)
    return s, u, forcing


def collect(s, u, forcing, t0, t1, nsnap, sam, cfl, workers=4):
    """Advance the DNS from t0 to t1 taking nsnap filtered pairs at
    t0 + (i+1) (t1 - t0) / nsnap; returns (pairs, t1, steps)."""
    p, q = api.scalarfield(s), api.vectorfield(s)
    futs = []
    t, steps = t0, 0
    with cf.ThreadPoolExecutor(max_workers=workers) as pool:
        for i in range(nsnap):
            tn = t0 + (i + 1) * (t1 - t0) / nsnap
            t, n = advance(u, p, q, s, t, tn, cfl, forcing, plain=True)
            steps += n
            futs.append(filtered_pair(u, s, sam, pool))
        pairs = [f.result() for f in futs]
    return pairs, t, steps


def _events():
    import torch

    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def timed(fn):
    """(result, device ms) of fn() on the current stream."""
    import torch

    a, b = _events()
    a.record()
    r = fn()
    b.record()
    torch.cuda.synchronize()
    return r, a.elapsed_time(b)


def pipeline(n_dns=256, M=64, visc=5e-4, energy=0.5, kpeak=4.0, shells=(1, 2), seed=0,
             t_train=10.0, nsnap=200, t_les=5.0, nsample=10, cfl=0.5, train_steps=20000, lr=1e-3,
             batch=8, crop=32, dfac=1.0, device=None, log=None):
    """The whole closure study on one GPU.

    1. DNS of the n_dns^3 periodic box from t = 0 to t_train, nsnap filtered
       pairs (Gaussian width dfac * l / M onto M^3) spaced t_train / nsnap.
    2. The closure trained on them (train_steps Adam steps, batches of
       `batch` crops of side `crop`).
    3. From the filtered DNS state at t_train: the closed and the unclosed
       (fallback) M^3 LES and the DNS itself advanced t_les, compared at
       nsample times (shell spectra 1..M/3, resolved dissipation, velocity
       correlation; a-priori stress error of the closure on those unseen
       snapshots), each run device-timed.
    Returns a dict of results."""
    import torch

    from .closure import Closure

    say = log or (lambda *a: None)
    dev = device or torch.device("cuda", torch.cuda.current_device())
    kc = M // 3
    res = dict(config=dict(n_dns=n_dns, M=M, visc=visc, energy=energy, kpeak=kpeak, shells=list(shells),
                           t_train=t_train, nsnap=nsnap, t_les=t_les, nsample=nsample, cfl=cfl,
                           train_steps=train_steps, lr=lr, batch=batch, crop=crop, dfac=dfac, kcut=kc))
    s, u, forcing = make_dns(n_dns, visc, energy, kpeak, seed, shells, dev)
    sam = sampler(s, M, dfac)
    t0 = time.perf_counter()
    (pairs, t, steps), ms = timed(lambda: collect(s, u, forcing, 0.0, t_train, nsnap, sam, cfl))
    res["dataset"] = dict(snapshots=len(pairs), dns_steps=steps, wall_s=time.perf_counter() - t0,
                          device_ms=ms)
    say(f"dataset: {len(pairs)} pairs, {steps} DNS steps, {time.perf_counter() - t0:.1f} s")
    data, insc, outsc = normalise(pairs)
    res["scales"] = dict(in_scale=insc.tolist(), out_scale=outsc.tolist())
    dset = torch.from_numpy(data).to(dev)
    cl = Closure(batch=batch, crop=crop, nfield=M, device=dev, seed=seed)
    cl.set_scales(insc, outsc)
    cl.set_dataset(dset)
    cl.profile(True)
    _, tms = timed(lambda: cl.train(train_steps, lr=lr, seed=seed + 1))
    prof = cl.profile_read()
    cl.profile(False)
    losses = cl.losses()
    flops = sum(v[2] for v in prof.values())
    res["training"] = dict(steps=int(train_steps), ms=tms, ms_per_step=tms / max(train_steps, 1),
                           loss_first=float(losses[:100].mean()), loss_last=float(losses[-100:].mean()),
                           tflops=flops / (tms / 1e3) / 1e12 if tms > 0 else None,
                           kernels={k: dict(ms=v[0], launches=v[1], tflops=(v[2] / (v[0] / 1e3) / 1e12
                                                                             if v[0] > 0 else None))
                                    for k, v in prof.items()})
    say(f"training: {train_steps} steps {tms:.0f} ms, loss {losses[:100].mean():.4f} -> {losses[-100:].mean():.4f}")
    del dset

    # ---- a posteriori, from the filtered state at t_train
    s_les = api.setup(n=(M,) * 3, visc=visc, device=dev)
    last = pairs[-1][0]
    u_cnn = les_initial_state(last["ubar"], s_les, n_dns)
    u_pl = api.vectorfield(s_les)
    for c in "xyz":
        u_pl[c].copy_(u_cnn[c])
    f_les = api.shellforcing(u_cnn, s_les, shells=shells, eref=forcing.eref)
    p1, q1, p2, q2 = api.scalarfield(s_les), api.vectorfield(s_les), api.scalarfield(s_les), api.vectorfield(s_les)
    tau = torch.zeros((6, M, M, M), dtype=torch.float64, device=dev)
    pd, qd = api.scalarfield(s), api.vectorfield(s)
    times, rows = [], []
    ms_dns = ms_cnn = ms_pl = 0.0
    st_dns = st_cnn = st_pl = 0
    tt = t_train
    apriori = []
    for i in range(nsample):
        tn = t_train + (i + 1) * t_les / nsample
        (_, n1), m1 = timed(lambda: advance(u, pd, qd, s, tt, tn, cfl, forcing, plain=True))
        (_, n2), m2 = timed(lambda: advance(u_cnn, p1, q1, s_les, tt, tn, cfl, f_les, cl, tau))
        (_, n3), m3 = timed(lambda: advance(u_pl, p2, q2, s_les, tt, tn, cfl, f_les))
        ms_dns, ms_cnn, ms_pl = ms_dns + m1, ms_cnn + m2, ms_pl + m3
        st_dns, st_cnn, st_pl = st_dns + n1, st_cnn + n2, st_pl + n3
        tt = tn
        out, ub, tref = filtered_pair(u, s, sam)
        Ef = out["spectrum"][:kc]
        Ec = spectrum(u_cnn, s_les, kc)
        Ep = spectrum(u_pl, s_les, kc)
        ref = face_values(out["ubar"], M, n_dns)
        # a priori: the closure's stress on this unseen filtered field
        tp = cl.infer_cells(torch.from_numpy(ub).to(dev)).cpu().numpy()
        sc = np.asarray(outsc, dtype=np.float64)[:, None, None, None]
        apriori.append(float(np.mean(((tp - tref) / sc) ** 2)) / float(np.mean((tref / sc) ** 2)))
        ec, ecm = spectrum_error(Ec, Ef)
        ep, epm = spectrum_error(Ep, Ef)
        rows.append(dict(t=tn, err_cnn=ec, err_cnn_max=ecm, err_plain=ep, err_plain_max=epm,
                         diss_dns=resolved_dissipation(Ef, visc), diss_cnn=resolved_dissipation(Ec, visc),
                         diss_plain=resolved_dissipation(Ep, visc),
                         corr_cnn=correlation(u_cnn, ref), corr_plain=correlation(u_pl, ref),
                         E_dns=list(map(float, Ef)), E_cnn=list(map(float, Ec)), E_plain=list(map(float, Ep))))
        say(f"t={tn:.2f}: E(k) err cnn {ec:.3f} plain {ep:.3f}; corr {rows[-1]['corr_cnn']:.3f} / "
            f"{rows[-1]['corr_plain']:.3f}; a priori {apriori[-1]:.3f}")
    simrate = lambda ms: t_les / (ms / 1e3)
    res["les"] = dict(
        samples=rows,
        spectrum_err_cnn=float(np.mean([r["err_cnn"] for r in rows])),
        spectrum_err_plain=float(np.mean([r["err_plain"] for r in rows])),
        spectrum_err_cnn_final=rows[-1]["err_cnn"], spectrum_err_plain_final=rows[-1]["err_plain"],
        diss_err_cnn=float(np.mean([abs(r["diss_cnn"] / r["diss_dns"] - 1) for r in rows])),
        diss_err_plain=float(np.mean([abs(r["diss_plain"] / r["diss_dns"] - 1) for r in rows])),
        corr_cnn_final=rows[-1]["corr_cnn"], corr_plain_final=rows[-1]["corr_plain"],
        apriori_rel_mse=float(np.mean(apriori)),
        simtime_per_s=dict(dns=simrate(ms_dns), les_cnn=simrate(ms_cnn), les_plain=simrate(ms_pl)),
        steps=dict(dns=st_dns, les_cnn=st_cnn, les_plain=st_pl),
        device_ms=dict(dns=ms_dns, les_cnn=ms_cnn, les_plain=ms_pl),
        speedup_cnn_vs_dns=ms_dns / ms_cnn, speedup_plain_vs_dns=ms_dns / ms_pl)
    res["closure_launches"] = cl.launch_count()
    cl.close()
    s_les.close()
    s.close()
    return res
