"""Benchmark: FP64 finite-volume channel DNS cell-steps/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload channel384_implicit|channel256_implicit|
                                channel64_explicit|ensemble64_periodic|les64_cnn|
                                spectral256_hit]

One "step" is one full RK3 time step (3 stages: momentum, semi-implicit
wall-normal Crank-Nicolson, FFT/Thomas projection, lagged-pressure update)
of the whole grid, preceded by its CFL reduction, as in the reference's
solve! loop.  The default workload is the production channel: 384x256x384,
domain 4pi x 2 x 4pi/3, tanh(1.5) stretching, nu = 1/395, body force 1,
ydiffusion = :implicit, CFL 0.8, initial condition = a Reichardt mean
profile (Re_tau = 395) plus seeded splitmix64 noise of amplitude 0.2.
Synthetic data of that shape: the reference publishes no dataset.

The line also carries `fft_vs_cufft`: cuFFT (torch.fft) timed on the
shapes of the four Poisson transforms beside the library's own kernels
(--no-cufft skips it).

Prints ONE JSON line on rank 0.  Under torchrun (N > 1) the channel is
decomposed over the ranks in z-slabs (the reference's (P,1) process grid:
z-halos and the Poisson solve's spectrum transposes over NCCL
point-to-point; strong scaling); --replicas runs independent replicas
instead (weak scaling, no collective on the data path).
--impl reference times the CPU oracle (a C/OpenMP restatement of the
reference's Julia path; the Julia reference cannot run here) on the host
cores, on rank 0 only.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))

WORKLOADS = {
    "channel384_implicit": dict(
        n=(384, 256, 384), ydiffusion="implicit", visc=1 / 395, cfl=0.8, amp=0.2, retau=395.0,
        bytes_per_cell_step=1080.0),
    "channel256_implicit": dict(
        n=(256, 192, 256), ydiffusion="implicit", visc=1 / 395, cfl=0.8, amp=0.2, retau=395.0,
        bytes_per_cell_step=1080.0),
    "channel64_explicit": dict(
        n=(64, 64, 64), ydiffusion="explicit", visc=1 / 180, cfl=0.5, amp=0.1, retau=None,
        bytes_per_cell_step=792.0),
    # batched ensemble of triply periodic boxes (2 pi)^3, explicit: 64 members,
    # sizes from SIZES and viscosities log-uniform in [1e-3, 1e-2] drawn with a
    # fixed seed, a fixed step per member (CFL 0.5 of its initial field)
    "ensemble64_periodic": dict(
        members=64, sizes=(32, 48, 64, 96, 128), visc=(1e-3, 1e-2), cfl=0.5, energy=0.5,
        kpeak=4.0, forced_shells=(1, 2), ydiffusion="explicit", bytes_per_cell_step=792.0),
    # the closure study: 256^3 periodic FV DNS (nu = 5e-4, random-phase
    # E(k) ~ k^4 exp(-2 (k/4)^2) field, shell-clamp forcing of shells 1-2)
    # to t = 10 with 200 filtered pairs (Gaussian width 4 dx_DNS onto 64^3);
    # the CNN trained on them (20k Adam steps, lr 1e-3, batches of 8 crops
    # of 32^3); then the CNN-closed and the unclosed 64^3 LES and the DNS
    # itself advanced from t = 10 for 5 time units and compared
    "les64_cnn": dict(
        closure=True, n_dns=256, M=64, visc=5e-4, energy=0.5, kpeak=4.0, shells=(1, 2),
        t_train=10.0, nsnap=200, t_les=5.0, nsample=10, cfl=0.5, train_steps=20000, lr=1e-3,
        batch=8, crop=32),
    # the pseudo-spectral solver on a 256^3 periodic cube (nu = 5e-4, kcut 85):
    # random-phase E(k) ~ k^4 exp(-2 (k/4)^2) initial field, shell-clamp
    # forcing of shells 1-2 after every step, CFL-adaptive Wray steps
    "spectral256_hit": dict(
        spectral=True, n=256, visc=5e-4, cfl=0.85, energy=0.5, kpeak=4.0, forced_shells=(1, 2)),
}
COMMON = dict(lims=((0.0, 4 * math.pi), (-1.0, 1.0), (0.0, 4 * math.pi / 3)),
              bc=("periodic", "wall", "periodic"), bodyforce=(1.0, 0.0, 0.0))

# Algorithmic HBM passes (one FP64 field = nx*ny*nz*8 bytes) per launch of
# each kernel kind on the default path; the half-spectrum counts
# (nx/2+1)/(nx/2) of a real field.  Momentum reads q only from stage 2 on.
# Momentum: r u3 q3 (p1), w q3 V3; q is not read at stage 1 (A = 0).  With
# the fused projection + momentum (grad_momentum: r u*3 delta1 p1 q3,
# w p1 q3 V3) the stand-alone momentum runs at stage 1 only.  The fused
# z-FFT / y-solve / inverse z-FFT (fft_z_y_solve) reads and writes the
# half spectrum once.
def passes(kind, implicit, spec, fused=False):
    if kind == "momentum":
        if fused:
            return 10.0
        return (10 + 13 + 13) / 3 if implicit else (9 + 12 + 12) / 3
    return {"cn_solve": 6.0, "div_rfft_x": 3 + spec, "fft_z": 2 * spec, "y_solve": 2 * spec,
            "ifft_z": 2 * spec, "irfft_x": spec + 1, "grad_update": 9.0 if implicit else 7.0,
            "grad_momentum": 15.0, "fft_z_y_solve": 2 * spec, "other": 0.0}[kind]


def tanhstretch(beta):
    return lambda t: (math.tanh(beta * (2 * t - 1)) / math.tanh(beta) + 1) / 2


def reichardt(y, retau):
    """Reichardt mean profile in wall units (u_tau = 1, half height 1)."""
    yp = (1 - np.abs(y)) * retau
    k = 0.41
    return (np.log1p(k * yp) / k + 7.8 * (1 - np.exp(-yp / 11) - (yp / 11) * np.exp(-yp / 3)))


def mean_profile(wl):
    if wl["retau"] is None:
        return lambda x, y, z: 1.5 * (1 - y ** 2)
    return lambda x, y, z: reichardt(y, wl["retau"]) + 0 * x


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------------------ CPU arm

def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or the platform string."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def cpu_oracle_run(wl, nsteps, nwarm, dt=None, per_step=None):
    """Advance the CPU oracle nwarm + nsteps steps; returns (seconds for
    nsteps, threads, dt used).  per_step, a list, receives each timed step's
    seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    s = O.Setup(wl["n"], lims=COMMON["lims"], bc=COMMON["bc"], stretch=tanhstretch(1.5),
                visc=wl["visc"], bodyforce=COMMON["bodyforce"], ydiffusion=wl["ydiffusion"])
    u = s.vectorfield()
    prof = mean_profile(wl)
    nx, ny, nz = s.n
    s.interior(u["x"])[:] = np.broadcast_to(
        prof(s.xf[None, None, :], s.yc[None, :, None], s.zc[:, None, None]), (nz, ny, nx))
    for c in "xyz":
        s.noise(u[c], c, 0, wl["amp"])
    s.exchange_halo(u)
    p = s.scalarfield()
    q = s.vectorfield()
    delta = s.scalarfield() if s.imexy else p
    s.project(u, delta)
    if dt is None:
        dt = s.cfl_timestep(u, wl["cfl"])
    for _ in range(nwarm):
        s.step(u, p, q, delta, dt)
    t0 = time.perf_counter()
    for _ in range(nsteps):
        t1 = time.perf_counter()
        s.step(u, p, q, delta, dt)
        if per_step is not None:
            per_step.append(time.perf_counter() - t1)
    return time.perf_counter() - t0, threads, dt


def step_stats(per_step):
    """min / median / mean seconds of the timed CPU steps."""
    v = sorted(per_step)
    return {"min": v[0], "median": v[len(v) // 2] if len(v) % 2 else 0.5 * (v[len(v) // 2 - 1] + v[len(v) // 2]),
            "mean": sum(v) / len(v)}


REF_MAX_STEPS = 10


def reference_arm(args, wl, world, rank):
    if rank != 0:
        return
    cells = math.prod(wl["n"])
    # a bounded sample: at most REF_MAX_STEPS full-grid steps are timed (about
    # 2 s each on 16 host cores), so that any --steps K finishes in minutes
    n_run = max(1, min(args.steps, REF_MAX_STEPS))
    n_warm = min(args.warmup, 1)
    per = []
    secs, threads, _ = cpu_oracle_run(wl, n_run, n_warm, per_step=per)
    value = cells * n_run / secs
    # "steps" / "warmup" are the counts this run executed (a bounded sample of
    # the requested ones, which are reported beside them)
    line = {
        "metric": "DNS cell-steps/s (FP64)", "impl": "reference", "value": value,
        "unit": "cell-steps/s", "n_gpus": args.gpus, "steps": n_run, "warmup": n_warm,
        "requested": {"steps": args.steps, "warmup": args.warmup},
        "ms_per_step": 1e3 * secs / n_run, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": list(wl["n"]),
                   "ydiffusion": wl["ydiffusion"], "parallelism": "host cores (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": threads, "kind": "port",
                         "cpu_model": cpu_model(), "step_seconds": step_stats(per),
                         "sample": f"{n_run} timed RK3 steps of the full grid (of the "
                                   f"{args.steps} requested) after {min(args.warmup, 1)} warm-up "
                                   "step (C/OpenMP restatement of the Julia reference; "
                                   "Julia is not available)"},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- GPU arm

def partition_members(cells, world):
    """Members (independent boxes) to ranks without any collective on the
    data path: largest first, each to the least-loaded rank (ties to the
    lower rank), so that every rank derives the same assignment."""
    load = [0] * world
    owner = [0] * len(cells)
    for i in sorted(range(len(cells)), key=lambda i: (-cells[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[i] = r
        load[r] += cells[i]
    return owner


def ensemble_arm(args, wl, world, rank, local):
    """The batched ensemble: one CUDA graph replay advances every member one
    RK3 step; timed against the same members stepped one after another.
    Under torchrun the members are partitioned across the ranks (each rank
    runs its share as its own graph; the job time is the max over ranks)."""
    import torch

    import distributednavierstokes_b200 as dns

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=dev)
    rng = np.random.default_rng(12345)
    ns = rng.choice(wl["sizes"], size=wl["members"])
    lo, hi = np.log(wl["visc"][0]), np.log(wl["visc"][1])
    viscs = np.exp(rng.uniform(lo, hi, size=wl["members"]))
    owner = partition_members([int(n) ** 3 for n in ns], world)
    total_cells = int(sum(int(n) ** 3 for n in ns))
    tunings, tune_report = {}, None
    if not args.no_autotune:
        from distributednavierstokes_b200 import autotune

        t0 = time.perf_counter()
        tunings, rep = autotune.tune_sizes(sorted(set(int(n) for n in ns)), device=dev)
        tune_report = {"seconds": time.perf_counter() - t0,
                       "choices": {str(n): {"tuning": r["tuning"], "ms_per_step": r["ms_per_step"],
                                            "default_ms_per_step": r["tried"].get("default"),
                                            "cached": r["cached"]} for n, r in rep.items()}}
    setups, states, dts, forcings = [], [], [], []
    for i, (n, nu) in enumerate(zip(ns, viscs)):
        if owner[i] != rank:
            continue
        s = dns.setup(n=(int(n),) * 3, visc=float(nu), device=dev, tuning=tunings.get(int(n)))
        # random-phase E(k) ~ k^4 exp(-2 (k/k0)^2) initial field, seed = member id
        u = dns.random_field(dns.vectorfield(s), s, totalenergy=wl["energy"], kpeak=wl["kpeak"],
                             seed=i)
        p = dns.scalarfield(s)
        q = dns.vectorfield(s)
        forcings.append(dns.shellforcing(u, s, shells=wl["forced_shells"]))
        dts.append(dns.cfl_timestep(u, s, wl["cfl"]))
        setups.append(s)
        states.append((u, p, q, None))
    cells = int(sum(int(n) ** 3 for i, n in enumerate(ns) if owner[i] == rank))
    E = dns.Ensemble(setups)
    for i, f in enumerate(forcings):
        E.set_forcing(i, f)
    E.run(states, dts, max(args.warmup, 1))  # captures the graph
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    clocks.start()
    ev0.record(stream)
    E.run(states, dts, args.steps)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    # the same members stepped one after another on one stream
    ev0.record(stream)
    for _ in range(args.steps):
        for s, (u, p, q, _), dt, f in zip(setups, states, dts, forcings):
            dns.step(u, p, q, None, s, dt)
            f(u, s)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms_seq = ev0.elapsed_time(ev1)
    for (u, _, _, _), s in zip(states, setups):
        assert dns.maxdiv(u, s) < 1e-10, "ensemble member lost incompressibility"
    # member-by-member check: the ensemble (tuned members, one graph launch)
    # against every member stepped and forced alone on a default setup, from
    # the same initial fields, args.verify_steps steps
    verify = None
    if args.verify_steps > 0:
        ver_e, ver_a, ver_f = [], [], []
        mine = [i for i in range(len(ns)) if owner[i] == rank]
        for k, i in enumerate(mine):
            s = setups[k]
            u = dns.random_field(dns.vectorfield(s), s, totalenergy=wl["energy"], kpeak=wl["kpeak"],
                                 seed=i)
            sa = dns.setup(n=s.n, visc=s.visc, device=dev)
            ua = dns.vectorfield(sa)
            for c in "xyz":
                ua[c].copy_(u[c])
            ver_e.append((u, dns.scalarfield(s), dns.vectorfield(s), None))
            ver_a.append((sa, ua, dns.scalarfield(sa), dns.vectorfield(sa)))
            ver_f.append(forcings[k])
        E.run(ver_e, dts, args.verify_steps)
        for (sa, ua, pa, qa), dt, f in zip(ver_a, dts, ver_f):
            for _ in range(args.verify_steps):
                dns.step(ua, pa, qa, None, sa, dt)
                f(ua, sa)
        torch.cuda.synchronize(dev)
        worst, identical = 0.0, 0
        for (u, _, _, _), (sa, ua, _, _) in zip(ver_e, ver_a):
            d = max(float((u[c] - ua[c]).abs().max()) / max(float(ua[c].abs().max()), 1e-300)
                    for c in "xyz")
            worst = max(worst, d)
            identical += int(all(torch.equal(u[c], ua[c]) for c in "xyz"))
            sa.close()
        verify = {"steps": args.verify_steps, "members": len(ver_e), "bit_identical": identical,
                  "max_rel_diff": worst,
                  "note": "ensemble (autotuned members, one graph launch) vs each member stepped "
                          "and forced alone with dnsb_step on a default setup"}
    E.close()
    if world > 1:
        t = torch.tensor([ms, ms_seq], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms, ms_seq = float(t[0]), float(t[1])
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    cells = total_cells
    peak, peak_kind = measured_peaks()
    value = cells * args.steps / (ms / 1e3)
    step_gbs = wl["bytes_per_cell_step"] * cells / (ms / args.steps / 1e3) / 1e9 / world
    if rank == 0:
        line = {
            "metric": "DNS cell-steps/s (FP64)", "value": value, "unit": "cell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: random-phase initial fields with E(k) ~ k^4 exp(-2 (k/4)^2) "
                    "from splitmix64 noise (seed = member id), shell-clamp forcing of shells 1-2 "
                    "after every step",
            "config": {"workload": args.workload, "members": wl["members"],
                       "sizes": sorted(set(int(n) for n in ns)), "total_cells": cells,
                       "visc_range": list(wl["visc"]),
                       "parallelism": "1 GPU, one launch of one CUDA graph for all steps" if world == 1 else
                       f"members partitioned over {world} GPUs (no collective on the data path), "
                       "one CUDA graph launch per GPU"},
            "autotune": tune_report,
            "member_check": verify,
            "sequential": {"value": cells * args.steps / (ms_seq / 1e3), "unit": "cell-steps/s",
                           "ms_per_step": ms_seq / args.steps,
                           "note": "the same members stepped one after another on one stream"},
            "step_roofline": {"bytes_per_cell_step": wl["bytes_per_cell_step"],
                              "achieved": step_gbs, "peak": peak, "unit": "GB/s",
                              "frac": step_gbs / peak, "peak_source": peak_kind,
                              "note": "bytes of the RK3 step alone; the shell forcing "
                                      "(direct low-mode sums: one read and one update "
                                      "pass per component per member-step) is "
                                      "extra work inside the timed region"},
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)


def spectral_arm(args, wl, world, rank, local):
    """The pseudo-spectral solver: K CFL-adaptive forced Wray steps of the
    n^3 cube, device-timed; the numpy oracle times one step on the host."""
    import torch

    from distributednavierstokes_b200 import spectral as S

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    s = S.spectral_setup(n=wl["n"], visc=wl["visc"], device=dev)
    uh = S.spectral_randomfield(S.specvelocity(s), s, totalenergy=wl["energy"], kpeak=wl["kpeak"],
                                seed=0)
    f = S.shellforcing(uh, s, shells=wl["forced_shells"])
    kmax = 2 * math.pi * s.kcut / s.l
    vmax = [S.vsummax(uh, s)]

    def one_step():
        dt = wl["cfl"] * math.sqrt(3) / (kmax * (vmax[0] + 1e-300))
        vmax[0] = S.spectral_step(uh, s, dt)
        f(uh, s)

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        one_step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    assert S.spectral_maxdiv(uh, s) < 1e-9, "spectral state lost incompressibility"
    n3 = wl["n"] ** 3
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import spectral_oracle as SO

        O = SO.Spectral(wl["n"], visc=wl["visc"])
        u0 = uh.cpu().numpy()
        t0 = time.perf_counter()
        O.step(u0, 1e-3)
        secs = time.perf_counter() - t0
        cpu = {"value": n3 / secs, "unit": "grid-point steps/s", "cores": 1, "kind": "port",
               "sample": "1 Wray step of the full grid by the numpy oracle (numpy's FFTs, "
                         "one thread; the Julia reference is not available)"}
    if rank == 0:
        print(json.dumps({
            "metric": "spectral grid-point steps/s (FP64)", "value": world * n3 * args.steps / (ms / 1e3),
            "unit": "grid-point steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: random-phase E(k) ~ k^4 exp(-2 (k/4)^2) initial field (seed 0), "
                    "shell-clamp forcing of shells 1-2",
            "config": {"workload": args.workload, "n": wl["n"], "kcut": s.kcut, "visc": wl["visc"],
                       "cfl": wl["cfl"], "parallelism": "1 GPU" if world == 1 else f"replicas x{world}"},
            "clocks": clk, "cpu_baseline": cpu}), flush=True)
    s.close()


def closure_arm(args, wl, world, rank, local):
    """The closure study (les_closure.pipeline): the headline is the
    simulated time per second of the CNN-closed 64^3 LES over that of the
    256^3 DNS on the same GPU, both device-timed over the same 5 time units,
    reported beside the LES's filtered energy-spectrum error for k <= 64/3
    against the filtered DNS (and the unclosed LES's, the fallback).  Runs
    on rank 0; other ranks only join the barrier (replicas, no collective
    on the data path)."""
    import torch

    from distributednavierstokes_b200 import les_closure

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    keys = ("n_dns", "M", "visc", "energy", "kpeak", "shells", "t_train", "nsnap", "t_les", "nsample",
            "cfl", "train_steps", "lr", "batch", "crop")
    kw = {k: wl[k] for k in keys}
    if args.train_steps is not None:
        kw["train_steps"] = args.train_steps
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    res = les_closure.pipeline(device=dev, log=(lambda m: print(m, file=sys.stderr, flush=True)), **kw)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    if rank != 0:
        return
    les = res["les"]
    tr = res["training"]
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    bf16 = float(peaks.get("bf16_tflops_sustained", 1418.6))
    line = {
        "metric": "CNN-LES vs 256^3 DNS simulated-time/s ratio (64^3 LES, E(k) error for k <= kcut)",
        "value": les["speedup_cnn_vs_dns"], "unit": "x", "n_gpus": 1, "steps": les["steps"]["les_cnn"],
        "warmup": 0, "ms_per_step": les["device_ms"]["les_cnn"] / max(les["steps"]["les_cnn"], 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 flow, bf16/fp32 network",
        "data": "synthetic: the library's own DNS (random-phase initial field, seed 0, shell forcing)",
        "config": {"workload": args.workload, **res["config"]},
        "les": {k: v for k, v in les.items() if k != "samples"},
        "les_samples": [{k: v for k, v in r.items() if not k.startswith("E_")} for r in les["samples"]],
        "spectra_final": {k: les["samples"][-1][k] for k in ("E_dns", "E_cnn", "E_plain")},
        "training": tr,
        "dataset": res["dataset"],
        "roofline": {"bound": "tensor", "kernel": "training step (all tensor-core kernels)",
                     "achieved": tr["tflops"], "peak": bf16, "unit": "TFLOP/s",
                     "frac": (tr["tflops"] or 0) / bf16, "traffic": None,
                     "peak_source": "measured (sustained cuBLAS bf16)" if peaks else "fallback",
                     "note": "algorithmic FLOPs (2 x 27 x cin x cout per output voxel and "
                             "pass) over the CUDA-event time of the training loop"},
        "e2e": {"value": les["speedup_cnn_vs_dns"], "unit": "x", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 24.0 * kw["nsample"] / max(les["steps"]["les_cnn"], 1),
                "note": "device-resident state; every advance between two sample times (one "
                        "CUDA-graph launch, the CFL step computed on the device) reads back its "
                        "time and step count (24 bytes) inside the timed region, for both the "
                        "LES and the DNS"},
        "gpu_launches": res.get("closure_launches"),
        "wall_s": wall,
        "clocks": clk,
        "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


def slab_arm(args, wl, world, rank, local):
    """The production channel decomposed over the ranks (strong scaling):
    z-slabs of nz / world planes, z-halos and the Poisson solve's spectrum
    transposes over NCCL point-to-point (slab.py, the reference's (P,1)
    process grid).  Every rank builds the global initial field on its GPU
    and keeps its slab."""
    import datetime

    import torch
    import torch.distributed as dist

    import distributednavierstokes_b200 as dns
    from distributednavierstokes_b200 import slab

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    comm = slab.TorchComm()
    kw = dict(n=wl["n"], stretch=tanhstretch(1.5), visc=wl["visc"], ydiffusion=wl["ydiffusion"], **COMMON)
    sg = dns.setup(device=dev, **kw)
    u = dns.vectorfield(sg)
    dns.velocityfield(u, sg, x=mean_profile(wl))
    for c in "xyz":
        dns.noise(u[c], c, sg, 0, wl["amp"])
    dns.exchange_halo(u, sg)
    delta = dns.scalarfield(sg)
    dns.project(u, delta, sg)
    parts, _ = slab.make_parts(comm, kw, device=dev)
    part = parts[rank]
    us = {c: slab.scatter(parts, u[c])[rank] for c in "xyz"}
    del u, delta
    uu = dns.VectorField(x=us["x"], y=us["y"], z=us["z"])
    st = (uu, dns.scalarfield(part.s), dns.vectorfield(part.s), dns.scalarfield(part.s))
    nx, ny, nz = wl["n"]
    cells = nx * ny * nz

    def one_step():
        dt = slab.cfl_timestep(parts, comm, lambda p: st[0], wl["cfl"])
        slab.step(parts, comm, lambda p: st, dt)

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize(dev)
    dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    clocks.start()
    stream = torch.cuda.current_stream(dev)
    from distributednavierstokes_b200 import _lib

    lib = _lib.load()
    ctxs = [part.s._ctx, sg._ctx]
    n0 = sum(lib.dnsb_launch_count(cx) for cx in ctxs)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        one_step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    launches = sum(lib.dnsb_launch_count(cx) for cx in ctxs) - n0
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    # end to end: the same K steps with this rank's slab of u copied in from
    # pinned host memory first and its u and p copied back after, inside the
    # timed region (the same collective sequence on every rank)
    e2e_err, ms_e2e, slab_bytes = None, 0.0, 0
    try:
        hu = {c: st[0][c].detach().to("cpu").pin_memory() for c in "xyz"}
        hp = st[1].detach().to("cpu").pin_memory()
        slab_bytes = hu["x"].numel() * 8
    except Exception as exc:  # reported in the line; the timing below keeps every rank in step
        e2e_err = f"{type(exc).__name__}: {exc}"
    torch.cuda.synchronize(dev)
    dist.barrier()
    torch.cuda.synchronize(dev)
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    if e2e_err is None:
        for c in "xyz":
            st[0][c].copy_(hu[c], non_blocking=True)
    for _ in range(args.steps):
        one_step()
    if e2e_err is None:
        for c in "xyz":
            hu[c].copy_(st[0][c], non_blocking=True)
        hp.copy_(st[1], non_blocking=True)
    ev3.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = ev2.elapsed_time(ev3)
    t = torch.tensor([ms, ms_e2e, 1.0 if e2e_err else 0.0], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, ms_e2e, e2e_failed = float(t[0].item()), float(t[1].item()), float(t[2].item()) > 0
    md = slab.maxdiv(parts, comm, lambda p: st[0])
    dist.barrier()
    if rank == 0:
        peak, peak_kind = measured_peaks()
        value = cells * args.steps / (ms / 1e3)
        print(json.dumps({
            "metric": "DNS cell-steps/s (FP64)", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "grid": [nx, ny, nz], "ydiffusion": wl["ydiffusion"],
                       "cfl": wl["cfl"], "parallelism": f"z-slabs over {world} GPUs (NCCL halos and "
                                                        "spectrum transposes)"},
            "maxdiv": md, "clocks": clk,
            "step_roofline": {"bytes_per_cell_step": wl["bytes_per_cell_step"],
                              "achieved": wl["bytes_per_cell_step"] * value / 1e9 / world, "peak": peak,
                              "unit": "GB/s per GPU", "peak_source": peak_kind},
            "e2e": ({"unavailable": e2e_err or "the host copies failed on a rank"} if e2e_failed else
                    {"value": cells * args.steps / (ms_e2e / 1e3), "unit": "cell-steps/s",
                     "h2d_bytes_per_step": 3 * slab_bytes * world / args.steps,
                     "d2h_bytes_per_step": 4 * slab_bytes * world / args.steps,
                     "note": "each rank's slab of u from pinned host memory before the K steps, "
                             "u and p back after, inside the timed region (max over ranks)"}),
            "gpu_launches": launches, "cpu_baseline": None}), flush=True)
    for p in parts.values():
        p.close()
    sg.close()
    dist.destroy_process_group()


def b200_arm(args, wl, world, rank, local):
    import ctypes

    import torch

    import distributednavierstokes_b200 as dns
    from distributednavierstokes_b200 import _lib

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    lib = _lib.load()
    s = dns.setup(n=wl["n"], stretch=tanhstretch(1.5), visc=wl["visc"],
                  ydiffusion=wl["ydiffusion"], device=dev, **COMMON)
    nx, ny, nz = s.n
    cells = nx * ny * nz
    G = s.shape[0] * s.shape[1] * s.shape[2]
    u = dns.vectorfield(s)
    dns.velocityfield(u, s, x=mean_profile(wl))
    for c in "xyz":
        dns.noise(u[c], c, s, 0, wl["amp"])
    dns.exchange_halo(u, s)
    host_ic = {c: u[c].cpu().pin_memory() for c in "xyz"}   # for the end-to-end leg
    p = dns.scalarfield(s)
    q = dns.vectorfield(s)
    delta = dns.scalarfield(s) if s.imexy else p
    dns.project(u, delta, s)
    stream = torch.cuda.current_stream(dev)

    def one_step(cached):
        dt = dns.cfl_timestep(u, s, wl["cfl"], use_step_max=cached)
        dns.step(u, p, q, delta, s, dt)
        return dt

    for i in range(args.warmup):
        one_step(i > 0)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    ctx = s.ctx
    n0 = lib.dnsb_launch_count(ctx)
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for i in range(args.steps):
        one_step(True)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    launches = lib.dnsb_launch_count(ctx) - n0
    # Per-kernel device times: the same K steps again with a CUDA event pair
    # around every launch on the library's stream (dnsb_profile).  The event
    # pairs add about 4 % to a step, so the headline pass above runs without
    # them.
    lib.dnsb_profile(ctx, 1)
    evp0 = torch.cuda.Event(enable_timing=True)
    evp1 = torch.cuda.Event(enable_timing=True)
    evp0.record(stream)
    for i in range(args.steps):
        one_step(True)
    evp1.record(stream)
    torch.cuda.synchronize(dev)
    ms_profiled = evp0.elapsed_time(evp1)
    kinds = {}
    for k, name in enumerate(_lib.KINDS):
        t, n = ctypes.c_double(), ctypes.c_long()
        lib.dnsb_profile_read(ctx, k, ctypes.byref(t), ctypes.byref(n))
        kinds[name] = (t.value, n.value)
    lib.dnsb_profile(ctx, 0)
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        torch.distributed.barrier()
    assert dns.maxdiv(u, s) < 1e-10, "benchmark state lost incompressibility"
    value = world * cells * args.steps / (ms / 1e3)

    # roofline of the dominant kernel kind (by device time in the timed region)
    peak, peak_kind = measured_peaks()
    spec = (nx // 2 + 1) / (nx // 2)
    fused = kinds.get("grad_momentum", (0.0, 0))[1] > 0
    dom = max((k for k in kinds if k != "other"), key=lambda k: kinds[k][0])
    t_dom, n_dom = kinds[dom]
    bytes_launch = passes(dom, s.imexy, spec, fused) * cells * 8
    achieved = bytes_launch / (t_dom / n_dom / 1e3) / 1e9
    traffic = step_traffic = None
    tpath = os.path.join(ROOT, "profiles", f"traffic_{args.workload}.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        traffic = tj.get(dom)
        step_traffic = tj.get("_step_dram_bytes_per_cell_step")
    per_kernel = {}
    for k, (t, n) in kinds.items():
        if n == 0:
            continue
        b = passes(k, s.imexy, spec, fused) * cells * 8
        per_kernel[k] = {"launches": n, "ms_avg": t / n, "share": t / sum(v[0] for v in kinds.values()),
                         "gbs": (b / (t / n / 1e3) / 1e9) if b else None}
    step_bytes = wl["bytes_per_cell_step"] * cells
    step_gbs = step_bytes / (ms / args.steps / 1e3) / 1e9

    fftcmp = None
    if rank == 0 and not args.no_cufft and "div_rfft_x" in kinds:
        fftcmp = cufft_leg(s, dev, kinds)
    e2e_line = None
    if not args.no_e2e:
        e2e_line = e2e_leg(lib, s, host_ic, wl, args, world, dev, cells, G)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        per = []
        secs, threads, _ = cpu_oracle_run(wl, args.cpu_steps, 1, per_step=per)
        cpu = {"value": cells * args.cpu_steps / secs, "unit": "cell-steps/s", "cores": threads,
               "kind": "port", "cpu_model": cpu_model(), "step_seconds": step_stats(per),
               "sample": f"{args.cpu_steps} RK3 steps of the full {nx}x{ny}x{nz} grid after 1 "
                         "warm-up step, CPU oracle (C/OpenMP restatement of the Julia "
                         "reference) on all host threads"}

    if rank == 0:
        line = {
            "metric": "DNS cell-steps/s (FP64)", "value": value, "unit": "cell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "grid": [nx, ny, nz],
                       "ydiffusion": wl["ydiffusion"], "cfl": wl["cfl"],
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (each field %.0f MB)" % (G * 8 / 1e6)},
            "e2e": e2e_line,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": bytes_launch,
                         "timing": "CUDA event pair around every launch, over a second pass "
                                   "of the same K steps (%.3f ms/step with the events)"
                                   % (ms_profiled / args.steps)},
            "step_roofline": {"bytes_per_cell_step": wl["bytes_per_cell_step"],
                              "achieved": step_gbs, "peak": peak, "unit": "GB/s",
                              "frac": step_gbs / peak,
                              # ncu DRAM bytes of one whole step per cell-step
                              # (a smaller grid; writes still in L2 at kernel
                              # ends not counted) and the fraction at that figure
                              "dram_bytes_per_cell_step": step_traffic,
                              "dram_frac": (step_traffic * cells / (ms / args.steps / 1e3)
                                            / 1e9 / peak) if step_traffic else None},
            "kernels": per_kernel,
            "fft_vs_cufft": fftcmp,
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def cufft_leg(s, dev, kinds, reps=20):
    """cuFFT (through torch.fft, a library) on the shapes of the Poisson
    solve's four transforms, timed beside the library's own kernels.  Each
    cuFFT transform runs along the contiguous axis of its own tensor, its
    best case: no transposed spectrum, no fused divergence, no ghost images.
    The library's x-transform also forms the divergence from the three
    velocity fields and writes the kz-fastest spectrum; its inverse writes
    the ghosted pressure with its images."""
    import torch

    nx, ny, nz = s.n
    stream = torch.cuda.current_stream(dev)
    gen = torch.Generator(device=dev).manual_seed(0)
    r = torch.randn((nz, ny, nx), dtype=torch.float64, device=dev, generator=gen)
    sx = torch.fft.rfft(r, dim=2)                                   # (nz, ny, nx/2+1)
    sz = torch.randn((nx // 2 + 1, ny, nz), dtype=torch.complex128, device=dev,
                     generator=gen)                                 # kz fastest

    def timed(fn):
        for _ in range(3):
            fn()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    cu = {"rfft_x": timed(lambda: torch.fft.rfft(r, dim=2)),
          "fft_z": timed(lambda: torch.fft.fft(sz, dim=2)),
          "ifft_z": timed(lambda: torch.fft.ifft(sz, dim=2)),
          "irfft_x": timed(lambda: torch.fft.irfft(sx, n=nx, dim=2))}
    cu["total"] = sum(cu.values())
    own = {}
    for k in ("div_rfft_x", "fft_z", "ifft_z", "irfft_x"):
        t, n = kinds.get(k, (0.0, 0))
        if n:
            own[k] = t / n
    if len(own) == 4:
        own["total"] = sum(own.values())
    del r, sx, sz
    torch.cuda.empty_cache()
    return {"shape": [nx, ny, nz], "cufft_ms": cu, "dnsb_ms": own,
            "timing": f"CUDA events, {reps} calls after 3 (cuFFT); live event pairs of the "
                      "timed steps (library)",
            "note": "cuFFT via torch.fft along the contiguous axis of separate tensors "
                    "(complex128 / float64): no transposes, divergence or ghost images"}


def e2e_leg(lib, s, host_ic, wl, args, world, dev, cells, G):
    """End to end through the C ABI with host buffers (dnsb_solve_host)."""
    import ctypes

    import torch

    from distributednavierstokes_b200 import _lib

    # end to end through the C ABI with host buffers (dnsb_solve_host):
    # H2D of the initial velocity, initial projection, K CFL steps, D2H of u, p
    hu = {c: host_ic[c].clone().pin_memory() for c in "xyz"}
    hp = torch.zeros_like(hu["x"]).pin_memory()
    t_out, n_out = ctypes.c_double(), ctypes.c_long()
    # warm-up call (one step): grows the stream-ordered memory pool once
    rc = lib.dnsb_solve_host(s.ctx, *(ctypes.c_void_p(h.data_ptr()) for h in
                                      (hu["x"], hu["y"], hu["z"], hp)),
                             0.0, 1e9, 0.0, wl["cfl"], 1, ctypes.byref(t_out), ctypes.byref(n_out))
    _lib.check(rc, s._ctx)
    for c in "xyz":
        hu[c].copy_(host_ic[c])
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(dev.index or 0)
    clocks.start()
    t0 = time.perf_counter()
    rc = lib.dnsb_solve_host(s.ctx, *(ctypes.c_void_p(h.data_ptr()) for h in
                                      (hu["x"], hu["y"], hu["z"], hp)),
                             0.0, 1e9, 0.0, wl["cfl"], args.steps, ctypes.byref(t_out),
                             ctypes.byref(n_out))
    e2e_s = time.perf_counter() - t0
    clk = clocks.stop()
    _lib.check(rc, s._ctx)
    if world > 1:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = world * cells * n_out.value / e2e_s
    h2d = 3 * G * 8 / n_out.value
    d2h = (4 * G * 8 + 24 * n_out.value) / n_out.value
    return {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "clocks": clk,
            "note": "dnsb_solve_host: pinned host u in, initial projection, "
                    f"{n_out.value} CFL steps, u and p out"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="channel384_implicit", choices=list(WORKLOADS))
    ap.add_argument("--cpu-steps", type=int, default=5,
                    help="timed full-grid CPU oracle steps of the cpu_baseline (about 2 s each)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--replicas", action="store_true",
                    help="under torchrun: independent replicas per GPU instead of the z-slab decomposition")
    ap.add_argument("--no-autotune", action="store_true",
                    help="ensemble workload: default launch shapes instead of autotuned ones")
    ap.add_argument("--verify-steps", type=int, default=500,
                    help="ensemble workload: steps of the member-by-member check (0: skip)")
    ap.add_argument("--train-steps", type=int, default=None,
                    help="closure workload: Adam steps (default: the workload's 20000)")
    ap.add_argument("--no-cufft", action="store_true",
                    help="skip timing cuFFT beside the library's transforms")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "b200" else args.warmup
    wl = WORKLOADS[args.workload]
    world, rank, local = dist_init()
    if wl.get("closure"):
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference has no learned closure or LES path"}), flush=True)
        else:
            closure_arm(args, wl, world, rank, local)
    elif wl.get("spectral"):
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the spectral workload has no CPU reference arm (Julia is absent; "
                                  "the b200 line carries the numpy oracle's one-step time)"}),
                      flush=True)
        else:
            spectral_arm(args, wl, world, rank, local)
    elif "members" in wl:
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference has no ensemble path"}), flush=True)
        else:
            ensemble_arm(args, wl, world, rank, local)
    elif args.impl == "reference":
        reference_arm(args, wl, world, rank)
    elif world > 1 and not args.replicas:
        slab_arm(args, wl, world, rank, local)
    else:
        b200_arm(args, wl, world, rank, local)


if __name__ == "__main__":
    main()
