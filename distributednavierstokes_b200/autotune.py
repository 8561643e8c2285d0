"""Launch-shape autotuner for the batched ensemble (no counterpart in the
reference).

For a periodic box of side n it times one RK3 step under candidate launch
shapes (dnsb_tuning: lines per CTA of the Stockham x-, y- and z-transforms
and of the four-step z-transform, the per-cell kernels' block shape) by
coordinate descent from the defaults: each field in turn takes the value
of its candidates that makes the step fastest (CUDA events over `steps`
steps after two warm-up steps; the best of `repeats` timings), the others
held.  The results do not depend on the shapes, only the time does.
Choices are cached per device name and box in a JSON file.
"""
import json
import os
import time

import torch

from . import api

CANDIDATES = {
    "lines_z4": (2, 4, 8, 16),
    "lines_y": (2, 4, 8, 16),
    "lines_x": (2, 4, 8),
    "cell": ((64, 2), (32, 4), (128, 2), (32, 8)),
}


def default_cache():
    root = os.environ.get("DNSB_TUNE_CACHE") or os.path.join(
        os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache"), "dnsb")
    return os.path.join(root, "tuning.json")


def _time_step(n, visc, tuning, steps, repeats, device):
    s = api.setup(n=(n, n, n), visc=visc, device=device, tuning=tuning)
    try:
        u = api.random_field(api.vectorfield(s), s, totalenergy=0.5, kpeak=4.0, seed=1)
        p, q = api.scalarfield(s), api.vectorfield(s)
        dt = 0.5 * api.cfl_timestep(u, s, 0.5)
        for _ in range(2):
            api.step(u, p, q, None, s, dt)
        best = float("inf")
        stream = torch.cuda.current_stream(device)
        for _ in range(repeats):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(steps):
                api.step(u, p, q, None, s, dt)
            b.record(stream)
            torch.cuda.synchronize(device)
            best = min(best, a.elapsed_time(b) / steps)
        return best, s.tuning()
    finally:
        s.close()


def tune(n, visc=1e-3, steps=10, repeats=3, device=None, log=None):
    """Coordinate descent over CANDIDATES for an n^3 periodic explicit box;
    returns (tuning dict in effect, ms per step, {candidate: ms})."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    cur = {}
    best_ms, eff = _time_step(n, visc, cur, steps, repeats, device)
    tried = {"default": best_ms}
    for field, values in CANDIDATES.items():
        for v in values:
            trial = dict(cur)
            if field == "cell":
                trial["cell_bx"], trial["cell_by"] = v
            else:
                trial[field] = v
            ms, e2 = _time_step(n, visc, trial, steps, repeats, device)
            tried[f"{field}={v}"] = ms
            if ms < best_ms * 0.99:   # keep a change only if it gains more than 1 %
                best_ms, cur, eff = ms, trial, e2
        if log:
            log(f"n={n}: after {field}: {best_ms:.4f} ms {cur}")
    return eff, best_ms, tried


def tune_sizes(sizes, visc=1e-3, cache=None, device=None, log=None, refresh=False):
    """{n: tuning dict} for every box side in `sizes`, from the cache file
    (keyed by device name and side) or measured now and stored."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    cache = cache or default_cache()
    name = torch.cuda.get_device_name(device)
    data = {}
    if os.path.exists(cache) and not refresh:
        try:
            with open(cache) as f:
                data = json.load(f)
        except (OSError, ValueError):
            data = {}
    out, report = {}, {}
    for n in sorted(set(int(v) for v in sizes)):
        key = f"{name}|periodic|{n}"
        if key in data and not refresh:
            out[n] = data[key]["tuning"]
            report[n] = dict(data[key], cached=True)
            continue
        t0 = time.perf_counter()
        eff, ms, tried = tune(n, visc, device=device, log=log)
        data[key] = {"tuning": eff, "ms_per_step": ms, "tried": tried,
                     "seconds": time.perf_counter() - t0}
        out[n] = eff
        report[n] = dict(data[key], cached=False)
    try:
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        with open(cache + ".tmp", "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(cache + ".tmp", cache)
    except OSError:
        pass
    return out, report
