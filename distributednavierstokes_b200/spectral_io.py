"""Snapshot and checkpoint IO of the spectral state in the reference's own
file format (src/spectral/io.jl:30-230), one rank.

<prefix>.bin holds the three components of the compact state in global
index order — the column-major (kcut+1, m, m) ComplexF64 arrays one after
another, which is the byte order of this package's (3, m, m, kcut+1)
complex128 tensors — and <prefix>.toml the metadata (format, version,
eltype, n, kcut, m, l, visc, time, step, order, data, meta).  Both files
are written under temporary names and renamed, the sidecar first, so a
complete pair is all or nothing; snapshots written here load in the
reference and vice versa.
"""
import math
import os
import re
import time as _time
import tomllib

import numpy as np
import torch

FORMAT = "DistributedNavierStokes spectral state"
ORDER = ("column-major (kx, ky, kz, component) complex; "
         "kx = 0:kcut, ky/kz wrapped 0:kcut then -kcut:-1")


def _toml_value(v):
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        f = float(v)
        if math.isnan(f):
            return "nan"
        if math.isinf(f):
            return "inf" if f > 0 else "-inf"
        r = repr(f)
        return r if ("." in r or "e" in r or "n" in r) else r + ".0"
    if isinstance(v, str):
        return '"' + v.replace("\\", "\\\\").replace('"', '\\"') + '"'
    if isinstance(v, (list, tuple, np.ndarray)):
        return "[" + ", ".join(_toml_value(x) for x in list(np.asarray(v).tolist())) + "]"
    raise TypeError(f"cannot write {type(v).__name__} to TOML")


def _toml_dump(d):
    """The sidecar as TOML with sorted keys (TOML.print(...; sorted = true))."""
    lines = [f"{k} = {_toml_value(v)}" for k, v in sorted(d.items()) if not isinstance(v, dict)]
    for k, v in sorted(d.items()):
        if isinstance(v, dict):
            lines.append("")
            lines.append(f"[{k}]")
            lines += [f"{kk} = {_toml_value(vv)}" for kk, vv in sorted(v.items())]
    return "\n".join(lines) + "\n"


def spectral_save(prefix, uh, s, time=0.0, step=0, meta=None):
    """spectral_save(prefix, uh, s; time, step, meta) (src/spectral/io.jl:30-75)."""
    datafile, metafile = prefix + ".bin", prefix + ".toml"
    a = uh.detach().cpu().numpy() if hasattr(uh, "detach") else np.asarray(uh)
    if a.shape != (3, s.m, s.m, s.kcut + 1):
        raise ValueError(f"state of shape {a.shape}, setup expects {(3, s.m, s.m, s.kcut + 1)}")
    with open(datafile + ".tmp", "wb") as fh:
        fh.write(np.ascontiguousarray(a, dtype=np.complex128).tobytes())
    d = {"format": FORMAT, "version": 1, "eltype": "Float64", "n": s.n, "kcut": s.kcut, "m": s.m,
         "l": float(s.l), "visc": float(s.visc), "time": float(time), "step": int(step),
         "order": ORDER, "data": os.path.basename(datafile)}
    if meta:
        d["meta"] = {str(k): (v if isinstance(v, (int, float, str, bool)) else np.asarray(v).tolist())
                     for k, v in dict(meta).items()}
    with open(metafile + ".tmp", "w") as fh:
        fh.write(_toml_dump(d))
    os.replace(metafile + ".tmp", metafile)
    os.replace(datafile + ".tmp", datafile)
    return prefix


def spectral_load(uh, prefix, s):
    """spectral_load!(uh, prefix, s) (src/spectral/io.jl:77-104): the
    retained modes must match (kcut, l, eltype); the transform grid n need
    not.  Returns dict(time, step, meta)."""
    with open(prefix + ".toml", "rb") as fh:
        d = tomllib.load(fh)
    if not (d["eltype"] == "Float64" and d["kcut"] == s.kcut and d["l"] == float(s.l)):
        raise ValueError(f"snapshot {prefix} (eltype {d['eltype']}, kcut {d['kcut']}, l {d['l']}) "
                         f"does not match setup (eltype Float64, kcut {s.kcut}, l {s.l})")
    a = np.fromfile(prefix + ".bin", dtype=np.complex128)
    if a.size != 3 * s.m * s.m * (s.kcut + 1):
        raise ValueError(f"snapshot {prefix}: {a.size} values, expected {3 * s.m * s.m * (s.kcut + 1)}")
    a = a.reshape(3, s.m, s.m, s.kcut + 1)
    if hasattr(uh, "copy_"):
        uh.copy_(torch.from_numpy(a))
    else:
        uh[...] = a
    return dict(time=d["time"], step=d["step"], meta=d.get("meta", {}))


def checkpointlist(prefix):
    """checkpointlist(prefix) (src/spectral/io.jl:106-120): prefixes
    <prefix>_<step> with complete file pairs, ascending by step."""
    dirname = os.path.dirname(prefix) or "."
    base = os.path.basename(prefix)
    if not os.path.isdir(dirname):
        return []
    pat = re.compile("^" + re.escape(base) + r"_(\d+)\.toml$")
    steps = []
    for f in os.listdir(dirname):
        mm = pat.match(f)
        if mm and os.path.isfile(os.path.join(dirname, f"{base}_{mm.group(1)}.bin")):
            steps.append(int(mm.group(1)))
    return [os.path.join(dirname, "%s_%09d" % (base, st)) for st in sorted(steps)]


def spectral_latest(prefix):
    """spectral_latest(prefix, s): the newest complete checkpoint or None."""
    lst = checkpointlist(prefix)
    return lst[-1] if lst else None


def checkpointer(prefix, interval=900.0, stopfile=None, keep=2, meta=None):
    """checkpointer(prefix; interval, stopfile, keep, meta) (src/spectral/
    io.jl:150-184): a spectral_solve processor writing <prefix>_<step> every
    `interval` wall-clock seconds and when `stopfile` exists (then returning
    "stop"), keeping the newest `keep`."""
    tlast = [_time.time()]

    def proc(state, s):
        due = _time.time() - tlast[0] >= interval
        stop = stopfile is not None and os.path.isfile(stopfile)
        if not (due or stop):
            return None
        spectral_save("%s_%09d" % (prefix, state.n), state.uh, s, time=state.t, step=state.n,
                      meta=meta)
        tlast[0] = _time.time()
        old = checkpointlist(prefix)
        for p in old[:len(old) - min(keep, len(old))]:
            for ext in (".bin", ".toml"):
                try:
                    os.remove(p + ext)
                except FileNotFoundError:
                    pass
        return "stop" if stop else None

    return proc


def snapshotsaver(prefix, times, meta=None, stats=True, tstart=-math.inf):
    """snapshotsaver(prefix; times, meta, stats, tstart) (src/spectral/
    io.jl:186-229): saves <prefix>_0001, ... the first time t reaches each
    entry of `times` (pass them as tstops); with stats the sidecar's meta
    also carries eta, t_int, e, diss of spectral_stats; entries before
    tstart are skipped on restart."""
    times = sorted(float(t) for t in times)
    i0 = next((i for i, t in enumerate(times) if t >= tstart - 1e-10 * (abs(t) + 1)), len(times))
    inext = [i0]

    def proc(state, s):
        while inext[0] < len(times) and state.t >= times[inext[0]] - 1e-10 * (abs(times[inext[0]]) + 1):
            m = dict(meta or {})
            if stats:
                from .spectral import spectral_stats

                st = spectral_stats(state.uh, s)
                m.update(eta=st["l_kol"], t_int=st["t_int"], e=st["e"], diss=st["diss"])
            spectral_save("%s_%04d" % (prefix, inext[0] + 1), state.uh, s, time=state.t,
                          step=state.n, meta=m)
            inext[0] += 1
        return None

    return proc


def spectral_from_rfft(uh, F, s):
    """spectral_from_rfft!(uh, F, s) (src/spectral/io.jl:264-292): the
    truncated state from three full rfft arrays, numpy shape
    (nf, nf, nf//2+1) = [kz, ky, kx] with wrapped frequencies; nf >= 3 kcut."""
    Fs = list(F.values()) if isinstance(F, dict) else list(F)
    if len(Fs) != 3:
        raise ValueError("F must hold three velocity components")
    nf = Fs[0].shape[0]
    if any(f.shape != (nf, nf, nf // 2 + 1) for f in Fs):
        raise ValueError("expected full rfft layout")
    if nf < 3 * s.kcut:
        raise ValueError(f"source grid nf = {nf} cannot hold kcut = {s.kcut} retained modes")
    cf = np.array([j if j <= s.kcut else j - s.m for j in range(s.m)])
    idx = cf % nf
    A = np.stack([np.asarray(f)[np.ix_(idx, idx, np.arange(s.kcut + 1))] for f in Fs])
    if hasattr(uh, "copy_"):
        uh.copy_(torch.from_numpy(np.ascontiguousarray(A, dtype=np.complex128)))
    else:
        uh[...] = A
    return uh


# ---------------------------------------------------- the SFS bank writers
# sfscollector / sfswriter / sfs_offline (src/spectral/les.jl:384-540) with
# the reference's directory layout and array names; the archives are numpy
# .npz files (there is no JLD2/HDF5 writer in this environment), written
# atomically like jldsave_atomic.

def etacells(deta, eta, l, Ms, kernels=("gaussian",), window=(2.0, 5.0)):
    """etacells(; deta, eta, l, Ms, kernels, window) (src/spectral/les.jl:207-224):
    for each width (in units of the Kolmogorov length eta) and kernel, every
    coarse grid M whose Delta/h = deta eta M / l lies inside the window."""
    out = []
    for de in deta:
        for kernel in kernels:
            for M in sorted(Ms):
                r = de * eta * M / l
                if window[0] - 1e-9 <= r <= window[1] + 1e-9:
                    out.append(dict(M=int(M), kernel=str(kernel), dfac=float(f"{r:.4g}"),
                                    deta=float(de)))
    return out


def celldir(d, cell, legacy):
    """celldir (src/spectral/les.jl:397-407)."""
    if legacy:
        return os.path.join(d, f"delta={cell['dfac']}")
    return os.path.join(d, f"filter={cell['kernel']}", f"M={cell['M']}", f"delta={cell['dfac']}")


def _save_npz_atomic(path, **arrays):
    tmp = path + ".tmp.npz"
    try:
        np.savez(tmp, **arrays)
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.remove(tmp)
        raise


def sfscollector(sam, s, d):
    """sfscollector (src/spectral/les.jl:409-475): record(t, uh) samples the
    bank; finish() writes dns_meta.npz and, per cell, fields.npz and
    les_meta.npz."""
    from . import spectral as S

    cells = sam["cells"]
    tstart = _time.time()
    st = dict(times=[], spectra_dns=[], statistics=[], inputs=[[] for _ in cells],
              outputs=[[] for _ in cells], redelta=[[] for _ in cells],
              spectra_les=[[] for _ in cells])

    def record(t, uh):
        stats = S.spectral_stats(uh, s)
        sp = S.spectral_spectrum(uh, s)
        samples = S.sfs_sample(sam, uh, s)
        st["times"].append(float(t))
        st["spectra_dns"].append(np.asarray(sp["E"][1:], dtype=np.float64))
        st["statistics"].append(stats)
        for k, smp in enumerate(samples):
            st["inputs"][k].append(np.stack([smp["ubar"][c] for c in "xyz"]))
            st["outputs"][k].append(np.stack([smp["tau"][c]
                                              for c in ("xx", "yy", "zz", "xy", "yz", "zx")]))
            st["redelta"][k].append(smp["redelta"])
            st["spectra_les"][k].append(smp["spectrum"])

    def finish():
        if not st["times"]:
            return
        os.makedirs(d, exist_ok=True)
        keys = list(st["statistics"][0].keys())
        _save_npz_atomic(os.path.join(d, "dns_meta.npz"), times=np.array(st["times"]),
                         spectra_dns=np.array(st["spectra_dns"]),
                         statistics_dns=np.array([[x[k] for k in keys] for x in st["statistics"]]),
                         statistics_names=np.array(keys),
                         t_int=st["statistics"][0]["t_int"], walltime=_time.time() - tstart)
        legacy = all(c["kernel"] == "gaussian" and c["M"] == sam["nles"] and c.get("deta") is None
                     for c in cells)
        for k, cell in enumerate(cells):
            dd = celldir(d, cell, legacy)
            os.makedirs(dd, exist_ok=True)
            _save_npz_atomic(os.path.join(dd, "fields.npz"),
                             inputs=np.array(st["inputs"][k]), outputs=np.array(st["outputs"][k]),
                             redelta=np.array(st["redelta"][k]),
                             **{"Δ": cell["dfac"] * s.l / cell["M"], "Δ_factor": cell["dfac"]},
                             visc=s.visc, kernel=cell["kernel"], M=cell["M"],
                             delta_eta=np.nan if cell.get("deta") is None else cell["deta"])
            _save_npz_atomic(os.path.join(dd, "les_meta.npz"),
                             spectra_les=np.array(st["spectra_les"][k]),
                             redelta_mean=float(np.mean(st["redelta"][k])))

    return record, finish


def sfswriter(s, d, times, nles=None, filters=None, cells=None, protectshells=2,
              outtype=lambda M: np.float64):
    """sfswriter(s; dir, times, ...) (src/spectral/les.jl:477-519): a
    spectral_solve processor sampling the bank at `times` (pass them as
    tstops) and writing it after the last one."""
    from . import spectral as S

    sam = S.lessampler(s, nles, filters, cells, protectshells, outtype)
    record, finish = sfscollector(sam, s, d)
    times = sorted(float(t) for t in times)
    inext = [0]

    def proc(state, _s):
        while inext[0] < len(times) and state.t >= times[inext[0]] - 1e-10 * (abs(times[inext[0]]) + 1):
            record(state.t, state.uh)
            inext[0] += 1
            if inext[0] == len(times):
                finish()
        return None

    return proc


def sfs_offline(prefixes, s, d, nles=None, filters=None, cells=None, protectshells=2,
                outtype=lambda M: np.float64, phaseseed=None):
    """sfs_offline(prefixes, s; dir, ..., phaseseed) (src/spectral/les.jl:521-540):
    the bank over stored snapshots, in order; phaseseed applies the phase
    randomisation (the kinematic null) to each snapshot first."""
    from . import spectral as S

    sam = S.lessampler(s, nles, filters, cells, protectshells, outtype)
    record, finish = sfscollector(sam, s, d)
    uh = S.specvelocity(s)
    for prefix in prefixes:
        md = spectral_load(uh, prefix, s)
        if phaseseed is not None:
            S.spectral_phaserandomize(uh, s, seed=phaseseed)
        record(md["time"], uh)
    finish()
