"""Filtered-field / sub-filter-stress sampler and snapshot IO for the FV
state of a periodic box: the dataset generator that feeds LES closure
training.

The reference computes this on its pseudo-spectral state
(src/spectral/les.jl): the distributed half (LES-cube gather of u_hat and
sigma_hat = F[v_i v_j], :313-334) runs on every rank, the rest on rank 0 on
small coarse rfft arrays with plain loops and FFTW (:335-370).  Here the
distributed half is `dnsb_les_cube` (libdnsb: cell-centred velocity, the
six products, the 3-D transforms and the cube extraction on the GPU) and
the coarse-grid half is this module, on the host as in the reference
(numpy FFTs on M^3 arrays).  Coarse arrays have numpy shape (M, M, M//2+1),
i.e. index [kz, ky, kx], the reference's column-major (M/2+1, M, M) rfft
layout; u_hat = F[u]/M^3 on the coarse grid as in the reference.
"""
import ctypes
import json
import math
import os

import numpy as np

from . import _lib
from ._lib import check
from .api import _ptr

LES_KERNELS = ("gaussian", "cutoff", "tophat", "helmholtz")
SIGMA = (("xx", 0, 0), ("yy", 1, 1), ("zz", 2, 2), ("xy", 0, 1), ("yz", 1, 2), ("zx", 2, 0))


def _freqs(n):
    """(kx, ky, kz) integer frequency grids of an (n, n, n//2+1) rfft array:
    lesfreq (src/spectral/les.jl:42) along the wrapped axes."""
    kz = np.fft.fftfreq(n, 1.0 / n).round().astype(np.int64)
    kx = np.arange(n // 2 + 1)
    return kx[None, None, :], kz[None, :, None], kz[:, None, None]


def les_twothirds(a, n):
    """les_twothirds! (src/spectral/les.jl:45-54): zero |k_i| > n//3 and the
    mean (in place)."""
    kx, ky, kz = _freqs(n)
    kc = n // 3
    keep = (kx <= kc) & (np.abs(ky) <= kc) & (np.abs(kz) <= kc) & ~((kx == 0) & (ky == 0) & (kz == 0))
    a *= keep
    return a


def _sinc(x):
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(x == 0, 1.0, np.sin(x) / np.where(x == 0, 1.0, x))


def les_filterkernel(a, n, l, delta, protectshells, kernel):
    """les_filterkernel! (src/spectral/les.jl:59-85): spectral filter of
    width delta, shells |k| < protectshells + 1 (in units of 2 pi / l) left
    untouched (in place)."""
    kf = 2 * math.pi / l
    kx, ky, kz = _freqs(n)
    k1, k2, k3 = kf * kx, kf * ky, kf * kz
    kk = k1 ** 2 + k2 ** 2 + k3 ** 2
    if kernel == "gaussian":
        w = np.exp(-delta ** 2 * kk / 24)
    elif kernel == "cutoff":
        w = np.where(kk <= (math.pi / delta) ** 2, 1.0, 0.0)
    elif kernel == "tophat":
        w = _sinc(k1 * delta / 2) * _sinc(k2 * delta / 2) * _sinc(k3 * delta / 2)
    elif kernel == "helmholtz":
        w = 1 / (1 + delta ** 2 * kk / 24)
    else:
        raise ValueError(f"unknown filter kernel {kernel}")
    w = np.where(kk < (kf * (protectshells + 1)) ** 2, 1.0, w)
    a *= w
    return a


def les_nonlinearity(ub, n):
    """les_nonlinearity! (src/spectral/les.jl:88-101): sigma2[c] =
    F[v_i v_j]/n^3 from the dealiased coarse velocity ub (6 components)."""
    fac = n ** 3
    vs = []
    for i in range(3):
        tmp = les_twothirds(ub[i].copy(), n)
        vs.append(np.fft.irfftn(tmp, s=(n, n, n), axes=(0, 1, 2)) * fac)
    return [np.fft.rfftn(vs[i] * vs[j]) / fac for _, i, j in SIGMA]


def les_filter_reynolds(ub, n, l, visc, delta):
    """les_filter_reynolds (src/spectral/les.jl:104-116)."""
    kf = 2 * math.pi / l
    kx, ky, kz = _freqs(n)
    kk = kf ** 2 * (kx ** 2 + ky ** 2 + kz ** 2)
    u2 = sum(np.abs(c) ** 2 for c in ub)
    w = np.where((kx > 0) & (kx < n // 2), 2.0, 1.0)
    return delta ** 2 * math.sqrt(float(np.sum(w * kk * u2))) / visc


def les_spectrum(ub, n):
    """les_spectrum (src/spectral/les.jl:119-131): shells 1..n//3 by the
    integer square root of |k|^2."""
    kc = n // 3
    kx, ky, kz = _freqs(n)
    s2 = kx ** 2 + ky ** 2 + kz ** 2
    sh = np.floor(np.sqrt(s2.astype(np.float64))).astype(np.int64)
    sh -= sh * sh > s2
    sh += (sh + 1) ** 2 <= s2
    u2 = sum(np.abs(c) ** 2 for c in ub)
    w = np.where((kx > 0) & (kx < n // 2), 2.0, 1.0)
    e = np.broadcast_to(w * u2 / 2, u2.shape)
    sh = np.broadcast_to(sh, u2.shape)
    m = (sh >= 1) & (sh <= kc)
    E = np.zeros(kc)
    np.add.at(E, sh[m] - 1, e[m])
    return E


def les_tracefree(tau):
    """les_tracefree! (src/spectral/les.jl:134-143)."""
    tr = (tau[0] + tau[1] + tau[2]) / 3
    for c in range(3):
        tau[c] = tau[c] - tr
    return tau


def les_extract(src, M, Mmax):
    """les_extract! (src/spectral/les.jl:176-184): the M-cube of a coarse
    array on grid Mmax (wrapped frequencies)."""
    idx = np.r_[0:M // 2, Mmax - M // 2:Mmax]
    return src[np.ix_(idx, idx, np.arange(M // 2 + 1))].copy()


def lescells(nles=None, filters=None, cells=None):
    """lescells (src/spectral/les.jl:188-205)."""
    if cells is None:
        if nles is None or filters is None:
            raise ValueError("pass `cells`, or the legacy `nles` + `filters`")
        cells = [dict(M=nles, kernel="gaussian", dfac=f) for f in filters]
    out = []
    for c in cells:
        c = dict(c)
        out.append(dict(M=int(c["M"]), kernel=str(c.get("kernel", "gaussian")),
                        dfac=float(c.get("dfac", c.get("Δfac"))), deta=c.get("deta")))
    return out


def lessampler(s, nles=None, filters=None, cells=None, protectshells=2, outtype=lambda M: np.float64):
    """lessampler (src/spectral/les.jl:239-300) for a periodic cube: the
    bank cells, checked; the cube is taken once at the largest M."""
    if s.bc != ("periodic",) * 3:
        raise ValueError("the sampler needs a fully periodic box")
    lengths = [b - a for a, b in s.lims]
    if len(set(s.n)) != 1 or max(lengths) - min(lengths) > 1e-12 * max(lengths):
        raise ValueError("the sampler needs a cube (equal n and lengths), as the spectral setup")
    cells = lescells(nles, filters, cells)
    for c in cells:
        if c["M"] % 2:
            raise ValueError(f"coarse grid M must be even (got {c['M']})")
        if c["kernel"] not in LES_KERNELS:
            raise ValueError(f"kernel must be one of {LES_KERNELS}")
        if not c["dfac"] > 0:
            raise ValueError("dfac must be positive")
    Mmax = max(c["M"] for c in cells)
    if Mmax // 2 > s.n[0] // 2:
        raise ValueError(f"LES cube needs M/2 <= n/2 (M = {Mmax}, n = {s.n[0]})")
    return dict(cells=cells, nles=Mmax, protectshells=int(protectshells), outtype=outtype,
                l=lengths[0])


def les_cube(u, s, M):
    """dnsb_les_cube: the 9 coarse arrays (u_hat x, y, z, sigma_hat xx, yy,
    zz, xy, yz, zx) of the cell-centred state, shape (9, M, M, M//2+1)."""
    h = M // 2 + 1
    out = np.zeros((9, M, M, h), dtype=np.complex128)
    ptr = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    check(_lib.load().dnsb_les_cube(s.ctx, _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]), int(M), ptr),
          s._ctx)
    return out


def sfs_from_cube(sam, cube, visc):
    """The rank-0 half of sfs_sample! (src/spectral/les.jl:335-370) on the
    gathered cube: per cell, u_bar = filter(cutoff(u_hat)) dealiased, tau =
    filter(sigma_hat) - F[u_bar_i u_bar_j] dealiased and trace-free, the
    filter Reynolds number and the shell spectrum."""
    nles, ps, l = sam["nles"], sam["protectshells"], sam["l"]
    cubes = {}
    out = []
    for cell in sam["cells"]:
        M, kernel = cell["M"], cell["kernel"]
        if M not in cubes:
            cubes[M] = cube if M == nles else np.stack([les_extract(c, M, nles) for c in cube])
        cb = cubes[M]
        delta = cell["dfac"] * l / M
        ubf = [les_twothirds(les_filterkernel(cb[c].copy(), M, l, delta, ps, kernel), M)
               for c in range(3)]
        tau = [les_filterkernel(cb[3 + c].copy(), M, l, delta, ps, kernel) for c in range(6)]
        s2 = les_nonlinearity(ubf, M)
        tau = les_tracefree([les_twothirds(tau[c] - s2[c], M) for c in range(6)])
        ct = np.dtype(sam["outtype"](M))
        cdt = np.complex64 if ct == np.float32 else np.complex128
        out.append(dict(
            ubar={k: ubf[i].astype(cdt) for i, k in enumerate("xyz")},
            tau={name: tau[i].astype(cdt) for i, (name, _, _) in enumerate(SIGMA)},
            redelta=les_filter_reynolds(ubf, M, l, visc, delta),
            spectrum=les_spectrum(ubf, M),
        ))
    return out


def sfs_sample(sam, u, s):
    """sfs_sample!(sam, uh, s) (src/spectral/les.jl:302-370) on the FV state
    (valid halos): list over sam["cells"] of dict(ubar, tau, redelta,
    spectrum)."""
    return sfs_from_cube(sam, les_cube(u, s, sam["nles"]), s.visc)


# ------------------------------------------------------------ snapshot IO
# After spectral_save / spectral_load! (src/spectral/io.jl:30-104): one raw
# binary file with the fields in the reference's column-major ghosted
# layout and a JSON sidecar with the metadata, both written atomically
# (temporary names, then renamed: the pair is complete or absent).

def save_snapshot(prefix, u, s, p=None, time=0.0, step=0, meta=None):
    """Writes <prefix>.bin (u.x, u.y, u.z[, p], float64 ghosted arrays, x
    fastest) and <prefix>.json; returns prefix."""
    fields = [u["x"], u["y"], u["z"]] + ([p] if p is not None else [])
    datafile, metafile = prefix + ".bin", prefix + ".json"
    with open(datafile + ".tmp", "wb") as fh:
        for f in fields:
            a = f.detach().cpu().numpy() if hasattr(f, "detach") else np.asarray(f)
            fh.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    d = {
        "format": "DistributedNavierStokes FV state",
        "version": 1,
        "eltype": "Float64",
        "n": list(s.n),
        "lims": [list(v) for v in s.lims],
        "bc": list(s.bc),
        "visc": s.visc,
        "time": float(time),
        "step": int(step),
        "fields": ["u.x", "u.y", "u.z"] + (["p"] if p is not None else []),
        "order": "column-major (nx+2, ny+2, nz+2) per field, ghost width 1",
        "data": os.path.basename(datafile),
    }
    if meta:
        d["meta"] = {k: (np.asarray(v).tolist() if not isinstance(v, (int, float, str)) else v)
                     for k, v in dict(meta).items()}
    with open(metafile + ".tmp", "w") as fh:
        json.dump(d, fh, indent=1, sort_keys=True)
    os.replace(metafile + ".tmp", metafile)
    os.replace(datafile + ".tmp", datafile)
    return prefix


def load_snapshot(u, prefix, s, p=None):
    """Loads a save_snapshot pair into u (and p, if stored and given);
    returns dict(time, step, meta).  The grid must match the setup."""
    with open(prefix + ".json") as fh:
        d = json.load(fh)
    if d["eltype"] != "Float64" or tuple(d["n"]) != tuple(s.n) or tuple(d["bc"]) != tuple(s.bc):
        raise ValueError(f"snapshot {prefix} (n {d['n']}, bc {d['bc']}) does not match the setup "
                         f"(n {list(s.n)}, bc {list(s.bc)})")
    size = int(np.prod(s.shape))
    raw = np.fromfile(prefix + ".bin", dtype=np.float64)
    if raw.size != size * len(d["fields"]):
        raise ValueError(f"snapshot {prefix}: data file has {raw.size} values, "
                         f"expected {size * len(d['fields'])}")
    targets = {"u.x": u["x"], "u.y": u["y"], "u.z": u["z"], "p": p}
    for i, name in enumerate(d["fields"]):
        t = targets.get(name)
        if t is None:
            continue
        a = raw[i * size:(i + 1) * size].reshape(s.shape)
        if hasattr(t, "copy_"):
            import torch

            t.copy_(torch.from_numpy(a))
        else:
            t[...] = a
    return dict(time=d["time"], step=d["step"], meta=d.get("meta", {}))
