"""Host mirror of the reference's pseudo-spectral solver for a periodic cube
(src/spectral/setup.jl, step.jl, operators.jl, ic.jl), single rank, on
libdnsb's dnsb_spectral_* entry points.

The state `uh` is a complex128 CUDA tensor of shape (3, m, m, kcut+1) —
component, kz, ky, kx in C order, i.e. the reference's column-major
(kcut+1, m, m, 3) compact spectrum with kx fastest — and u_hat = F[u]/n^3.
Physical fields are float64 tensors of shape (3, n, n, n) (component, z, y,
x) at the cell centres (i - 1/2) l / n.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib


class SpectralError(RuntimeError):
    pass


def _ptr(t):
    if not (t.is_cuda and t.is_contiguous() and t.dtype in (torch.float64, torch.complex128)):
        raise ValueError("arrays must be contiguous float64/complex128 CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


class SpectralSetup:
    """spectral_setup(; n, l, visc, kcut) (src/spectral/setup.jl:28-110),
    one rank."""

    def __init__(self, n, l=2 * math.pi, visc=1e-3, kcut=None, device=None):
        if n % 2:
            raise ValueError("n must be even")
        kcut = n // 3 if kcut is None else int(kcut)
        if kcut < 1:
            raise ValueError("kcut must be at least 1")
        if 3 * kcut > n:
            raise ValueError("aliasing: 3kcut <= n is required (2/3 rule)")
        self.n, self.l, self.visc, self.kcut = int(n), float(l), float(visc), kcut
        self.m = 2 * kcut + 1
        self.device = torch.device(device if device is not None else "cuda")
        self.T = torch.float64
        self._sp = None
        lib = _lib.load()
        sp = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            rc = lib.dnsb_spectral_create(self.n, kcut, self.l, self.visc, self.device.index or 0,
                                          ctypes.c_void_p(stream), ctypes.byref(sp))
        if rc != 0:
            raise _lib.DNSBError(f"spectral setup failed: {lib.dnsb_spectral_last_error(None).decode()}")
        self._sp = sp
        kf = 2 * math.pi / self.l
        cf = np.array([j if j <= kcut else j - self.m for j in range(self.m)], dtype=np.float64)
        self.kx, self.ky, self.kz = kf * np.arange(kcut + 1), kf * cf, kf * cf

    @property
    def sp(self):
        if self._sp is None:
            raise RuntimeError("spectral setup has been closed")
        lib = _lib.load()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        self._call(lib.dnsb_spectral_set_stream(self._sp, ctypes.c_void_p(stream)))
        return self._sp

    def _call(self, rc):
        if rc != 0:
            raise _lib.DNSBError(_lib.load().dnsb_spectral_last_error(self._sp).decode())

    def close(self):
        if self._sp is not None:
            _lib.load().dnsb_spectral_destroy(self._sp)
            self._sp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spectral_setup(*, n, l=2 * math.pi, visc=1e-3, kcut=None, device=None):
    return SpectralSetup(n, l, visc, kcut, device)


def specvelocity(s):
    """specvelocity(s): a zero spectral state."""
    return torch.zeros((3, s.m, s.m, s.kcut + 1), dtype=torch.complex128, device=s.device)


def physvelocity(s):
    return torch.zeros((3, s.n, s.n, s.n), dtype=torch.float64, device=s.device)


def spec_to_phys(v, uh, s):
    """spec_to_phys!(v, uh, s): the physical velocity of uh."""
    s._call(_lib.load().dnsb_spectral_to_phys(s.sp, _ptr(uh), _ptr(v)))
    return v


def phys_to_spec(uh, v, s):
    """phys_to_spec!(uh, v, s) with the truncation to the retained modes."""
    s._call(_lib.load().dnsb_spectral_from_phys(s.sp, _ptr(v), _ptr(uh)))
    return uh


def spectral_rhs(du, uh, s):
    """spectral_rhs!(du, uh, s) (src/spectral/operators.jl:66-96)."""
    s._call(_lib.load().dnsb_spectral_rhs(s.sp, _ptr(uh), _ptr(du)))
    return du


def spectral_project(uh, s):
    """spectral_project!(uh, s) (src/spectral/operators.jl:25-29)."""
    s._call(_lib.load().dnsb_spectral_project(s.sp, _ptr(uh)))
    return uh


def spectral_step(uh, s, dt):
    """spectral_step!(uh, s, dt, cache) (src/spectral/step.jl:60-92);
    returns the first stage's vsummax."""
    out = ctypes.c_double()
    s._call(_lib.load().dnsb_spectral_step(s.sp, _ptr(uh), float(dt), ctypes.byref(out)))
    return out.value


def vsummax(uh, s):
    out = ctypes.c_double()
    s._call(_lib.load().dnsb_spectral_vsummax(s.sp, _ptr(uh), ctypes.byref(out)))
    return out.value


def _diag(uh, s, which):
    out = ctypes.c_double()
    s._call(_lib.load().dnsb_spectral_diagnostic(s.sp, _ptr(uh), which, ctypes.byref(out)))
    return out.value


def spectral_energy(uh, s):
    """spectral_energy(uh, s): <|u|^2>/2 (src/spectral/operators.jl:98-99)."""
    return _diag(uh, s, 0)


def spectral_dissipation(uh, s):
    """spectral_dissipation(uh, s): nu sum k^2 |u_hat|^2 (:101-107)."""
    return _diag(uh, s, 1)


def spectral_maxdiv(uh, s):
    """spectral_maxdiv(uh, s): max |k . u_hat| (:109-110)."""
    return _diag(uh, s, 2)


def spectral_velocityfield(uh, s, x, y, z, project=True):
    """spectral_velocityfield!(uh, s; x, y, z, project) (src/spectral/ic.jl:6-25):
    the three functions at the cell centres, forward transformed."""
    c = s.l / s.n * (np.arange(s.n) + 0.5)
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    h = np.stack([np.vectorize(f)(X, Y, Z) if f is not None else np.zeros_like(X)
                  for f in (x, y, z)]).astype(np.float64)
    v = torch.from_numpy(h).to(s.device)
    phys_to_spec(uh, v, s)
    if project:
        spectral_project(uh, s)
    return uh


def taylorgreen(uh, s, V0=1.0):
    """taylorgreen!(uh, s; V0) (src/spectral/ic.jl:86-97)."""
    l = s.l
    return spectral_velocityfield(
        uh, s,
        x=lambda x, y, z: V0 * math.sin(2 * math.pi * x / l) * math.cos(2 * math.pi * y / l)
        * math.cos(2 * math.pi * z / l),
        y=lambda x, y, z: -V0 * math.cos(2 * math.pi * x / l) * math.sin(2 * math.pi * y / l)
        * math.cos(2 * math.pi * z / l),
        z=lambda x, y, z: 0.0)


SpectralState = __import__("collections").namedtuple("SpectralState", "uh t n")


def spectral_solve(*, uh, setup, tlims, dt=None, cfl=0.85, forcing=None, tstops=(), nstart=0,
                   processors=None):
    """spectral_solve!(; uh, setup, tlims, Δt, cfl, forcing, tstops, nstart,
    processors) (src/spectral/step.jl:94-170).  forcing(uh, s) after every
    step; a processor returning "stop" ends the solve after that step."""
    s = setup
    processors = dict(processors or {})
    spectral_project(uh, s)
    kmax = 2 * math.pi * s.kcut / s.l
    eps = np.finfo(np.float64).eps
    vmax = vsummax(uh, s) if dt is None else 0.0
    t, tend = float(tlims[0]), float(tlims[1])
    tol = 1e-10 * (abs(tend) + 1)
    stops = sorted(x for x in tstops if t + tol < x < tend - tol)
    istop = 0
    n = nstart
    stop = False
    state = SpectralState(uh, t, n)
    for proc in processors.values():
        stop |= proc(state, s) == "stop"
    while not stop and t < tend - tol:
        while istop < len(stops) and stops[istop] <= t + tol:
            istop += 1
        tnext = stops[istop] if istop < len(stops) else tend
        dtn = min(dt if dt is not None else cfl * math.sqrt(3) / (kmax * (vmax + eps)), tnext - t)
        vloc = spectral_step(uh, s, dtn)
        if forcing is not None:
            forcing(uh, s)
        if dt is None:
            vmax = vloc
        t += dtn
        n += 1
        state = SpectralState(uh, t, n)
        for proc in processors.values():
            stop |= proc(state, s) == "stop"
    return state


# ----------------------------------------------- shells, random field, forcing
# src/spectral/ic.jl:53-84 and src/spectral/forcing.jl:1-56 on the compact
# state: shell s = the modes with s <= |k_int| < s+1.

def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def shell_count(s):
    """floor(sqrt(3) kcut) + 1: the shells 0..kdiag of spectral_randomfield!."""
    return int(_lib.load().dnsb_spectral_shell_count(s.sp))


def shell_energies(uh, s, shells):
    """shell_energies(uh, s, shells) (src/spectral/forcing.jl:12-24)."""
    shells = [int(v) for v in shells]
    nb = max(shells) + 1
    E = np.zeros(nb)
    s._call(_lib.load().dnsb_spectral_shell_energies(s.sp, _ptr(uh), _dptr(E), nb))
    return np.array([E[v] for v in shells])


def rescale_shell(uh, s, sh, factor):
    """rescale_shell!(uh, s, sh, factor) (src/spectral/forcing.jl:26-35)."""
    f = np.ones(int(sh) + 1)
    f[int(sh)] = factor
    s._call(_lib.load().dnsb_spectral_shell_rescale(s.sp, _ptr(uh), _dptr(f), len(f)))
    return uh


def spectral_randomfield(uh, s, totalenergy=1.0, kpeak=4.0, seed=0, profile=None):
    """spectral_randomfield!(uh, s; totalenergy, kpeak, seed, profile)
    (src/spectral/ic.jl:53-84)."""
    if profile is None:
        prof, ptr, nprof = None, None, 0
    else:
        prof = np.array([profile(k) for k in range(shell_count(s))], dtype=np.float64)
        ptr, nprof = _dptr(prof), len(prof)
    s._call(_lib.load().dnsb_spectral_random_field(s.sp, _ptr(uh), float(totalenergy), float(kpeak),
                                                   int(seed), ptr, nprof))
    return uh


def shellforcing(uh, s, shells=(1, 2), eref=None):
    """shellforcing(uh, s; shells, eref) (src/spectral/forcing.jl:37-56):
    the closure forcing(uh, s) clamps the shells back to eref on the device."""
    shells = [int(v) for v in shells]
    eref = shell_energies(uh, s, shells) if eref is None else np.asarray(eref, dtype=np.float64)
    table = -np.ones(max(shells) + 1)
    for sh, e in zip(shells, eref):
        table[sh] = e

    def forcing(uh2, s2):
        s2._call(_lib.load().dnsb_spectral_shell_clamp(s2.sp, _ptr(uh2), _dptr(table), len(table)))

    forcing.eref = np.array(eref)
    forcing._table = table
    return forcing


# ------------------------------------------- filtered-field / SFS sampling
# sfs_sample! (src/spectral/les.jl:302-370) on the spectral state: the cube
# on the GPU (dnsb_spectral_les_cube), the coarse-grid half on the host
# (les.sfs_from_cube, the reference's rank-0 code).

def les_cube(uh, s, M):
    """The 9 coarse cubes (u_hat x, y, z, sigma_hat xx, yy, zz, xy, yz, zx),
    numpy (9, M, M, M//2+1)."""
    out = np.zeros((9, M, M, M // 2 + 1), dtype=np.complex128)
    s._call(_lib.load().dnsb_spectral_les_cube(s.sp, _ptr(uh), int(M), _dptr(out.view(np.float64))))
    return out


def lessampler(s, nles=None, filters=None, cells=None, protectshells=2,
               outtype=lambda M: np.float64):
    """lessampler(s; nles, filters, cells, protectshells, outtype)
    (src/spectral/les.jl:239-300), one rank."""
    from .les import LES_KERNELS, lescells

    cells = lescells(nles, filters, cells)
    for c in cells:
        if c["M"] % 2:
            raise ValueError(f"coarse grid M must be even (got {c['M']})")
        if c["kernel"] not in LES_KERNELS:
            raise ValueError(f"kernel must be one of {LES_KERNELS}")
        if not c["dfac"] > 0:
            raise ValueError("dfac must be positive")
    Mmax = max(c["M"] for c in cells)
    if Mmax // 2 > s.kcut:
        raise ValueError(f"LES cube needs M/2 <= kcut (M = {Mmax}, kcut = {s.kcut})")
    return dict(cells=cells, nles=Mmax, protectshells=int(protectshells), outtype=outtype, l=s.l)


def sfs_sample(sam, uh, s):
    """sfs_sample!(sam, uh, s): per bank cell dict(ubar, tau, redelta, spectrum)."""
    from .les import sfs_from_cube

    return sfs_from_cube(sam, les_cube(uh, s, sam["nles"]), s.visc)


# ------------------------------------------------------------ statistics

def spectral_stats(uh, s):
    """spectral_stats(uh, s) (src/spectral/stats.jl:5-25): the K41
    statistics of the state (single rank)."""
    visc, n, l = s.visc, s.n, s.l
    e = spectral_energy(uh, s)
    diss = spectral_dissipation(uh, s)
    uavg = math.sqrt(2 * e / 3)
    l_kol = (visc ** 3 / diss) ** 0.25
    l_tay = math.sqrt(15 * visc / diss) * uavg
    l_int = uavg ** 3 / diss
    return dict(e=e, uavg=uavg, diss=diss, l_int=l_int, l_tay=l_tay, l_kol=l_kol,
                t_int=l_int / uavg, t_tay=l_tay / uavg, t_kol=math.sqrt(visc / diss),
                Re_int=l_int * uavg / visc, Re_tay=l_tay * uavg / visc,
                kmax_eta=(math.pi * n / l) * l_kol)


def spectral_spectrum(uh, s):
    """spectral_spectrum(uh, s) (src/spectral/stats.jl:27-36): shells 0..kcut."""
    return dict(k=np.arange(s.kcut + 1), E=shell_energies(uh, s, range(s.kcut + 1)))


def statswriter(file, nupdate=10):
    """statswriter(; file, nupdate) (src/spectral/io.jl:231-262): appends a
    CSV row t, step, the statistics, walltime every nupdate steps."""
    import os
    import time as _time

    def proc(state, s):
        if state.n % nupdate:
            return None
        st = spectral_stats(state.uh, s)
        d = os.path.dirname(os.path.abspath(file))
        os.makedirs(d, exist_ok=True)
        fresh = not os.path.isfile(file) or os.path.getsize(file) == 0
        with open(file, "a") as fh:
            if fresh:
                fh.write(",".join(["t", "step", *st.keys(), "walltime"]) + "\n")
            fh.write(",".join(str(v) for v in (state.t, state.n, *st.values(), _time.time())) + "\n")
        return None

    return proc


def spectral_phaserandomize(uh, s, seed=0):
    """spectral_phaserandomize!(uh, s; seed) (src/spectral/ic.jl:130-143)."""
    s._call(_lib.load().dnsb_spectral_phaserandomize(s.sp, _ptr(uh), int(seed)))
    return uh
