"""Host-side mirror of the DistributedNavierStokes FV API, on libdnsb.so.

Same names, arguments and semantics as the reference's Julia API for the
single-GPU path (the Julia mutating suffix `!` is dropped):

    reference (src/...)                     here
    setup(; n, lims, bc, stretch, ...)      setup(n=..., lims=..., ...)
    scalarfield / vectorfield               scalarfield / vectorfield
    velocityfield!(u, s; x, y, z)           velocityfield(u, s, x=, y=, z=)
    exchange_halo!(φ, stag, s) / (u, s)     exchange_halo(φ, stag, s) / (u, s)
    divergence!, momentum!, poisson!,       divergence, momentum, poisson,
    pressuregrad_component!/update!,        pressuregrad_component/update,
    project!, imex_update!, step!           project, imex_update, step
    cfl_timestep(u, s; cfl)                 cfl_timestep(u, s, cfl=)
    solve!(; u, setup, tlims, Δt, cfl,      solve(u=, setup=, tlims=, dt=, cfl=,
           processors)                            processors=)
    maxdiv, kinetic_energy, logger          maxdiv, kinetic_energy, logger
    channelstats/channelprofiles,           channelstats/channelprofiles,
    spectrumstats/energyspectrum            spectrumstats/energyspectrum

Fields are torch.float64 CUDA tensors of shape (nz+2, ny+2, nx+2): the
memory of the reference's column-major (nx+2, ny+2, nz+2) ghosted arrays,
x fastest, so `phi[K, J, I]` is the reference's `phi[I+1, J+1, K+1]`.
Every operator runs in libdnsb.so on the tensors' memory; torch is used
only to allocate device memory and to provide the current CUDA stream.
Errors raise like the reference's `error(...)` (src/setup.jl:49-54).
"""
import ctypes
import math
from collections import namedtuple

import numpy as np
import torch

from . import _lib
from ._lib import check

RK3 = {
    "A": (0.0, -5 / 9, -153 / 128),
    "B": (1 / 3, 15 / 16, 8 / 15),
    "alpha": (1 / 3, 5 / 12, 1 / 4),
}
"""Low-storage Williamson RK3 coefficients (src/timestep.jl:10-14)."""

STAG = {"x": 0, "y": 1, "z": 2, "p": 3}

State = namedtuple("State", "u p t n")


class VectorField(dict):
    """(; x, y, z) of ghosted fields; attribute and key access."""

    __getattr__ = dict.__getitem__

    def __iter__(self):
        return iter(("x", "y", "z"))

    def values(self):
        return [self["x"], self["y"], self["z"]]


def _ptr(t):
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise ValueError("fields must be contiguous float64 CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


class Setup:
    """The reference's setup NamedTuple (src/setup.jl:34-113), single rank,
    holding the libdnsb context (plans, coefficient tables, scratch)."""

    def __init__(self, n, lims, bc, stretch, visc, bodyforce, ydiffusion, order, device,
                 tuning=None):
        self.n = tuple(int(v) for v in n)
        self.lims = tuple((float(a), float(b)) for a, b in lims)
        self.bc = tuple(bc)
        self.visc = float(visc)
        self.bodyforce = tuple(float(f) for f in bodyforce)
        self.order = order
        self.w = order // 2
        self.imexy = ydiffusion == "implicit"
        self.epsy = 0.0 if self.imexy else 1.0
        self.rk = RK3
        self.device = torch.device(device)
        self.T = torch.float64
        self.procgrid = (1, 1)
        self._griddata(stretch)
        self.ranges = {c: self.active(c) for c in ("x", "y", "z", "p")}
        self._ctx = None
        lib = _lib.load()
        g = _lib.dnsb_grid()
        g.nx, g.ny, g.nz = self.n
        g.bc_y = 1 if self.wall else 0
        g.ydiffusion = 1 if self.imexy else 0
        g.dx, g.dz = self.dx, self.dz
        self._dy_c = np.ascontiguousarray(self.dy, dtype=np.float64)
        self._dyu_c = np.ascontiguousarray(self.dyu, dtype=np.float64)
        g.dy = self._dy_c.ctypes.data_as(ctypes.c_void_p)
        g.dyu = self._dyu_c.ctypes.data_as(ctypes.c_void_p)
        g.visc = self.visc
        for i in range(3):
            g.bodyforce[i] = self.bodyforce[i]
        self._grid = g  # (with _dy_c, _dyu_c) also describes the setup to an Ensemble
        self._tuning = make_tuning(tuning)
        ctx = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            rc = lib.dnsb_create_tuned(ctypes.byref(g), ctypes.byref(self._tuning),
                                       self.device.index or 0, ctypes.c_void_p(stream),
                                       ctypes.byref(ctx))
        if rc != 0:
            raise _lib.DNSBError(f"setup failed: {lib.dnsb_last_error(None).decode()}")
        self._ctx = ctx
        nx, ny, nz = self.n
        # setup.poisson.r: the real input/output buffer of poisson!
        self.poisson = {"r": torch.zeros((nz, ny, nx), dtype=torch.float64, device=self.device)}

    def tuning(self):
        """The launch shapes in effect (dnsb_get_tuning), as a dict."""
        t = _lib.dnsb_tuning()
        check(_lib.load().dnsb_get_tuning(self.ctx, ctypes.byref(t)), self._ctx)
        return {k: getattr(t, k) for k, _ in _lib.dnsb_tuning._fields_}

    # -------------------------------------------------------------- grid
    def _griddata(self, stretch):
        for k, v in griddata(self.n, self.lims, self.bc, stretch).items():
            setattr(self, k, v)

    def active(self, c):
        """activeranges (src/setup.jl:132-138) as an index (K, J, I)."""
        nx, ny, nz = self.n
        jh = ny - 1 if (c == "y" and self.wall) else ny
        return (slice(1, nz + 1), slice(1, jh + 1), slice(1, nx + 1))

    @property
    def shape(self):
        nx, ny, nz = self.n
        return (nz + 2, ny + 2, nx + 2)

    # ----------------------------------------------------------- context
    @property
    def ctx(self):
        if self._ctx is None:
            raise RuntimeError("setup has been closed")
        lib = _lib.load()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        check(lib.dnsb_set_stream(self._ctx, ctypes.c_void_p(stream)), self._ctx)
        return self._ctx

    def close(self):
        if self._ctx is not None:
            _lib.load().dnsb_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def griddata(n, lims, bc, stretch=None):
    """griddata (src/setup.jl:148-193), single rank, w = 1: uniform x/z
    spacings, y cell widths dy and centre distances dyu over the ghosted
    rows J = 0..ny+1 (mirrored at walls, wrapped when periodic), the
    smallest interior dy and the face/centre coordinate vectors."""
    nx, ny, nz = n
    (x0, x1), (y0, y1), (z0, z1) = lims
    Lx, Ly, Lz = x1 - x0, y1 - y0, z1 - z0
    wall = bc[1] == "wall"
    stretch = stretch or (lambda t: t)
    yf = np.array([y0 + Ly * stretch(j / ny) for j in range(ny + 1)], dtype=np.float64)
    yfe = np.zeros(ny + 3)
    yfe[1:ny + 2] = yf
    if not wall:
        yfe[0] = yf[0] - (yf[ny] - yf[ny - 1])
        yfe[ny + 2] = yf[ny] + (yf[1] - yf[0])
    else:
        yfe[0] = 2 * yf[0] - yf[1]
        yfe[ny + 2] = 2 * yf[ny] - yf[ny - 1]
    dye = yfe[1:] - yfe[:-1]
    yce = (yfe[:-1] + yfe[1:]) / 2
    dyue = np.concatenate([yce[1:] - yce[:-1], dye[-1:]])
    return dict(
        wall=wall, dx=Lx / nx, dz=Lz / nz, dy=dye, dyu=dyue,
        dymin=float(np.min(dye[1:ny + 1])),
        xf=np.array([x0 + i * Lx / nx for i in range(1, nx + 1)]),
        xc=np.array([x0 + (i - 0.5) * Lx / nx for i in range(1, nx + 1)]),
        zf=np.array([z0 + k * Lz / nz for k in range(1, nz + 1)]),
        zc=np.array([z0 + (k - 0.5) * Lz / nz for k in range(1, nz + 1)]),
        yf=yfe[2:ny + 2], yc=yce[1:ny + 1], ycg=yce[1:ny + 1], yfg=yf,
    )


def make_tuning(tuning):
    """dnsb_tuning from a dict of its fields (missing / None: 0 = default)."""
    t = _lib.dnsb_tuning()
    for k, v in dict(tuning or {}).items():
        if k not in dict(_lib.dnsb_tuning._fields_):
            raise ValueError(f"unknown tuning field {k}")
        setattr(t, k, int(v or 0))
    return t


def setup(*, n, lims=((0.0, 2 * math.pi),) * 3, bc=("periodic", "periodic", "periodic"),
          stretch=None, visc=1e-3, bodyforce=(0.0, 0.0, 0.0), procgrid=None,
          ydiffusion="explicit", mpibuf="auto", order=2, device=None, T=torch.float64,
          tuning=None):
    """setup(; n, kwargs...) (src/setup.jl:34-113) on one GPU.  `tuning` (not
    in the reference): launch shapes, a dict of dnsb_tuning fields."""
    bc = tuple(b.lstrip(":") if isinstance(b, str) else b for b in bc)
    if not (bc[0] == bc[2] == "periodic"):
        raise ValueError("x and z must be periodic")
    if bc[1] not in ("periodic", "wall"):
        raise ValueError("bc[2] must be :periodic or :wall")
    if ydiffusion not in ("explicit", "implicit"):
        raise ValueError("ydiffusion must be :explicit or :implicit")
    if mpibuf not in ("auto", "device", "host"):
        raise ValueError("mpibuf must be :auto, :device, or :host")
    if order != 2:
        raise ValueError("only order 2 is implemented so far")
    if T not in (torch.float64, "float64", np.float64):
        raise ValueError("the FV step computes in Float64")
    if procgrid not in (None, (1, 1)):
        raise ValueError("this build runs one rank per GPU; procgrid must be (1, 1)")
    if ydiffusion == "implicit" and bc[1] != "wall":
        raise ValueError("implicit y-diffusion requires bc[2] == :wall")
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    return Setup(n, lims, bc, stretch, visc, bodyforce, ydiffusion, order, device, tuning)


# ----------------------------------------------------------------- fields

def scalarfield(s):
    """Ghosted scalar field of zeros (src/fields.jl:4-5)."""
    return torch.zeros(s.shape, dtype=torch.float64, device=s.device)


def vectorfield(s):
    """Ghosted velocity field (; x, y, z) of zeros (src/fields.jl:8-9)."""
    return VectorField(x=scalarfield(s), y=scalarfield(s), z=scalarfield(s))


def interior(phi, w=1):
    """Interior (ghost-free) view (src/timestep.jl:17)."""
    return phi[w:-w, w:-w, w:-w]


def _eval_component(f, cx, cy, cz):
    X, Y, Z = np.meshgrid(cx, cy, cz, indexing="ij")
    try:
        v = np.asarray(f(X, Y, Z), dtype=np.float64)
        if v.shape == X.shape:
            return v
        return np.broadcast_to(v, X.shape).copy()
    except Exception:
        out = np.empty(X.shape)
        for i in range(len(cx)):
            for j in range(len(cy)):
                for k in range(len(cz)):
                    out[i, j, k] = f(cx[i], cy[j], cz[k])
        return out


def velocityfield(u, s, x=None, y=None, z=None):
    """velocityfield! (src/fields.jl:28-35): components from functions of
    the staggered coordinates, on active DOFs only, then halos.  Functions
    may be numpy-vectorised (called once on coordinate arrays) or scalar."""
    coords = {"x": (s.xf, s.yc, s.zc), "y": (s.xc, s.yf, s.zc), "z": (s.xc, s.yc, s.zf)}
    for c, f in (("x", x), ("y", y), ("z", z)):
        if f is None:
            continue
        cx, cy, cz = coords[c]
        sl = s.active(c)
        nj = sl[1].stop - 1
        v = _eval_component(f, cx, cy[:nj], cz)  # (nx, nj, nz)
        h = np.zeros(s.shape)
        h[sl] = np.transpose(v, (2, 1, 0))
        u[c].copy_(torch.from_numpy(h))
    exchange_halo(u, s)
    return u


def noise(phi, c, s, seed=0, amp=1.0):
    """Add amp*(2U-1) counter-based splitmix64 noise on the active DOFs of
    component c (channel initial conditions; see include/dnsb.h)."""
    check(_lib.load().dnsb_noise(s.ctx, _ptr(phi), STAG[c], int(seed), float(amp)), s._ctx)
    return phi


# ----------------------------------------------- wavenumber shells (periodic)
# Finite-volume counterparts of the reference's pseudo-spectral random
# initial condition and shell-clamp forcing (src/spectral/ic.jl:53-84,
# src/spectral/forcing.jl:1-56).  Shell s = modes with s <= |k| < s+1.

def _dbuf(values):
    a = np.ascontiguousarray(values, dtype=np.float64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _u3(u):
    return _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"])


def shell_count(s):
    """Number of integer shells of a periodic box (floor(|k|max) + 1)."""
    return int(_lib.load().dnsb_shell_count(s.ctx))


def shell_energies(u, s, shells):
    """shell_energies(uh, s, shells) (src/spectral/forcing.jl:12-24)."""
    shells = [int(v) for v in shells]
    nb = max(shells) + 1 if shells else 1
    E, ptr = _dbuf(np.zeros(nb))
    check(_lib.load().dnsb_shell_energies(s.ctx, *_u3(u), ptr, nb), s._ctx)
    return np.array([E[v] for v in shells])


def rescale_shell(u, s, sh, factor):
    """rescale_shell!(uh, s, sh, factor) (src/spectral/forcing.jl:26-35)."""
    f = np.ones(int(sh) + 1)
    f[int(sh)] = factor
    f, ptr = _dbuf(f)
    check(_lib.load().dnsb_shell_rescale(s.ctx, *_u3(u), ptr, len(f)), s._ctx)
    return u


def random_field(u, s, totalenergy=1.0, kpeak=4.0, seed=0, profile=None):
    """spectral_randomfield!(uh, s; totalenergy, kpeak, seed, profile)
    (src/spectral/ic.jl:53-84) on the staggered velocity of a periodic box:
    Gaussian counter-based noise, FV projection, shells rescaled to the
    profile (default k^4 exp(-2 (k/kpeak)^2))."""
    lib = _lib.load()
    if profile is None:
        ptr, nprof = None, 0
    else:
        prof, ptr = _dbuf([profile(k) for k in range(shell_count(s))])
        nprof = len(prof)
    check(lib.dnsb_random_field(s.ctx, *_u3(u), float(totalenergy), float(kpeak), int(seed),
                                ptr, nprof), s._ctx)
    return u


def shellforcing(u, s, shells=(1, 2), eref=None):
    """shellforcing(uh, s; shells, eref) (src/spectral/forcing.jl:37-56):
    records the energies of `shells` (or takes `eref`) and returns the
    closure forcing(u, s) that clamps them back, entirely on the device."""
    shells = [int(v) for v in shells]
    eref = shell_energies(u, s, shells) if eref is None else np.asarray(eref, dtype=np.float64)
    table = -np.ones(max(shells) + 1)
    for sh, e in zip(shells, eref):
        table[sh] = e
    table, ptr = _dbuf(table)

    def forcing(u2, s2):
        check(_lib.load().dnsb_shell_clamp(s2.ctx, *_u3(u2), ptr, len(table)), s2._ctx)

    forcing.eref = np.array(eref)
    forcing._table = table
    return forcing


# -------------------------------------------------------------- operators

def exchange_halo(phi, stag, s=None):
    """exchange_halo!(φ, stag, setup) or exchange_halo!(u, setup)
    (src/halo.jl:81-133), single rank."""
    lib = _lib.load()
    if isinstance(phi, dict):
        s = stag
        for c in ("x", "y", "z"):
            check(lib.dnsb_fill_ghosts(s.ctx, _ptr(phi[c]), STAG[c]), s._ctx)
        return phi
    check(lib.dnsb_fill_ghosts(s.ctx, _ptr(phi), STAG[stag]), s._ctx)
    return phi


def divergence(r, u, s):
    """divergence!(r, u, setup) (src/operators.jl:29-42)."""
    check(_lib.load().dnsb_divergence(s.ctx, _ptr(r), _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"])),
          s._ctx)
    return r


def momentum(q, u, A, dt, s):
    """momentum!(q, u, A, Δt, setup) (src/operators.jl:155-178)."""
    check(_lib.load().dnsb_momentum(s.ctx, _ptr(q["x"]), _ptr(q["y"]), _ptr(q["z"]),
                                    _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]),
                                    float(A), float(dt)), s._ctx)
    return q


def pressuregrad_component(phi, p, c, scale, s):
    """pressuregrad_component!(φ, p, c, s, setup) (src/operators.jl:204-216)."""
    check(_lib.load().dnsb_pressuregrad(s.ctx, _ptr(phi), _ptr(p), STAG[c], float(scale)),
          s._ctx)
    return phi


def pressuregrad_update(u, p, s):
    """pressuregrad_update! (src/operators.jl:219-220)."""
    for c in ("x", "y", "z"):
        pressuregrad_component(u[c], p, c, 1.0, s)
    return u


def poisson(p, s):
    """poisson!(p, setup) (src/poisson.jl:147-161): solves with the
    right-hand side in s.poisson["r"], writes the interior of p."""
    check(_lib.load().dnsb_poisson(s.ctx, _ptr(s.poisson["r"]), _ptr(p)), s._ctx)
    return p


def project(u, psi, s):
    """project!(u, ψ, setup) (src/timestep.jl:25-31)."""
    check(_lib.load().dnsb_project(s.ctx, _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]), _ptr(psi)),
          s._ctx)
    return u


def imex_update(u, q, p, B, alpha, dt, s):
    """imex_update!(u, q, p, B, α, Δt, setup) (src/ydiffusion.jl:119-154)."""
    check(_lib.load().dnsb_imex_update(s.ctx, _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]),
                                       _ptr(q["x"]), _ptr(q["y"]), _ptr(q["z"]), _ptr(p),
                                       float(B), float(alpha), float(dt)), s._ctx)
    return u


def step(u, p, q, delta, s, dt):
    """step!(u, p, q, δ, setup, Δt) (src/timestep.jl:41-63)."""
    d = delta if delta is not None else p
    check(_lib.load().dnsb_step(s.ctx, _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]), _ptr(p),
                                _ptr(q["x"]), _ptr(q["y"]), _ptr(q["z"]), _ptr(d), float(dt)),
          s._ctx)
    return u


class Ensemble:
    """A batched ensemble of independent setups (no counterpart in the
    reference: periodic boxes of uneven sizes and viscosities).  run() advances every member nsteps RK3 steps of a fixed
    step in one launch of a CUDA graph (a conditional while loop over one
    step of all members, member branches concurrent; captured once); the
    result equals stepping each member alone with step().  Members take the
    launch shapes of their setups (setup(..., tuning=...))."""

    def __init__(self, setups):
        self.setups = list(setups)
        if not self.setups:
            raise ValueError("an ensemble needs at least one setup")
        dev = self.setups[0].device
        if any(s.device != dev for s in self.setups):
            raise ValueError("all members must live on the same device")
        self.device = dev
        lib = _lib.load()
        grids = (_lib.dnsb_grid * len(self.setups))(*[s._grid for s in self.setups])
        # each member takes its setup's launch shapes
        tunings = (_lib.dnsb_tuning * len(self.setups))(*[s._tuning for s in self.setups])
        ens = ctypes.c_void_p()
        with torch.cuda.device(dev):
            stream = torch.cuda.current_stream(dev).cuda_stream
            rc = lib.dnsb_ensemble_create_tuned(len(self.setups), grids, tunings, dev.index or 0,
                                                ctypes.c_void_p(stream), ctypes.byref(ens))
        if rc != 0:
            raise _lib.DNSBError(f"ensemble failed: {lib.dnsb_ensemble_last_error(None).decode()}")
        self._ens = ens

    def run(self, states, dts, nsteps):
        """states[i] = (u, p, q, delta) of member i (delta None when explicit)."""
        if len(states) != len(self.setups) or len(dts) != len(self.setups):
            raise ValueError("one state and one dt per member")
        ptrs = []
        for (u, p, q, delta), s in zip(states, self.setups):
            if s.imexy and delta is None:
                raise ValueError("semi-implicit members need a delta field")
            ptrs += [_ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]), _ptr(p), _ptr(q["x"]),
                     _ptr(q["y"]), _ptr(q["z"]), _ptr(delta) if delta is not None else None]
        arr = (ctypes.c_void_p * len(ptrs))(*[x.value if x is not None else None for x in ptrs])
        d = (ctypes.c_double * len(dts))(*[float(x) for x in dts])
        lib = _lib.load()
        rc = lib.dnsb_ensemble_run(self._ens, arr, d, int(nsteps))
        if rc != 0:
            raise _lib.DNSBError(lib.dnsb_ensemble_last_error(self._ens).decode())
        return states

    def set_forcing(self, i, forcing):
        """Applies the shell-clamp forcing `forcing` (from shellforcing(u, s)
        on member i's setup) to member i after each of its steps, inside the
        graph; None removes it."""
        lib = _lib.load()
        if forcing is None:
            rc = lib.dnsb_ensemble_forcing(self._ens, int(i), None, 0)
        else:
            table = forcing._table
            rc = lib.dnsb_ensemble_forcing(self._ens, int(i),
                                           table.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                           len(table))
        if rc != 0:
            raise _lib.DNSBError(lib.dnsb_ensemble_last_error(self._ens).decode())

    def close(self):
        if getattr(self, "_ens", None) is not None:
            _lib.load().dnsb_ensemble_destroy(self._ens)
            self._ens = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cfl_timestep(u, s, cfl=0.5, use_step_max=False):
    """cfl_timestep(u, setup; cfl) (src/timestep.jl:69-80)."""
    out = ctypes.c_double()
    check(_lib.load().dnsb_cfl(s.ctx, _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]), float(cfl),
                               int(bool(use_step_max)), ctypes.byref(out)), s._ctx)
    return out.value


def maxdiv(u, s):
    """maxdiv(u, setup) (src/fields.jl:38-42)."""
    out = ctypes.c_double()
    check(_lib.load().dnsb_maxdiv(s.ctx, _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]),
                                  ctypes.byref(out)), s._ctx)
    return out.value


def kinetic_energy(u, s):
    """kinetic_energy(u, setup) (src/fields.jl:45-60)."""
    out = ctypes.c_double()
    check(_lib.load().dnsb_kinetic_energy(s.ctx, _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]),
                                          ctypes.byref(out)), s._ctx)
    return out.value


def solve(*, u, setup, tlims, dt=None, cfl=0.5, processors=None, max_steps=None, forcing=None):
    """solve!(; u, setup, tlims, Δt, cfl, processors) (src/timestep.jl:92-111).

    Each processor is called as proc(state, setup) after every step (and
    once initially) with state = State(u, p, t, n).  Returns the final state.
    `max_steps` (not in the reference) stops the loop after that many steps.
    `forcing(u, setup)` is applied after every step, before the processors,
    as the spectral solver's hook (src/spectral/step.jl:109,162).
    """
    s = setup
    processors = dict(processors or {})
    p = scalarfield(s)
    q = vectorfield(s)
    delta = scalarfield(s) if s.imexy else p
    exchange_halo(u, s)
    project(u, delta, s)
    t, tend = float(tlims[0]), float(tlims[1])
    n = 0
    state = State(u, p, t, n)
    for proc in processors.values():
        proc(state, s)
    stepped = False
    while t < tend - 1e-10 * (abs(tend) + 1):
        if max_steps is not None and n >= max_steps:
            break
        if dt is None:
            dtn = cfl_timestep(u, s, cfl, use_step_max=stepped and not processors and forcing is None)
        else:
            dtn = dt
        dtn = min(dtn, tend - t)
        step(u, p, q, delta, s, dtn)
        if forcing is not None:
            forcing(u, s)
        stepped = True
        t += dtn
        n += 1
        state = State(u, p, t, n)
        for proc in processors.values():
            proc(state, s)
    return state


def logger(nupdate=1):
    """logger (src/fields.jl:63-68)."""
    def proc(state, s):
        if state.n % nupdate == 0:
            print(f"n = {state.n:6d}  t = {state.t:10.6g}")
    return proc


# ------------------------------------------------------------------ stats

class _Acc(dict):
    __getattr__ = dict.__getitem__


def channelstats(s, nupdate=1):
    """channelstats(setup; nupdate) (src/stats.jl:15-37): plane sums are
    accumulated on the device by libdnsb (dnsb_channel_sample)."""
    ny = s.n[1]
    nf = ny - 1 if s.wall else ny
    acc = _Acc(nsamples=[0], acc=torch.zeros(4 * ny + 4 * nf, dtype=torch.float64, device=s.device),
               ny=ny, nf=nf)

    def sample(state, s2):
        if state.n % nupdate == 0:
            u = state.u
            check(_lib.load().dnsb_channel_sample(s2.ctx, _ptr(u["x"]), _ptr(u["y"]), _ptr(u["z"]),
                                                  _ptr(acc["acc"])), s2._ctx)
            acc["nsamples"][0] += 1

    acc["sample"] = sample
    return acc


def channelprofiles(cs, s):
    """channelprofiles(cs, setup) (src/stats.jl:65-98), one rank."""
    nx, ny, nz = s.n
    nf = cs["nf"]
    ns = cs["nsamples"][0]
    a = cs["acc"].cpu().numpy() / (max(ns, 1) * nx * nz)
    Uc, Wc, uuc, wwc = a[0:ny], a[ny:2 * ny], a[2 * ny:3 * ny], a[3 * ny:4 * ny]
    o = 4 * ny
    Vf, vvf, Uf, uvf = a[o:o + nf], a[o + nf:o + 2 * nf], a[o + 2 * nf:o + 3 * nf], a[o + 3 * nf:]
    return _Acc(y=s.ycg.copy(), yf=s.yfg[1:ny] if s.wall else s.yfg[1:ny + 1],
                U=Uc, V=Vf, W=Wc, uu=uuc - Uc ** 2, vv=vvf - Vf ** 2, ww=wwc - Wc ** 2,
                uv=uvf - Uf * Vf, nsamples=ns)


def spectrumstats(s, nupdate=1):
    """spectrumstats(setup; nupdate) (src/stats.jl:108-118)."""
    if s.bc != ("periodic", "periodic", "periodic"):
        raise ValueError("spectra require a fully periodic box")
    nbins = math.ceil(math.sqrt(sum((v // 2) ** 2 for v in s.n))) + 1
    acc = _Acc(nsamples=[0], E=torch.zeros(nbins, dtype=torch.float64, device=s.device))

    def sample(state, s2):
        if state.n % nupdate == 0:
            u = state.u
            check(_lib.load().dnsb_spectrum_sample(s2.ctx, _ptr(u["x"]), _ptr(u["y"]),
                                                   _ptr(u["z"]), _ptr(acc["E"]), nbins), s2._ctx)
            acc["nsamples"][0] += 1

    acc["sample"] = sample
    return acc


def energyspectrum(sp, s):
    """energyspectrum(sp, setup) (src/stats.jl:164-167): (κ, E)."""
    E = sp["E"].cpu().numpy() / max(sp["nsamples"][0], 1)
    return _Acc(k=np.arange(len(E)), E=E)
