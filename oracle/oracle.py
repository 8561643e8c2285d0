"""CPU oracle for the finite-volume step -- TEST INFRASTRUCTURE ONLY.

ctypes front end of ``libdnsoracle.so`` (oracle/dns_oracle.c), a plain-C
restatement of the single-rank FV path of DistributedNavierStokes (Julia).
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module; the product package never does.

The Python part restates the host side of the reference that the C part
needs: the ``setup`` keywords (src/setup.jl:34-113), the y-face
distribution ``yface(j) = y0 + Ly*stretch(j/ny)`` (src/setup.jl:155), the
face/centre coordinate vectors (src/setup.jl:182-187), ``velocityfield!``
(src/fields.jl:28-35), ``solve!`` (src/timestep.jl:92-111), ``channelstats``
/ ``channelprofiles`` (src/stats.jl:15-98) and ``spectrumstats`` /
``energyspectrum`` (src/stats.jl:108-167).

Fields are numpy float64 arrays of shape (nz+2, ny+2, nx+2) (C order), i.e.
the reference's column-major (nx+2, ny+2, nz+2) ghosted arrays with x
fastest; ``phi[K, J, I]`` is the reference's ``phi[I+1, J+1, K+1]``.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

STAG = {"x": 0, "y": 1, "z": 2, "p": 3}
RK3 = {
    "A": (0.0, -5 / 9, -153 / 128),
    "B": (1 / 3, 15 / 16, 8 / 15),
    "alpha": (1 / 3, 5 / 12, 1 / 4),
}


def build():
    """Compile libdnsoracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libdnsoracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        d = ctypes.c_double
        P = ctypes.c_void_p
        i = ctypes.c_int
        L.dnso_create.restype = P
        L.dnso_create.argtypes = [i, i, i, i, i, d, d, P, d, d, d, d]
        L.dnso_destroy.argtypes = [P]
        L.dnso_set_threads.argtypes = [i]
        L.dnso_grid.argtypes = [P, P, P, P, P, P]
        L.dnso_poisson_coeffs.argtypes = [P] * 7
        L.dnso_ydiff_coeffs.argtypes = [P] * 7
        L.dnso_fill_halo.argtypes = [P, P, i]
        L.dnso_divergence.argtypes = [P, P, P, P, P]
        L.dnso_momentum.argtypes = [P, P, P, P, P, P, P, d, d]
        L.dnso_pressuregrad.argtypes = [P, P, P, i, d]
        L.dnso_poisson.argtypes = [P, P, P]
        L.dnso_project.argtypes = [P, P, P, P, P]
        L.dnso_imex_update.argtypes = [P, P, P, P, P, P, P, P, d, d, d]
        L.dnso_step.argtypes = [P, P, P, P, P, P, P, P, P, d]
        L.dnso_cfl.restype = d
        L.dnso_cfl.argtypes = [P, P, P, P, d]
        L.dnso_maxdiv.restype = d
        L.dnso_maxdiv.argtypes = [P, P, P, P]
        L.dnso_kinetic_energy.restype = d
        L.dnso_kinetic_energy.argtypes = [P, P, P, P]
        L.dnso_channel_sample.argtypes = [P, P, P, P, P]
        L.dnso_spectrum_sample.argtypes = [P, P, P, P, P, i]
        L.dnso_cfft.argtypes = [i, i, i, P]
        L.dnso_rfft.argtypes = [i, i, P, P]
        L.dnso_irfft.argtypes = [i, i, P, P]
        L.dnso_noise.argtypes = [P, P, i, ctypes.c_ulonglong, d]
        _LIB = L
    return _LIB


def _p(a):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


def tanhstretch(beta):
    """test/serialtests.jl:4"""
    return lambda t: (math.tanh(beta * (2 * t - 1)) / math.tanh(beta) + 1) / 2


def set_threads(n):
    lib().dnso_set_threads(int(n))


class Setup:
    """Oracle counterpart of ``setup(; ...)`` (src/setup.jl:34-113), single rank."""

    def __init__(self, n, lims=((0.0, 2 * math.pi),) * 3,
                 bc=("periodic", "periodic", "periodic"), stretch=None,
                 visc=1e-3, bodyforce=(0.0, 0.0, 0.0), ydiffusion="explicit"):
        if not (bc[0] == bc[2] == "periodic"):
            raise ValueError("x and z must be periodic")
        if bc[1] not in ("periodic", "wall"):
            raise ValueError("bc[2] must be :periodic or :wall")
        if ydiffusion not in ("explicit", "implicit"):
            raise ValueError("ydiffusion must be :explicit or :implicit")
        self.n = tuple(int(v) for v in n)
        nx, ny, nz = self.n
        self.lims = tuple((float(a), float(b)) for a, b in lims)
        self.bc = tuple(bc)
        self.wall = bc[1] == "wall"
        self.imexy = ydiffusion == "implicit"
        self.visc = float(visc)
        self.bodyforce = tuple(float(f) for f in bodyforce)
        stretch = stretch or (lambda t: t)
        Lx, Ly, Lz = (b - a for a, b in self.lims)
        y0 = self.lims[1][0]
        # yface(j) = lims[2][1] + Ly * stretch(j / ny)  (src/setup.jl:155)
        self.yfaces = np.array([y0 + Ly * stretch(j / ny) for j in range(ny + 1)])
        ptr = lib().dnso_create(nx, ny, nz, int(self.wall), int(self.imexy), Lx, Lz,
                                _p(self.yfaces), self.visc, *self.bodyforce)
        if not ptr:
            raise ValueError("invalid configuration")
        self._h = ctypes.c_void_p(ptr)
        dx, dz, dymin = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self.dy = np.zeros(ny + 2)
        self.dyu = np.zeros(ny + 2)
        lib().dnso_grid(self._h, ctypes.byref(dx), ctypes.byref(dz), _p(self.dy),
                        _p(self.dyu), ctypes.byref(dymin))
        self.dx, self.dz, self.dymin = dx.value, dz.value, dymin.value
        # coordinates (src/setup.jl:182-187), global == local on one rank
        self.xf = np.array([self.lims[0][0] + i * Lx / nx for i in range(1, nx + 1)])
        self.xc = np.array([self.lims[0][0] + (i - 0.5) * Lx / nx for i in range(1, nx + 1)])
        self.zf = np.array([self.lims[2][0] + k * Lz / nz for k in range(1, nz + 1)])
        self.zc = np.array([self.lims[2][0] + (k - 0.5) * Lz / nz for k in range(1, nz + 1)])
        yfe = np.zeros(ny + 3)
        yfe[1:ny + 2] = self.yfaces
        if self.wall:
            yfe[0] = 2 * self.yfaces[0] - self.yfaces[1]
            yfe[ny + 2] = 2 * self.yfaces[ny] - self.yfaces[ny - 1]
        else:
            yfe[0] = self.yfaces[0] - (self.yfaces[ny] - self.yfaces[ny - 1])
            yfe[ny + 2] = self.yfaces[ny] + (self.yfaces[1] - self.yfaces[0])
        yce = (yfe[:-1] + yfe[1:]) / 2
        self.yf = yfe[2:ny + 2]          # faces 1..ny
        self.yc = yce[1:ny + 1]          # centres 1..ny
        self.jymax = ny - 1 if self.wall else ny

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _LIB is not None:
            _LIB.dnso_destroy(h)
            self._h = None

    # ------------------------------------------------------------ fields
    @property
    def shape(self):
        nx, ny, nz = self.n
        return (nz + 2, ny + 2, nx + 2)

    def scalarfield(self):
        return np.zeros(self.shape)

    def vectorfield(self):
        return {c: self.scalarfield() for c in "xyz"}

    def active(self, c):
        """ranges[c] (src/setup.jl:132-138) as a numpy index (K, J, I)."""
        nx, ny, nz = self.n
        jh = ny - 1 if (c == "y" and self.wall) else ny
        return (slice(1, nz + 1), slice(1, jh + 1), slice(1, nx + 1))

    def interior(self, phi):
        return phi[1:-1, 1:-1, 1:-1]

    def velocityfield(self, u, x=None, y=None, z=None):
        """velocityfield! (src/fields.jl:28-35)"""
        coords = {"x": (self.xf, self.yc, self.zc), "y": (self.xc, self.yf, self.zc),
                  "z": (self.xc, self.yc, self.zf)}
        for c, f in (("x", x), ("y", y), ("z", z)):
            if f is None:
                continue
            cx, cy, cz = coords[c]
            sl = self.active(c)
            nk = sl[0].stop - 1
            nj = sl[1].stop - 1
            ni = sl[2].stop - 1
            h = np.zeros(self.shape)
            for k in range(nk):
                for j in range(nj):
                    for i in range(ni):
                        h[k + 1, j + 1, i + 1] = f(cx[i], cy[j], cz[k])
            u[c][...] = h
        self.exchange_halo(u)
        return u

    # --------------------------------------------------------- operators
    def fill_halo(self, phi, stag):
        lib().dnso_fill_halo(self._h, _p(phi), STAG[stag])

    def exchange_halo(self, u):
        for c in "xyz":
            self.fill_halo(u[c], c)

    def divergence(self, u, r=None):
        nx, ny, nz = self.n
        if r is None:
            r = np.zeros((nz, ny, nx))
        lib().dnso_divergence(self._h, _p(u["x"]), _p(u["y"]), _p(u["z"]), _p(r))
        return r

    def momentum(self, q, u, A, dt):
        lib().dnso_momentum(self._h, _p(q["x"]), _p(q["y"]), _p(q["z"]),
                            _p(u["x"]), _p(u["y"]), _p(u["z"]), float(A), float(dt))

    def pressuregrad_component(self, phi, p, c, s):
        lib().dnso_pressuregrad(self._h, _p(phi), _p(p), STAG[c], float(s))

    def pressuregrad_update(self, u, p):
        for c in "xyz":
            self.pressuregrad_component(u[c], p, c, 1.0)

    def poisson(self, r, p):
        lib().dnso_poisson(self._h, _p(np.ascontiguousarray(r)), _p(p))

    def project(self, u, psi):
        lib().dnso_project(self._h, _p(u["x"]), _p(u["y"]), _p(u["z"]), _p(psi))

    def imex_update(self, u, q, p, B, alpha, dt):
        lib().dnso_imex_update(self._h, _p(u["x"]), _p(u["y"]), _p(u["z"]),
                               _p(q["x"]), _p(q["y"]), _p(q["z"]), _p(p),
                               float(B), float(alpha), float(dt))

    def step(self, u, p, q, delta, dt):
        lib().dnso_step(self._h, _p(u["x"]), _p(u["y"]), _p(u["z"]), _p(p),
                        _p(q["x"]), _p(q["y"]), _p(q["z"]), _p(delta), float(dt))

    def cfl_timestep(self, u, cfl):
        return lib().dnso_cfl(self._h, _p(u["x"]), _p(u["y"]), _p(u["z"]), float(cfl))

    def maxdiv(self, u):
        return lib().dnso_maxdiv(self._h, _p(u["x"]), _p(u["y"]), _p(u["z"]))

    def kinetic_energy(self, u):
        return lib().dnso_kinetic_energy(self._h, _p(u["x"]), _p(u["y"]), _p(u["z"]))

    def noise(self, phi, c, seed, amp):
        lib().dnso_noise(self._h, _p(phi), STAG[c], int(seed), float(amp))

    def solve(self, u, tlims, dt=None, cfl=0.5, processors=(), max_steps=None, forcing=None):
        """solve! (src/timestep.jl:92-111); returns (p, t, n).  forcing(u) is
        applied after every step, as spectral_solve! does (src/spectral/step.jl:162)."""
        p = self.scalarfield()
        q = self.vectorfield()
        delta = self.scalarfield() if self.imexy else p
        self.exchange_halo(u)
        self.project(u, delta)
        t, tend = float(tlims[0]), float(tlims[1])
        n = 0
        for proc in processors:
            proc(u, p, t, n)
        while t < tend - 1e-10 * (abs(tend) + 1):
            if max_steps is not None and n >= max_steps:
                break
            dtn = min(dt if dt is not None else self.cfl_timestep(u, cfl), tend - t)
            self.step(u, p, q, delta, dtn)
            if forcing is not None:
                forcing(u)
            t += dtn
            n += 1
            for proc in processors:
                proc(u, p, t, n)
        return p, t, n

    # ------------------------------------------- wavenumber shells (numpy)
    # FV restatement of the pseudo-spectral random initial condition and
    # shell-clamp forcing (src/spectral/ic.jl:37-84,
    # src/spectral/forcing.jl:1-56) on a fully periodic box.  Every velocity
    # component is transformed on its own staggered grid with a full 3-D
    # FFT, so no rfft double-counting weights are needed.

    def gauss_noise(self, phi, c, seed):
        """noise_kernel! (src/spectral/ic.jl:37-51): Box-Muller of two
        splitmix64 uniforms per point, key = ((c*nz + K-1)*ny + J-1)*nx + I-1."""
        nx, ny, nz = self.n
        K, J, I = np.meshgrid(np.arange(nz, dtype=np.uint64), np.arange(ny, dtype=np.uint64),
                              np.arange(nx, dtype=np.uint64), indexing="ij")
        cc = np.uint64(STAG[c])
        key = ((cc * np.uint64(nz) + K) * np.uint64(ny) + J) * np.uint64(nx) + I
        seed = np.uint64(seed)
        two = np.uint64(2)
        r1 = _splitmix64(seed + two * key)
        r2 = _splitmix64(seed + two * key + np.uint64(1))
        u1 = ((r1 >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
        u2 = ((r2 >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
        phi[1:-1, 1:-1, 1:-1] = np.sqrt(-2 * np.log(u1)) * np.cos(2 * np.pi * u2)

    def _shells(self):
        nx, ny, nz = self.n
        kz = np.fft.fftfreq(nz, 1.0 / nz).round().astype(np.int64)
        ky = np.fft.fftfreq(ny, 1.0 / ny).round().astype(np.int64)
        kx = np.fft.fftfreq(nx, 1.0 / nx).round().astype(np.int64)
        k2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
        sh = np.floor(np.sqrt(k2.astype(np.float64))).astype(np.int64)
        sh -= sh * sh > k2
        sh += (sh + 1) ** 2 <= k2
        return sh

    def shell_count(self):
        return int(self._shells().max()) + 1

    def shell_energies(self, u, nshells):
        """shell_energies (src/spectral/forcing.jl:12-24) for shells 0..nshells-1."""
        sh = self._shells()
        N = float(np.prod(self.n))
        e = sum(np.abs(np.fft.fftn(self.interior(u[c]))) ** 2 for c in "xyz") / 2 / N ** 2
        E = np.zeros(nshells)
        m = sh < nshells
        np.add.at(E, sh[m], e[m])
        return E

    def rescale_shells(self, u, factors):
        """rescale_shell! (src/spectral/forcing.jl:26-35), every shell s <
        len(factors) times factors[s]; halos refilled."""
        sh = self._shells()
        f = np.ones(sh.shape)
        m = sh < len(factors)
        f[m] = np.asarray(factors)[sh[m]]
        for c in "xyz":
            u[c][1:-1, 1:-1, 1:-1] = np.fft.ifftn(np.fft.fftn(self.interior(u[c])) * f).real
        self.exchange_halo(u)

    def random_field(self, u, totalenergy=1.0, kpeak=4.0, seed=0, profile=None):
        """spectral_randomfield! (src/spectral/ic.jl:59-84) on the staggered
        velocity: noise, halos, FV projection, shells rescaled to the profile."""
        for c in "xyz":
            self.gauss_noise(u[c], c, seed)
        self.exchange_halo(u)
        self.project(u, self.scalarfield())
        nb = self.shell_count()
        E = self.shell_energies(u, nb)
        k = np.arange(nb, dtype=np.float64)
        prof = (np.array([profile(v) for v in range(nb)]) if profile is not None
                else k ** 4 * np.exp(-2 * (k / kpeak) ** 2))
        e0 = totalenergy * prof / prof.sum()
        f = np.where(E > 0, np.sqrt(e0 / np.where(E > 0, E, 1.0)), 0.0)
        self.rescale_shells(u, f)
        return u

    def shellforcing(self, u, shells=(1, 2), eref=None):
        """shellforcing (src/spectral/forcing.jl:37-56): returns forcing(u)."""
        shells = list(shells)
        nb = max(shells) + 1
        eref = self.shell_energies(u, nb)[shells] if eref is None else np.asarray(eref)

        def forcing(u2):
            e = self.shell_energies(u2, nb)
            f = np.ones(nb)
            for sh, e0 in zip(shells, eref):
                f[sh] = np.sqrt(e0 / e[sh]) if e[sh] > 0 else 1.0
            self.rescale_shells(u2, f)

        forcing.eref = eref
        return forcing

    # ------------------------------------------------------------- stats
    def channel_sample(self, u, acc):
        lib().dnso_channel_sample(self._h, _p(u["x"]), _p(u["y"]), _p(u["z"]), _p(acc))

    def channelstats(self, nupdate=1):
        ny = self.n[1]
        nf = ny - 1 if self.wall else ny
        st = {"nsamples": 0, "acc": np.zeros(4 * ny + 4 * nf), "ny": ny, "nf": nf}

        def sample(u, p, t, n):
            if n % nupdate == 0:
                self.channel_sample(u, st["acc"])
                st["nsamples"] += 1

        st["sample"] = sample
        return st

    def channelprofiles(self, cs):
        """channelprofiles (src/stats.jl:65-98) on one rank."""
        nx, ny, nz = self.n
        nf = cs["nf"]
        norm = max(cs["nsamples"], 1) * nx * nz
        a = cs["acc"] / norm
        Uc, Wc, uuc, wwc = a[0:ny], a[ny:2 * ny], a[2 * ny:3 * ny], a[3 * ny:4 * ny]
        o = 4 * ny
        Vf, vvf, Uf, uvf = a[o:o + nf], a[o + nf:o + 2 * nf], a[o + 2 * nf:o + 3 * nf], a[o + 3 * nf:o + 4 * nf]
        return {
            "y": self.yc.copy(),
            "yf": self.yfaces[1:ny] if self.wall else self.yfaces[1:ny + 1],
            "U": Uc, "V": Vf, "W": Wc,
            "uu": uuc - Uc ** 2, "vv": vvf - Vf ** 2, "ww": wwc - Wc ** 2,
            "uv": uvf - Uf * Vf, "nsamples": cs["nsamples"],
        }

    def spectrumstats(self, nupdate=1):
        if self.bc != ("periodic",) * 3:
            raise ValueError("spectra require a fully periodic box")
        nbins = math.ceil(math.sqrt(sum((v // 2) ** 2 for v in self.n))) + 1
        st = {"nsamples": 0, "E": np.zeros(nbins)}

        def sample(u, p, t, n):
            if n % nupdate == 0:
                lib().dnso_spectrum_sample(self._h, _p(u["x"]), _p(u["y"]), _p(u["z"]),
                                           _p(st["E"]), nbins)
                st["nsamples"] += 1

        st["sample"] = sample
        return st

    def energyspectrum(self, sp):
        E = sp["E"] / max(sp["nsamples"], 1)
        return np.arange(len(E)), E


def _splitmix64(x):
    """splitmix64 (src/spectral/ic.jl:31-36) on uint64 arrays (wrapping)."""
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def cfft(x, inverse=False):
    """Oracle complex FFT along the last axis (AbstractFFTs conventions)."""
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    n = a.shape[-1]
    lib().dnso_cfft(n, a.size // n, int(inverse), _p(a))
    return a


def rfft(x):
    a = np.ascontiguousarray(x, dtype=np.float64)
    n = a.shape[-1]
    out = np.zeros(a.shape[:-1] + (n // 2 + 1,), dtype=np.complex128)
    lib().dnso_rfft(n, a.size // n, _p(a), _p(out))
    return out


def irfft(X, n):
    a = np.ascontiguousarray(X, dtype=np.complex128)
    out = np.zeros(a.shape[:-1] + (n,))
    lib().dnso_irfft(n, a.size // (n // 2 + 1), _p(a), _p(out))
    return out
