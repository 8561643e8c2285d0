"""Oracle for the pseudo-spectral solver -- TEST INFRASTRUCTURE ONLY
(imported by tests/ alone; the product never does).

A numpy restatement of the reference's single-rank spectral solver on a
periodic cube: the compact truncated state of spectral_setup
(src/spectral/setup.jl:62-73, compactfreq operators.jl:7), spec_to_phys! /
phys_to_spec! as zero-padded / truncated numpy real FFTs with
u_hat = F[u]/n^3, spectral_rhs! (operators.jl:66-96, divergence form with
the reference's grouping of the off-diagonal terms), project_kernel!
(:10-23), Wray's RK3 with the integrating-factor viscosity
(step.jl:1-43,60-92) and the diagnostics (:98-110).  The state is numpy
complex (3, m, m, kcut+1) = [component, kz, ky, kx].
"""
import math

import numpy as np

from oracle import _splitmix64

WRAY_A = (8 / 15, 5 / 12, 3 / 4)
WRAY_B = (1 / 4, 0.0, 0.0)
WRAY_DC = (8 / 15, 2 / 15, 1 / 3)


class Spectral:
    def __init__(self, n, l=2 * math.pi, visc=1e-3, kcut=None):
        self.n, self.l, self.visc = n, l, visc
        self.kcut = n // 3 if kcut is None else kcut
        self.m = 2 * self.kcut + 1
        cf = np.array([j if j <= self.kcut else j - self.m for j in range(self.m)])
        self.idx = cf % n                       # compact -> full index along y and z
        kf = 2 * math.pi / l
        self.kx = kf * np.arange(self.kcut + 1)[None, None, :]
        self.ky = kf * cf[None, :, None]
        self.kz = kf * cf[:, None, None]
        self.kk = self.kx ** 2 + self.ky ** 2 + self.kz ** 2

    def zeros(self):
        return np.zeros((3, self.m, self.m, self.kcut + 1), dtype=np.complex128)

    def to_phys(self, uh):
        n = self.n
        v = np.zeros((3, n, n, n))
        for c in range(3):
            full = np.zeros((n, n, n // 2 + 1), dtype=np.complex128)
            full[np.ix_(self.idx, self.idx, np.arange(self.kcut + 1))] = uh[c]
            v[c] = np.fft.irfftn(full, s=(n, n, n), axes=(0, 1, 2)) * n ** 3
        return v

    def from_phys(self, v):
        n = self.n
        out = self.zeros()
        for c in range(3):
            F = np.fft.rfftn(v[c], axes=(0, 1, 2)) / n ** 3
            out[c] = F[np.ix_(self.idx, self.idx, np.arange(self.kcut + 1))]
        return out

    def _spec(self, r):
        F = np.fft.rfftn(r, axes=(0, 1, 2)) / self.n ** 3
        return F[np.ix_(self.idx, self.idx, np.arange(self.kcut + 1))]

    def rhs(self, uh):
        v = self.to_phys(uh)
        sxx, syy, szz = (self._spec(v[c] * v[c]) for c in range(3))
        du = np.stack([-1j * self.kx * sxx, -1j * self.ky * syy, -1j * self.kz * szz])
        sxy, syz, szx = self._spec(v[0] * v[1]), self._spec(v[1] * v[2]), self._spec(v[2] * v[0])
        du[0] -= 1j * (self.ky * sxy + self.kz * szx)
        du[1] -= 1j * (self.kx * sxy + self.kz * syz)
        du[2] -= 1j * (self.kx * szx + self.ky * syz)
        return du, v

    def project(self, uh):
        kk = np.where(self.kk == 0, 1.0, self.kk)
        p = (self.kx * uh[0] + self.ky * uh[1] + self.kz * uh[2]) / kk
        p = np.where(self.kk == 0, 0.0, p)
        return np.stack([uh[0] - self.kx * p, uh[1] - self.ky * p, uh[2] - self.kz * p])

    def step(self, uh, dt):
        ustart = uh.copy()
        vmax = 0.0
        for i in range(3):
            du, v = self.rhs(uh)
            if i == 0:
                vmax = float(np.max(np.abs(v[0]) + np.abs(v[1]) + np.abs(v[2])))
            phi = np.exp(-self.visc * WRAY_DC[i] * dt * self.kk)
            uh = phi * (ustart + WRAY_A[i] * dt * du)
            ustart = phi * (ustart + WRAY_B[i] * dt * du)
            uh = self.project(uh)
        return uh, vmax

    def _w(self):
        return np.where(np.arange(self.kcut + 1) > 0, 2.0, 1.0)[None, None, :]

    def energy(self, uh):
        return float(np.sum(self._w() * np.sum(np.abs(uh) ** 2, axis=0)) / 2)

    def dissipation(self, uh):
        return float(self.visc * np.sum(self._w() * self.kk * np.sum(np.abs(uh) ** 2, axis=0)))

    def maxdiv(self, uh):
        return float(np.max(np.abs(self.kx * uh[0] + self.ky * uh[1] + self.kz * uh[2])))

    def velocityfield(self, x, y, z):
        c = self.l / self.n * (np.arange(self.n) + 0.5)
        Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
        v = np.stack([np.vectorize(f)(X, Y, Z) if f is not None else np.zeros_like(X)
                      for f in (x, y, z)]).astype(np.float64)
        return self.project(self.from_phys(v))

    def random(self, seed, amp=1.0):
        """A random solenoidal state (test input): projected Gaussian noise."""
        rng = np.random.default_rng(seed)
        v = rng.standard_normal((3, self.n, self.n, self.n)) * amp
        return self.project(self.from_phys(v))

    # -------------------------------------------- shells, random field, forcing
    def shells(self):
        kx = np.arange(self.kcut + 1)[None, None, :]
        cf = np.array([j if j <= self.kcut else j - self.m for j in range(self.m)])
        k2 = kx ** 2 + cf[None, :, None] ** 2 + cf[:, None, None] ** 2
        sh = np.floor(np.sqrt(k2.astype(np.float64))).astype(np.int64)
        sh -= sh * sh > k2
        sh += (sh + 1) ** 2 <= k2
        return sh

    def shell_energies(self, uh, nb):
        """shell_energies (src/spectral/forcing.jl:12-24) for shells 0..nb-1."""
        sh = np.broadcast_to(self.shells(), uh.shape[1:])
        e = np.broadcast_to(self._w() * np.sum(np.abs(uh) ** 2, axis=0) / 2, uh.shape[1:])
        E = np.zeros(nb)
        m = sh < nb
        np.add.at(E, sh[m], e[m])
        return E

    def rescale(self, uh, f):
        sh = self.shells()
        fac = np.ones(sh.shape)
        m = sh < len(f)
        fac[m] = np.asarray(f)[sh[m]]
        return uh * fac[None]

    def noise(self, seed):
        """noise_kernel! (src/spectral/ic.jl:37-51), one rank."""
        n = self.n
        v = np.zeros((3, n, n, n))
        K, J, I = np.meshgrid(*(np.arange(n, dtype=np.uint64),) * 3, indexing="ij")
        for c in range(3):
            key = ((np.uint64(c) * np.uint64(n) + K) * np.uint64(n) + J) * np.uint64(n) + I
            sd = np.uint64(seed)
            r1 = _splitmix64(sd + np.uint64(2) * key)
            r2 = _splitmix64(sd + np.uint64(2) * key + np.uint64(1))
            u1 = ((r1 >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
            u2 = ((r2 >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
            v[c] = np.sqrt(-2 * np.log(u1)) * np.cos(2 * np.pi * u2)
        return v

    def randomfield(self, totalenergy=1.0, kpeak=4.0, seed=0, profile=None):
        """spectral_randomfield! (src/spectral/ic.jl:59-84)."""
        uh = self.project(self.from_phys(self.noise(seed)))
        kdiag = int(math.floor(math.sqrt(3) * self.kcut))
        E = self.shell_energies(uh, kdiag + 1)
        k = np.arange(kdiag + 1, dtype=np.float64)
        prof = (np.array([profile(v) for v in range(kdiag + 1)]) if profile is not None
                else k ** 4 * np.exp(-2 * (k / kpeak) ** 2))
        e0 = totalenergy * prof / prof.sum()
        f = np.where(E > 0, np.sqrt(e0 / np.where(E > 0, E, 1.0)), 0.0)
        return self.rescale(uh, f)

    def shellforcing(self, uh, shells=(1, 2), eref=None):
        shells = list(shells)
        nb = max(shells) + 1
        eref = self.shell_energies(uh, nb)[shells] if eref is None else np.asarray(eref)

        def forcing(u2):
            e = self.shell_energies(u2, nb)
            f = np.ones(nb)
            for sh, e0 in zip(shells, eref):
                f[sh] = math.sqrt(e0 / e[sh]) if e[sh] > 0 else 1.0
            return self.rescale(u2, f)

        forcing.eref = eref
        return forcing

    def les_cube(self, uh, M):
        """The LES cube of u_hat (truncation) and sigma_hat = F[v_i v_j]/n^3
        (src/spectral/les.jl:313-334), coarse rfft layout (M, M, M//2+1)."""
        h = M // 2 + 1
        wrap = np.array([j if j < M // 2 else j - M for j in range(M)])
        ci = wrap % self.m                       # compact index of ky / kz
        out = np.zeros((9, M, M, h), dtype=np.complex128)
        for c in range(3):
            out[c] = uh[c][np.ix_(ci, ci, np.arange(h))]
        v = self.to_phys(uh)
        for f, (a, b) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0))):
            F = np.fft.rfftn(v[a] * v[b], axes=(0, 1, 2)) / self.n ** 3
            fi = wrap % self.n
            out[3 + f] = F[np.ix_(fi, fi, np.arange(h))]
        return out

    def phaserandomize(self, uh, seed=0):
        """phaserand_kernel! (src/spectral/ic.jl:108-128)."""
        out = uh.copy()
        w = 2 * self.kcut + 2
        cf = [j if j <= self.kcut else j - self.m for j in range(self.m)]
        for k in range(self.m):
            for j in range(self.m):
                for i in range(self.kcut + 1):
                    k1, k2, k3 = i, cf[j], cf[k]
                    if (k1, k2, k3) == (0, 0, 0):
                        continue
                    canon = k1 > 0 or k2 > 0 or (k2 == 0 and k3 > 0)
                    c2, c3 = (k2, k3) if canon else (-k2, -k3)
                    key = (k1 * w + (c2 + self.kcut)) * w + (c3 + self.kcut)
                    r = int(_splitmix64(np.array([seed + key], dtype=np.uint64))[0])
                    u = ((r >> 11) + 0.5) * 2.0 ** -53
                    ph = complex(math.cos(2 * math.pi * u),
                                 (1 if canon else -1) * math.sin(2 * math.pi * u))
                    out[:, k, j, i] *= ph
        return out
