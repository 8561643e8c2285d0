"""Oracle for the filtered-field / sub-filter-stress sampler -- TEST
INFRASTRUCTURE ONLY (imported by tests/ alone; the product never does).

Restates, for small coarse grids, the reference's rank-0 pipeline of
src/spectral/les.jl with explicit per-mode loops in the reference's own
loop order (lesfreq :42, les_twothirds! :45-54, les_filterkernel! :59-85,
les_nonlinearity! :88-101, les_filter_reynolds :104-116, les_spectrum
:119-131, les_tracefree! :134-143, les_extract! :176-184, the cell loop of
sfs_sample! :347-370), and the distributed half (the LES cube of u_hat and
sigma_hat = F[v_i v_j] / N, :313-334) on an FV state of the C oracle with
numpy's full complex FFT.  Coarse arrays are numpy (M, M, M//2+1) =
[kz, ky, kx].
"""
import math

import numpy as np

PAIRS = ((0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0))


def lesfreq(i, n):
    """Integer frequency of 0-based index i on an n grid (fftfreq order)."""
    return i if i <= (n - 1) // 2 else i - n


def twothirds(a, n):
    kc = n // 3
    a = a.copy()
    for k in range(n):
        for j in range(n):
            for i in range(n // 2 + 1):
                k1, k2, k3 = i, lesfreq(j, n), lesfreq(k, n)
                keep = k1 <= kc and abs(k2) <= kc and abs(k3) <= kc and (k1, k2, k3) != (0, 0, 0)
                if not keep:
                    a[k, j, i] = 0
    return a


def _sinc(x):
    return 1.0 if x == 0 else math.sin(x) / x


def filterkernel(a, n, l, delta, protectshells, kernel):
    kf = 2 * math.pi / l
    kbound2 = (kf * (protectshells + 1)) ** 2
    a = a.copy()
    for k in range(n):
        for j in range(n):
            for i in range(n // 2 + 1):
                k1, k2, k3 = kf * i, kf * lesfreq(j, n), kf * lesfreq(k, n)
                kk = k1 ** 2 + k2 ** 2 + k3 ** 2
                if kk < kbound2:
                    continue
                if kernel == "gaussian":
                    w = math.exp(-delta ** 2 * kk / 24)
                elif kernel == "cutoff":
                    w = 1.0 if kk <= (math.pi / delta) ** 2 else 0.0
                elif kernel == "tophat":
                    w = _sinc(k1 * delta / 2) * _sinc(k2 * delta / 2) * _sinc(k3 * delta / 2)
                elif kernel == "helmholtz":
                    w = 1 / (1 + delta ** 2 * kk / 24)
                else:
                    raise ValueError(kernel)
                a[k, j, i] *= w
    return a


def _full(a, n):
    """Hermitian completion of an rfft array to the full (n, n, n) spectrum."""
    f = np.zeros((n, n, n), dtype=np.complex128)
    f[:, :, :n // 2 + 1] = a
    for i in range(n // 2 + 1, n):
        src = a[:, :, n - i]
        f[:, :, i] = np.conj(src[(-np.arange(n)) % n][:, (-np.arange(n)) % n])
    return f


def _inverse_real(a, n):
    """Real field of an rfft array (the Hermitian part of the kx = 0 and
    Nyquist planes, as a c2r transform reads them), unnormalised."""
    f = _full(a, n)
    for i in (0, n // 2):
        p = f[:, :, i]
        f[:, :, i] = (p + np.conj(p[(-np.arange(n)) % n][:, (-np.arange(n)) % n])) / 2
    return np.fft.ifftn(f).real * n ** 3


def nonlinearity(ub, n):
    vs = [_inverse_real(twothirds(ub[c], n), n) for c in range(3)]
    return [np.fft.fftn(vs[i] * vs[j])[:, :, :n // 2 + 1] / n ** 3 for i, j in PAIRS]


def filter_reynolds(ub, n, l, visc, delta):
    kf = 2 * math.pi / l
    a2 = 0.0
    for k in range(n):
        for j in range(n):
            for i in range(n // 2 + 1):
                kk = kf ** 2 * (i ** 2 + lesfreq(j, n) ** 2 + lesfreq(k, n) ** 2)
                u2 = sum(abs(ub[c][k, j, i]) ** 2 for c in range(3))
                w = 2 if 0 < i < n // 2 else 1
                a2 += w * kk * u2
    return delta ** 2 * math.sqrt(a2) / visc


def spectrum(ub, n):
    kc = n // 3
    E = np.zeros(kc)
    for k in range(n):
        for j in range(n):
            for i in range(n // 2 + 1):
                s2 = i ** 2 + lesfreq(j, n) ** 2 + lesfreq(k, n) ** 2
                sh = math.isqrt(s2)
                if not 1 <= sh <= kc:
                    continue
                u2 = sum(abs(ub[c][k, j, i]) ** 2 for c in range(3))
                w = 2 if 0 < i < n // 2 else 1
                E[sh - 1] += w * u2 / 2
    return E


def tracefree(tau):
    tau = [t.copy() for t in tau]
    tr = (tau[0] + tau[1] + tau[2]) / 3
    for c in range(3):
        tau[c] -= tr
    return tau


def extract(src, M, Mmax):
    dst = np.zeros((M, M, M // 2 + 1), dtype=src.dtype)
    for k in range(M):
        for j in range(M):
            for i in range(M // 2 + 1):
                js = j if j < M // 2 else j - M + Mmax
                ks = k if k < M // 2 else k - M + Mmax
                dst[k, j, i] = src[ks, js, i]
    return dst


def cube(so, u, M):
    """The 9 LES cubes of an oracle FV state (periodic, valid halos): the
    cell-centred velocity (the average of a cell's two faces), its six
    products, full 3-D FFTs / N, the modes |k_i| <= M/2."""
    v = [(u["x"][1:-1, 1:-1, :-2] + u["x"][1:-1, 1:-1, 1:-1]) / 2,
         (u["y"][1:-1, :-2, 1:-1] + u["y"][1:-1, 1:-1, 1:-1]) / 2,
         (u["z"][:-2, 1:-1, 1:-1] + u["z"][1:-1, 1:-1, 1:-1]) / 2]
    fields = v + [v[i] * v[j] for i, j in PAIRS]
    N = float(np.prod(so.n))
    out = []
    for f in fields:
        F = np.fft.fftn(f) / N  # [kz, ky, kx]
        nz, ny, nx = f.shape
        c = np.zeros((M, M, M // 2 + 1), dtype=np.complex128)
        for kc_ in range(M):
            for jc in range(M):
                kz = kc_ if kc_ < M // 2 else kc_ - M
                ky = jc if jc < M // 2 else jc - M
                c[kc_, jc, :] = F[kz % nz, ky % ny, :M // 2 + 1]
        out.append(c)
    return np.stack(out)


def sfs(cells, nles, protectshells, l, visc, cb9):
    """The cell loop of sfs_sample! (src/spectral/les.jl:347-370)."""
    res = []
    for cell in cells:
        M, kernel = cell["M"], cell["kernel"]
        cb = cb9 if M == nles else np.stack([extract(c, M, nles) for c in cb9])
        delta = cell["dfac"] * l / M
        ubf = [twothirds(filterkernel(cb[c], M, l, delta, protectshells, kernel), M) for c in range(3)]
        tau = [filterkernel(cb[3 + c], M, l, delta, protectshells, kernel) for c in range(6)]
        s2 = nonlinearity(ubf, M)
        tau = tracefree([twothirds(tau[c] - s2[c], M) for c in range(6)])
        res.append(dict(ubar=ubf, tau=tau, redelta=filter_reynolds(ubf, M, l, visc, delta),
                        spectrum=spectrum(ubf, M)))
    return res
