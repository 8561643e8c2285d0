// spectral.cuh -- pressure Poisson pipeline and the wall-normal solves.
//
// poisson! (src/poisson.jl:147-161) on one GPU: every transpose! of the
// reference is an identity copy on a single rank (src/transpose.jl:96-102),
// so the stages address one spectrum buffer S in the layout of sidx()
// (kz fastest, y, kx slowest) and no copy kernel exists:
//   k_rfftx  : [divergence of W] -> real FFT along x -> S       (x lines)
//   k_fftz   : complex FFT along z, in place                    (z lines)
//   k_thomas : Thomas along y per (kx, kz) (walls)              (y lines)
//   k_yfourier: FFT along y, divide by lambda, inverse (periodic y)
//   k_fftz<inv>, then k_irfftx: inverse real FFT -> psi (+ ghost images)
// and the semi-implicit wall-normal Crank-Nicolson solve (k_cn).
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include "tma.cuh"

namespace dnsb {

constexpr int SPEC_THREADS = 256;

enum RInMode { RIN_DIVERGENCE = 0, RIN_REAL = 1, RIN_FIELD = 2, RIN_PRODUCT = 3 };
enum ROutMode { ROUT_INTERIOR = 0, ROUT_IMAGES = 1, ROUT_REAL = 2 };

// Real forward FFT along x of L lines (j fixed, kz = k0..k0+L-1) through
// the half-length complex transform: z[m] = r[2m] + i r[2m+1],
// X[k] = E[k] + w^k O[k] with E = (Z[k] + conj Z[M-k])/2,
// O = (Z[k] - conj Z[M-k])/(2i), w = exp(-2 pi i/nx), k = 0..M.
// RIN_DIVERGENCE: r is the divergence of (in0, in1, in2) (operators.jl:10-26).
// RIN_REAL: r is the ghost-free array in0.  RIN_FIELD: the interior of the
// ghosted field in0.  RIN_PRODUCT (four-step kernel only): r = in0 * in1,
// both ghost-free (the velocity products of the spectral solver).
// Shared memory: 2*L*(M+1) complex (ping-pong lines) + M + (M+1) twiddles.
template <int INMODE>
__global__ void __launch_bounds__(SPEC_THREADS, 3) k_rfftx(Geo g, double2 *__restrict__ S,
                                                       const double *__restrict__ in0,
                                                       const double *__restrict__ in1,
                                                       const double *__restrict__ in2,
                                                       FFTPlan plan, int L,
                                                       const double2 *__restrict__ twM,
                                                       const double2 *__restrict__ twN) {
  extern __shared__ double2 smem[];
  const int M = g.nx / 2;
  const int ls = M + 1;
  double2 *buf = smem;
  double2 *buf2 = smem + L * ls;
  double2 *tw = buf2 + L * ls;
  double2 *tn = tw + M;
  const int ngrp = (g.nz + L - 1) / L;
  const int grp = blockIdx.x % ngrp;
  const int j = blockIdx.x / ngrp;  // 0-based row
  const int k0 = grp * L;
  for (int t = threadIdx.x; t < M; t += blockDim.x) tw[t] = twM[t];
  for (int t = threadIdx.x; t <= M; t += blockDim.x) tn[t] = twN[t];
  const long long sy = g.NX, sz = (long long)g.NX * g.NY;
  const int J = j + 1;
  const double rdyJ = __ldg(g.rdy + J);
  __syncthreads();
  auto ld = [&](int l, int m) {
    const int k = k0 + l;
    double2 z = make_double2(0.0, 0.0);
    if (k < g.nz) {
      if (INMODE == RIN_REAL) {
        const double *row = in0 + (long long)g.nx * (j + (long long)g.ny * k);
        z = __ldg(reinterpret_cast<const double2 *>(row + 2 * m));
      } else {
        const long long c0 = gidx(g, 2 * m + 1, J, k + 1);
        if (INMODE == RIN_FIELD) {
          z = make_double2(__ldg(in0 + c0), __ldg(in0 + c0 + 1));
        } else {
          const double a0 = __ldg(in0 + c0 - 1), a1 = __ldg(in0 + c0), a2 = __ldg(in0 + c0 + 1);
          const double b0 = __ldg(in1 + c0), b1 = __ldg(in1 + c0 - sy);
          const double b2 = __ldg(in1 + c0 + 1), b3 = __ldg(in1 + c0 + 1 - sy);
          const double d0 = __ldg(in2 + c0), d1 = __ldg(in2 + c0 - sz);
          const double d2 = __ldg(in2 + c0 + 1), d3 = __ldg(in2 + c0 + 1 - sz);
          const double r0 = (a1 - a0) * g.rdx + (b0 - b1) * rdyJ + (d0 - d1) * g.rdz;
          const double r1 = (a2 - a1) * g.rdx + (b2 - b3) * rdyJ + (d2 - d3) * g.rdz;
          z = make_double2(r0, r1);
        }
      }
    }
    return z;
  };
  auto nost = [](int, int, double2) {};
  const double2 *res = fft_lines_io<false>(ld, nost, buf, buf2, plan, L, 1, ls, true, tw, true, false);
  // post-process and store S(kx, j, k0 + l), l fastest (coalesced in kz)
  const int Lv = min(L, g.nz - k0);
  for (int t = threadIdx.x; t < Lv * (M + 1); t += blockDim.x) {
    const int kx = t / Lv, l = t - kx * Lv;
    const double2 zk = res[l * ls + (kx == M ? 0 : kx)];
    const double2 zc = cconj(res[l * ls + (kx == 0 ? 0 : M - kx)]);
    const double2 e = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
    // o = -i/2 (zk - zc)
    const double2 d = csub(zk, zc);
    const double2 o = make_double2(0.5 * d.y, -0.5 * d.x);
    S[sidx(g, kx, j, k0 + l)] = cadd(e, cmul(tn[kx], o));
  }
}

// Complex FFT along z of L contiguous lines of S; INV scales by 1/nz.  The
// first stage loads from HBM into registers, the last stores from registers.
template <bool INV>
__global__ void __launch_bounds__(SPEC_THREADS, 3) k_fftz(Geo g, double2 *__restrict__ S,
                                                      FFTPlan plan, int L,
                                                      const double2 *__restrict__ twz) {
  extern __shared__ double2 smem[];
  const int n = g.nz;
  const int ls = n + 1;
  double2 *buf = smem;
  double2 *buf2 = smem + L * ls;
  double2 *tw = buf2 + L * ls;
  const long long nlines = (long long)g.ny * g.nkx;
  const long long l0 = (long long)blockIdx.x * L;
  const int Lv = (int)min((long long)L, nlines - l0);
  for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twz[t];
  __syncthreads();
  double2 *src = S + l0 * n;
  const double sc = 1.0 / n;
  fft_lines_io<INV>(
      [&](int l, int e) { return l < Lv ? src[l * n + e] : make_double2(0.0, 0.0); },
      [&](int l, int e, double2 v) {
        if (l < Lv) src[l * n + e] = INV ? cscale(v, sc) : v;
      },
      buf, buf2, plan, L, 1, ls, true, tw, true, true);
}

// Persistent z-FFT: each CTA walks tiles of L contiguous z-lines; the next
// tile is fetched with one bulk asynchronous copy (TMA engine) into the other
// half of a double-buffered staging area while the current tile is
// transformed.  The first radix stage reads the staging buffer, the middle
// stages ping-pong in shared memory, the last stage writes HBM directly.
// Every thread waits for the tile at most wait_limit polls; if any thread
// ran out, the whole CTA (a uniform decision, __syncthreads_or) records err,
// lets the copies it has in flight land (drained with DNSB_WAIT_LIMIT polls
// by thread 0) and returns, so no bulk copy outlives its CTA.
template <bool INV>
__global__ void __launch_bounds__(SPEC_THREADS, 2) k_fftz_tma(Geo g, double2 *__restrict__ S,
                                                             FFTPlan plan, int L,
                                                             const double2 *__restrict__ twz,
                                                             int *err, unsigned wait_limit) {
  extern __shared__ __align__(128) double2 smem[];
  const int n = g.nz;
  const int ls = n + 1;
  double2 *stage0 = smem;
  double2 *stage1 = smem + L * n;
  double2 *A = stage1 + L * n;
  double2 *B = A + L * ls;
  double2 *tw = B + L * ls;
  uint64_t *bar = reinterpret_cast<uint64_t *>(tw + n);
  const long long nlines = (long long)g.ny * g.nkx;
  const long long ngroups = (nlines + L - 1) / L;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twz[t];
  __syncthreads();
  auto issue = [&](long long grp, int b) {
    const long long l0 = grp * L;
    const uint32_t bytes = (uint32_t)(min((long long)L, nlines - l0) * n * sizeof(double2));
    mbar_expect_tx(&bar[b], bytes);
    bulk_g2s(b ? stage1 : stage0, S + l0 * n, bytes, &bar[b]);
  };
  long long grp = blockIdx.x;
  if (grp < ngroups && threadIdx.x == 0) issue(grp, 0);
  const double sc = 1.0 / n;
  for (int it = 0; grp < ngroups; grp += gridDim.x, it++) {
    const int cur = it & 1;
    const long long nxt = grp + gridDim.x;
    if (nxt < ngroups && threadIdx.x == 0) {
      fence_proxy_async_smem();  // the previous readers of this buffer are past a barrier
      issue(nxt, cur ^ 1);
    }
    const bool ok = mbar_wait_n(&bar[cur], (it >> 1) & 1, wait_limit);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(err, DEVERR_TMA_TIMEOUT);
        mbar_wait_n(&bar[cur], (it >> 1) & 1, DNSB_WAIT_LIMIT);
        if (nxt < ngroups) mbar_wait_n(&bar[cur ^ 1], ((it + 1) >> 1) & 1, DNSB_WAIT_LIMIT);
      }
      __syncthreads();
      return;
    }
    const double2 *st = cur ? stage1 : stage0;
    const long long l0 = grp * L;
    const int Lv = (int)min((long long)L, nlines - l0);
    double2 *dst = S + l0 * n;
    fft_lines_io<INV>(
        [&](int l, int e) { return l < Lv ? st[l * n + e] : make_double2(0.0, 0.0); },
        [&](int l, int e, double2 v) {
          if (l < Lv) dst[l * n + e] = INV ? cscale(v, sc) : v;
        },
        A, B, plan, L, 1, ls, true, tw, true, true);
  }
}

// thomas_kernel! (src/poisson.jl:14-41): one thread per (kx, kz) line, in
// place on S, c' in the work array (same layout as S).  The mean mode
// (lambda == 0) is pinned by replacing its first row with x_1 = 0.  Rows are
// processed in groups of TP whose loads are issued together, so a thread
// keeps TP rows in flight while its recurrence runs.
constexpr int TP = 8;
__global__ void __launch_bounds__(128) k_thomas(Geo g, double2 *__restrict__ S,
                                                double *__restrict__ work,
                                                const double *__restrict__ ay,
                                                const double *__restrict__ by,
                                                const double *__restrict__ cy,
                                                const double *__restrict__ lam1,
                                                const double *__restrict__ lam3) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)g.nz * g.nkx) return;
  const int kz = (int)(t % g.nz), kx = (int)(t / g.nz);
  const double lam = lam1[kx] + lam3[kz];
  const long long st = g.nz;
  const int ny = g.ny;
  double2 *x = S + sidx(g, kx, 0, kz);
  double *cp = work + sidx(g, kx, 0, kz);
  const bool pin = lam == 0.0;
  double beta = pin ? 1.0 : by[0] + lam;
  double cprev = (pin ? 0.0 : cy[0]) / beta;
  cp[0] = cprev;
  double2 xprev = pin ? make_double2(0.0, 0.0) : x[0];
  xprev = make_double2(xprev.x / beta, xprev.y / beta);
  x[0] = xprev;
  for (int j0 = 1; j0 < ny; j0 += TP) {
    double2 xr[TP];
#pragma unroll
    for (int q = 0; q < TP; q++)
      if (j0 + q < ny) xr[q] = x[(j0 + q) * st];
#pragma unroll
    for (int q = 0; q < TP; q++) {
      const int j = j0 + q;
      if (j < ny) {
        const double a = __ldg(ay + j);
        beta = (__ldg(by + j) + lam) - a * cprev;
        cprev = __ldg(cy + j) / beta;
        cp[j * st] = cprev;
        xprev = make_double2((xr[q].x - a * xprev.x) / beta, (xr[q].y - a * xprev.y) / beta);
        x[j * st] = xprev;
      }
    }
  }
  double2 xn = xprev;
  for (int j0 = ny - 2; j0 >= 0; j0 -= TP) {
    double2 xr[TP];
    double cr[TP];
#pragma unroll
    for (int q = 0; q < TP; q++)
      if (j0 - q >= 0) {
        xr[q] = x[(j0 - q) * st];
        cr[q] = cp[(j0 - q) * st];
      }
#pragma unroll
    for (int q = 0; q < TP; q++) {
      const int j = j0 - q;
      if (j >= 0) {
        const double2 xj = make_double2(xr[q].x - cr[q] * xn.x, xr[q].y - cr[q] * xn.y);
        x[j * st] = xj;
        xn = xj;
      }
    }
  }
}

// Periodic y (src/poisson.jl:106-118,135-138, modedivide_kernel! :43-49):
// per CTA a tile of L consecutive kz for one kx with all ny rows: FFT along
// y, divide by lambda1+lambda2+lambda3 (0 for the mean), inverse, 1/ny.
// YF_FORWARD leaves the forward transform in S (spectra, shell operations);
// YF_INVERSE only applies the inverse (with 1/ny).
enum YFourierMode { YF_SOLVE = 0, YF_FORWARD = 1, YF_INVERSE = 2 };
template <int YMODE>
__global__ void __launch_bounds__(SPEC_THREADS, 3) k_yfourier(Geo g, double2 *__restrict__ S,
                                                          FFTPlan plan, int L,
                                                          const double2 *__restrict__ twy,
                                                          const double *__restrict__ lam1,
                                                          const double *__restrict__ lam2,
                                                          const double *__restrict__ lam3) {
  extern __shared__ double2 smem[];
  const int n = g.ny;
  double2 *buf = smem;  // buf[j*L + l]
  double2 *buf2 = smem + L * n;
  double2 *tw = buf2 + L * n;
  const int ngrp = (g.nz + L - 1) / L;
  const int grp = blockIdx.x % ngrp;
  const int kx = blockIdx.x / ngrp;
  const int k0 = grp * L;
  const int Lv = min(L, g.nz - k0);
  for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twy[t];
  __syncthreads();
  auto ld = [&](int l, int e) {
    return l < Lv ? S[sidx(g, kx, e, k0 + l)] : make_double2(0.0, 0.0);
  };
  const double sc = YMODE == YF_FORWARD ? 1.0 : 1.0 / n;
  auto st = [&](int l, int e, double2 v) {
    if (l < Lv) S[sidx(g, kx, e, k0 + l)] = YMODE == YF_FORWARD ? v : cscale(v, sc);
  };
  if (YMODE == YF_FORWARD) {
    fft_lines_io<false>(ld, st, buf, buf2, plan, L, L, 1, false, tw, true, true);
    return;
  }
  if (YMODE == YF_INVERSE) {
    fft_lines_io<true>(ld, st, buf, buf2, plan, L, L, 1, false, tw, true, true);
    return;
  }
  double2 *res = fft_lines_io<false>(ld, st, buf, buf2, plan, L, L, 1, false, tw, true, false);
  const double l1 = lam1[kx];
  for (int t = threadIdx.x; t < L * n; t += blockDim.x) {
    const int j = t / L, l = t - j * L;
    const int kz = min(k0 + l, g.nz - 1);
    const double lam = (l1 + lam2[j]) + lam3[kz];
    const double2 v = res[t];
    res[t] = lam == 0.0 ? make_double2(0.0, 0.0) : make_double2(v.x / lam, v.y / lam);
  }
  __syncthreads();
  fft_lines_io<true>(ld, st, res, res == buf ? buf2 : buf, plan, L, L, 1, false, tw, false, true);
}

// Inverse real FFT along x (normalised 1/nx, imaginary parts of the kx = 0
// and kx = nx/2 inputs ignored as in FFTW c2r) of L lines, written to
//   ROUT_INTERIOR: the interior of the ghosted psi (poisson!, no halo),
//   ROUT_IMAGES:   the interior plus pressure ghost images,
//   ROUT_REAL:     the ghost-free array out.
template <int OUTMODE>
__global__ void __launch_bounds__(SPEC_THREADS, 3) k_irfftx(Geo g, const double2 *__restrict__ S,
                                                        double *__restrict__ out, FFTPlan plan,
                                                        int L, const double2 *__restrict__ twM,
                                                        const double2 *__restrict__ twN) {
  extern __shared__ double2 smem[];
  const int M = g.nx / 2;
  const int ls = M + 2;
  double2 *buf = smem;
  double2 *buf2 = smem + L * ls;
  double2 *tw = buf2 + L * ls;
  double2 *tn = tw + M;
  const int ngrp = (g.nz + L - 1) / L;
  const int grp = blockIdx.x % ngrp;
  const int j = blockIdx.x / ngrp;
  const int k0 = grp * L;
  const int Lv = min(L, g.nz - k0);
  for (int t = threadIdx.x; t < M; t += blockDim.x) tw[t] = twM[t];
  for (int t = threadIdx.x; t <= M; t += blockDim.x) tn[t] = twN[t];
  batched_copy<8>(
      L * (M + 1),
      [&](int t) {
        const int kx = t / L, l = t - kx * L;
        return l < Lv ? S[sidx(g, kx, j, k0 + l)] : make_double2(0.0, 0.0);
      },
      [&](int t, double2 v) {
        const int kx = t / L, l = t - kx * L;
        buf[l * ls + kx] = v;
      });
  __syncthreads();
  // Z[k] = E[k] + i O[k], E = (X[k] + conj X[M-k])/2,
  // O = (X[k] - conj X[M-k]) conj(w^k)/2; one thread per pair (k, M-k).
  const int half = M / 2 + 1;
  for (int t = threadIdx.x; t < L * half; t += blockDim.x) {
    const int l = t / half, k = t - l * half;
    double2 *X = buf + l * ls;
    if (k == 0) {
      const double a = X[0].x, b = X[M].x;
      const double e = 0.5 * (a + b), o = 0.5 * (a - b);
      X[0] = make_double2(e, o);
    } else if (2 * k <= M) {
      const int k2 = M - k;
      const double2 a = X[k], b = X[k2];
      {
        const double2 bc = cconj(b);
        const double2 e = cscale(cadd(a, bc), 0.5);
        const double2 o = cmul(cscale(csub(a, bc), 0.5), cconj(tn[k]));
        X[k] = make_double2(e.x - o.y, e.y + o.x);
      }
      if (k2 != k) {
        const double2 ac = cconj(a);
        const double2 e = cscale(cadd(b, ac), 0.5);
        const double2 o = cmul(cscale(csub(b, ac), 0.5), cconj(tn[k2]));
        X[k2] = make_double2(e.x - o.y, e.y + o.x);
      }
    }
  }
  __syncthreads();
  const double sc = 1.0 / M;
  const int J = j + 1;
  auto noload = [](int, int) { return make_double2(0.0, 0.0); };
  auto st = [&](int l, int m, double2 z) {
    if (l >= Lv) return;
    const double x0 = z.x * sc, x1 = z.y * sc;
    const int K = k0 + l + 1;
    if (OUTMODE == ROUT_REAL) {
      double *row = out + (long long)g.nx * (j + (long long)g.ny * (K - 1));
      *reinterpret_cast<double2 *>(row + 2 * m) = make_double2(x0, x1);
    } else if (OUTMODE == ROUT_INTERIOR) {
      const long long c0 = gidx(g, 2 * m + 1, J, K);
      out[c0] = x0;
      out[c0 + 1] = x1;
    } else {
      store_img(out, g, 2 * m + 1, J, K, x0, STAG_P);
      store_img(out, g, 2 * m + 2, J, K, x1, STAG_P);
    }
  };
  fft_lines_io<true>(noload, st, buf, buf2, plan, L, 1, ls, true, tw, false, true);
}

// Per-stage Crank-Nicolson tables (imexsolve_kernel!, src/ydiffusion.jl:94-109).
// The Thomas coefficients of (I - theta Dy) depend on y only, so they are
// computed once per stage and set instead of once per line: beta_j,
// c'_j = -theta c_j / beta_j, theta a_j.  For the chunked sweeps of k_cn the
// forward multipliers f_j = theta a_j / beta_j and backward multipliers
// -c'_j are also accumulated per chunk of m rows:
//   g_j = prod_{i=s..j} f_i (s = chunk start), h_j = prod_{i=j..e} (-c'_i)
// (e = chunk end), G_k = g at the end of chunk k, H_k = h at its start.
// tab layout per (stage, set): [ta | cp | ib | g | h](ny each), [G | H](CN_CHUNKS
// each); ib = 1/beta; set 0 tangential, 1 normal.  coef: [at bt ct an bn cn].
// m is the number of rows per chunk (a power of two, CN_CHUNKS * m >= ny).
constexpr int CN_CHUNKS = 16;
constexpr int CN_LINES = 16;

constexpr int CN_MAXCHUNKS = 32;
__host__ __device__ constexpr long long cn_tab_stride(int ny) { return 5LL * ny + 2 * CN_MAXCHUNKS; }
// Shared-memory pitch of one k_cn table with rows skewed by their chunk.
__host__ __device__ constexpr int cn_skew_pitch(int ny, int mr) { return ny + (ny + mr - 1) / mr; }

// Launch with CN_TABLE_THREADS threads: threads 0..5 (stage, set) run the
// sequential factorisation, then thread (stage, set, chunk) forms the
// products of one chunk.
constexpr int CN_TABLE_THREADS = 6 * CN_MAXCHUNKS;
__global__ void k_cn_tables(int ny, int m, int nchunks, const double *__restrict__ coef,
                            double *__restrict__ tab, double dt, double visc, double al0,
                            double al1, double al2) {
  const int t = threadIdx.x;
  const int seq = t % 6, k = t / 6;
  const int st = seq / 2, set = seq % 2;
  double *ta = tab + (long long)(st * 2 + set) * cn_tab_stride(ny);
  double *cp = ta + ny, *ib = cp + ny, *gf = ib + ny, *hb = gf + ny;
  double *G = hb + ny, *H = G + CN_MAXCHUNKS;
  if (k == 0) {
    const double al = st == 0 ? al0 : st == 1 ? al1 : al2;
    const double th = al * dt * visc / 2;
    const double *a = coef + (set ? 3 : 0) * ny;
    const double *b = a + ny, *c = b + ny;
    double beta = 1 - th * b[0];
    double cprev = -th * c[0] / beta;
    ta[0] = th * a[0];
    cp[0] = cprev;
    ib[0] = 1.0 / beta;
    for (int j = 1; j < ny; j++) {
      beta = (1 - th * b[j]) + th * a[j] * cprev;
      cprev = -th * c[j] / beta;
      ta[j] = th * a[j];
      cp[j] = cprev;
      ib[j] = 1.0 / beta;
    }
  }
  __syncthreads();  // also orders the global writes above for the block
  if (k >= nchunks) return;
  const int s0 = k * m, e0 = min(ny, s0 + m) - 1;
  G[k] = 1.0;
  H[k] = 1.0;
  if (s0 > e0) return;
  double acc = 1.0;
  for (int j = s0; j <= e0; j++) {
    acc *= ta[j] * ib[j];
    gf[j] = acc;
  }
  G[k] = acc;
  acc = 1.0;
  for (int j = e0; j >= s0; j--) {
    acc *= -cp[j];
    hb[j] = acc;
  }
  H[k] = acc;
}

// imexsolve_kernel! (src/ydiffusion.jl:94-109) on right-hand sides that the
// producer (k_momentum<IMPLICIT> or k_vupdate) has already formed.
// A block owns CN_LINES consecutive x-lines (I) at one K for component
// c = blockIdx.z and splits every y-line into CN_CHUNKS chunks of MR rows,
// one thread per (line, chunk).  A thread loads its rows of V straight into
// registers (all loads issued together), runs the Thomas forward sweep from
// a zero carry; the chunks exchange their end values through shared memory
// and add the carried-in part with the per-chunk multiplier products
// (g, G); the backward sweep is split the same way (h, H).  Algebraically
// this is the reference's Thomas algorithm; every element is read from and
// written to HBM once.  The line-independent coefficient tables sit in
// shared memory.
template <int MR>
__global__ void __launch_bounds__(CN_LINES *CN_CHUNKS, 3) k_cn(Geo g, Fields3 out, CFields3 V,
                                                              const double *__restrict__ tab) {
  extern __shared__ double cs[];  // ta cp ib gf hb (ny each), G H, exchange
  const int i = threadIdx.x, ck = threadIdx.y;
  const int tid = i + CN_LINES * ck;
  const int I0 = blockIdx.x * CN_LINES + 1;
  const int I = I0 + i;
  const int K = blockIdx.y + 1;
  const int c = blockIdx.z;
  const int ny = g.ny;
  const int set = c == STAG_Y ? 1 : 0;
  const double *v = c == 0 ? V.x : c == 1 ? V.y : V.z;
  double *o = c == 0 ? out.x : c == 1 ? out.y : out.z;
  const int sy = g.NX;
  const bool active = I <= g.nx;
  const int base = gidx(g, active ? I : I0, 1, K);
  const int s0 = ck * MR;
  // 1. this thread's rows of the right-hand side
  double x[MR];
#pragma unroll
  for (int r = 0; r < MR; r++) {
    const int j = s0 + r;
    x[r] = (active && j < ny) ? v[base + j * sy] : 0.0;
  }
  // 2. stage the tables (line-independent) while the loads are in flight;
  // row j sits at j + j/MR so that the two chunks of a warp hit different
  // banks
  const int tp = cn_skew_pitch(ny, MR);
  double *ta_ = cs, *ib_ = cs + tp, *cp_ = cs + 2 * tp, *gf_ = cs + 3 * tp, *hb_ = cs + 4 * tp;
  double *G_ = cs + 5 * tp, *H_ = G_ + CN_CHUNKS;  // copies of G[0..CN_CHUNKS), H[...]
  double *xa = H_ + CN_CHUNKS, *xb = xa + CN_CHUNKS * CN_LINES;
  {
    const double *ts = tab + set * cn_tab_stride(ny);  // [ta cp ib gf hb] G H
    for (int t = tid; t < ny; t += CN_LINES * CN_CHUNKS) {
      const int u = t + t / MR;
      ta_[u] = ts[t];
      cp_[u] = ts[ny + t];
      ib_[u] = ts[2 * ny + t];
      gf_[u] = ts[3 * ny + t];
      hb_[u] = ts[4 * ny + t];
    }
    if (tid < CN_CHUNKS) {
      G_[tid] = ts[5 * ny + tid];
      H_[tid] = ts[5 * ny + CN_MAXCHUNKS + tid];
    }
  }
  __syncthreads();
  // 3. local forward sweep (zero carry)
  double z = 0.0;
#pragma unroll
  for (int r = 0; r < MR; r++) {
    const int j = s0 + r;
    if (j < ny) {
      z = r == 0 ? x[r] * ib_[j + ck] : fma(ta_[j + ck], z, x[r]) * ib_[j + ck];
      x[r] = z;
    }
  }
  xa[ck * CN_LINES + i] = z;
  __syncthreads();
  // 4. carry into this chunk from the earlier chunks (unrolled: the
  // shared-memory loads are independent of the FMA chain), backward sweep
  double cin = 0.0;
#pragma unroll
  for (int k = 0; k < CN_CHUNKS - 1; k++) {
    const double a = xa[k * CN_LINES + i], gk = G_[k];
    if (k < ck) cin = fma(gk, cin, a);
  }
  double bnext = 0.0;
#pragma unroll
  for (int r = MR - 1; r >= 0; r--) {
    const int j = s0 + r;
    if (j < ny) {
      const double xp = fma(gf_[j + ck], cin, x[r]);
      bnext = fma(-cp_[j + ck], bnext, xp);
      x[r] = bnext;
    }
  }
  xb[ck * CN_LINES + i] = s0 < ny ? bnext : 0.0;
  __syncthreads();
  // 5. carry from the later chunks, final values with ghost images
  double cout = 0.0;
#pragma unroll
  for (int k = CN_CHUNKS - 1; k > 0; k--) {
    const double a = xb[k * CN_LINES + i], hk = H_[k];
    if (k > ck) cout = fma(hk, cout, a);
  }
  if (active) {
    const bool normal_wall = g.wall && c == STAG_Y;
    const bool line_edge = (I == 1) | (I == g.nx) | (K == 1) | (K == g.nz);
#pragma unroll
    for (int r = 0; r < MR; r++) {
      const int j = s0 + r;
      if (j < ny) {
        const double xv = fma(hb_[j + ck], cout, x[r]);
        o[base + j * sy] = xv;
        // ghost images of edge lines and of the first/last rows (the
        // inactive wall face of the normal component has none)
        if ((line_edge || j == 0 || j >= ny - 2) && !(normal_wall && j == ny - 1))
          store_images_of(o, g.nx, g.ny, g.nz, g.NX, g.NY, g.wall, I, j + 1, K, xv, c);
      }
    }
  }
}

}  // namespace dnsb
