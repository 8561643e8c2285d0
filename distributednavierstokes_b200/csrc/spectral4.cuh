// spectral4.cuh -- the Poisson transform kernels on the four-step engine.
//
// Same contracts as k_fftz / k_rfftx / k_irfftx in spectral.cuh (which
// remain the path for lengths without a specialised split), with the
// transforms of fft4.cuh: every element crosses shared memory once per
// transform, so these kernels stay bound by HBM traffic.
#pragma once
#include "fft4.cuh"
#include "spectral.cuh"

namespace dnsb {

constexpr int F4_THREADS = 256;

// Complex FFT along z of L contiguous lines of S (n = N1*N2 = nz); INV
// scales by 1/nz.  Shared memory: transpose buffer + n twiddles.
template <int N1, int N2, bool INV>
__global__ void __launch_bounds__(F4_THREADS, 2) k_fftz4(Geo g, double2 *__restrict__ S, int L,
                                                         const double2 *__restrict__ twz) {
  constexpr int n = N1 * N2;
  extern __shared__ double2 smem[];
  double2 *buf = smem;
  double2 *tw = smem + fft4_buf<N1, N2>(L);
  const long long nlines = (long long)g.ny * g.nkx;
  const long long l0 = (long long)blockIdx.x * L;
  const int Lv = (int)min((long long)L, nlines - l0);
  for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twz[t];
  __syncthreads();
  double2 *src = S + l0 * n;
  const double sc = 1.0 / n;
  fft4_lines<N1, N2, INV>(
      [&](int l, int e) { return l < Lv ? src[l * n + e] : make_double2(0.0, 0.0); },
      [&](int l, int e, double2 v) {
        if (l < Lv) src[l * n + e] = INV ? cscale(v, sc) : v;
      },
      buf, L, tw);
}

// Real forward FFT along x of L lines (j fixed, kz = k0..k0+L-1) through the
// half-length complex transform (see k_rfftx).  The packed input
// z[m] = r[2m] + i r[2m+1] (r = divergence of in0..in2, a ghost-free real
// array, or a field's interior) is first staged in shared memory by all
// threads with batched loads, then transformed.  M = N1*N2 = nx/2.
// 3 CTAs per SM (80 registers; the small spill costs less than the third
// CTA gains: 0.377-0.384 ms against 0.392-0.398 ms at 2 CTAs, 384^2 x 256)
// POST: the second FFT pass forms the real-transform output X[k] (which
// needs Z[k] and Z[M-k]) in registers and stores it, instead of writing Z
// back to shared memory for a separate pass.  Its thread (line l, column
// k1) holds Z[k1 + N1 k2], k2 = 0..N2-1; Z[M - k1 - N1 k2] is element
// N2-1-k2 of column N1-k1, so columns k1 and N1-k1 share a warp (8 lines x
// 4 columns per warp) and swap it with one shuffle; columns 0 and N1/2 are
// their own partners.  The transpose buffer rows carry one pad value
// (N1*P + 1 per line) so those 8 lines read distinct banks.
template <int N1, int N2, int L, int INMODE, bool POST = false>
__global__ void __launch_bounds__(F4_THREADS, 3) k_rfftx4(Geo g, double2 *__restrict__ S,
                                                          const double *__restrict__ in0,
                                                          const double *__restrict__ in1,
                                                          const double *__restrict__ in2,
                                                          const double2 *__restrict__ twM,
                                                          const double2 *__restrict__ twN) {
  constexpr int M = N1 * N2;
  constexpr int ls = M + 1;
  constexpr int P = fft4_pitch<N2>();
  constexpr int LS1 = N1 * P + 1;  // transpose-buffer stride per line
  extern __shared__ double2 smem[];
  double2 *buf = smem;
  double2 *res = buf + L * LS1;
  double2 *tw = res + L * ls;
  double2 *tn = tw + M;
  const int ngrp = (g.nz + L - 1) / L;
  const int grp = blockIdx.x % ngrp;
  const int j = blockIdx.x / ngrp;
  const int k0 = grp * L;
  for (int t = threadIdx.x; t < M; t += blockDim.x) tw[t] = twM[t];
  for (int t = threadIdx.x; t <= M; t += blockDim.x) tn[t] = twN[t];
  const long long sy = g.NX, sz = (long long)g.NX * g.NY;
  const int J = j + 1;
  const double rdyJ = __ldg(g.rdy + J);
  batched_copy<4>(
      L * M,
      [&](int t) {
        const int l = t / M, m = t - l * M;
        const int k = k0 + l;
        double2 z = make_double2(0.0, 0.0);
        if (k < g.nz) {
          if (INMODE == RIN_REAL || INMODE == RIN_PRODUCT) {
            const long long ro = (long long)g.nx * (j + (long long)g.ny * k);
            z = __ldg(reinterpret_cast<const double2 *>(in0 + ro + 2 * m));
            if (INMODE == RIN_PRODUCT) {
              const double2 w = __ldg(reinterpret_cast<const double2 *>(in1 + ro + 2 * m));
              z = make_double2(z.x * w.x, z.y * w.y);
            }
          } else {
            const int c0 = gidx(g, 2 * m + 1, J, k + 1);
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
      },
      [&](int t, double2 z) {
        const int l = t / M, m = t - l * M;
        res[l * ls + m] = z;
      });
  __syncthreads();
  if (POST) {
    static_assert(!POST || (L == 8 && N1 % 4 == 0 && 8 * N1 <= F4_THREADS),
                  "8 lines x 4 columns per warp");
    // step 1: N1-point transforms of the stride-N2 subsequences
    for (int it = threadIdx.x; it < L * N2; it += blockDim.x) {
      const int l = it / N2, j2 = it - l * N2;
      double2 v[N1];
#pragma unroll
      for (int j1 = 0; j1 < N1; j1++) v[j1] = res[l * ls + j1 * N2 + j2];
      reg_fft<N1, false>(v, tw, N2);
      double2 *row = buf + l * LS1 + j2;
#pragma unroll
      for (int k1 = 0; k1 < N1; k1++) row[k1 * P] = k1 == 0 ? v[0] : cmul(v[k1], tw[j2 * k1]);
    }
    __syncthreads();
    // step 2 with the output pass, on N1/4 warps
    if (threadIdx.x < 8 * N1) {
      const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
      const int l = lane & 7, qd = lane >> 3;
      const int a = 2 * w + (qd >> 1);
      const int k1 = (w == 0 && qd == 1) ? N1 / 2 : ((qd & 1) ? N1 - a : a);
      const bool self0 = k1 == 0, selfh = k1 == N1 / 2;
      const double2 *col = buf + l * LS1 + k1 * P;
      double2 v[N2];
#pragma unroll
      for (int j2 = 0; j2 < N2; j2++) v[j2] = col[j2];
      reg_fft<N2, false>(v, tw, N1);
      const int Lv = min(L, g.nz - k0);
      const bool store = l < Lv;
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) {
        const double2 mine = v[N2 - 1 - k2];
        double2 other;
        other.x = __shfl_xor_sync(0xffffffffu, mine.x, 8);
        other.y = __shfl_xor_sync(0xffffffffu, mine.y, 8);
        const double2 zm = self0 ? v[(N2 - k2) % N2] : (selfh ? mine : other);
        const int kx = k1 + N1 * k2;
        const double2 zk = v[k2], zc = cconj(zm);
        const double2 e = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
        const double2 d = csub(zk, zc);
        const double2 o = make_double2(0.5 * d.y, -0.5 * d.x);
        if (store) S[sidx(g, kx, j, k0 + l)] = cadd(e, cmul(tn[kx], o));
        if (self0 && k2 == 0 && store) {  // kx = M from Z[0]
          const double2 z0c = cconj(zk);
          const double2 e0 = make_double2(0.5 * (zk.x + z0c.x), 0.5 * (zk.y + z0c.y));
          const double2 d0 = csub(zk, z0c);
          const double2 o0 = make_double2(0.5 * d0.y, -0.5 * d0.x);
          S[sidx(g, M, j, k0 + l)] = cadd(e0, cmul(tn[M], o0));
        }
      }
    }
    return;
  }
  // step 1 reads res, step 2 (after the barrier inside) overwrites it
  fft4_lines<N1, N2, false>([&](int l, int m) { return res[l * ls + m]; },
                            [&](int l, int e, double2 v) { res[l * ls + e] = v; }, buf, L, tw);
  // post-process (X = E + w^k O) and store S(kx, j, k0 + l), l fastest
  const int Lv = min(L, g.nz - k0);
  for (int t = threadIdx.x; t < L * (M + 1); t += blockDim.x) {
    const int kx = t / L, l = t - kx * L;
    if (l >= Lv) continue;
    const double2 zk = res[l * ls + (kx == M ? 0 : kx)];
    const double2 zc = cconj(res[l * ls + (kx == 0 ? 0 : M - kx)]);
    const double2 e = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
    const double2 d = csub(zk, zc);
    const double2 o = make_double2(0.5 * d.y, -0.5 * d.x);
    S[sidx(g, kx, j, k0 + l)] = cadd(e, cmul(tn[kx], o));
  }
}

// Inverse real FFT along x of one tile (see k_irfftx): the L lines
// (row j, kz = k0..k0+L-1; Lv valid) of X are in zb (pitch M+2).  The pairs
// (k, M-k) are pre-processed in place, then the four-step inverse writes
// the field in its step 2 (OUTMODE as in k_irfftx).  Ends with a barrier.
// PAIRS (L = 16, N2 % 4 == 0): the pre-processing runs inside the first
// FFT pass instead of as a pass of its own.  Thread (line l, column j2)
// needs X[j1 N2 + j2] and X[M - j1 N2 - j2], which is element N1-1-j1 of
// column N2-j2; columns j2 and N2-j2 share a warp (8 lines x 4 columns) and
// swap those values by shuffle; columns 0 and N2/2 are their own partners.
// The transpose buffer then has N1*P + 1 values per line.
template <int N1, int N2, int OUTMODE, bool PAIRS = false>
__device__ __forceinline__ void irfftx4_tile(const Geo &g, double2 *zb, int L, int Lv, int j,
                                             int k0, double *__restrict__ out, double2 *buf,
                                             const double2 *tw, const double2 *tn) {
  constexpr int M = N1 * N2;
  constexpr int ls = M + 2;
  // Z[k] = E[k] + i O[k], E = (X[k] + conj X[M-k])/2,
  // O = (X[k] - conj X[M-k]) conj(w^k)/2; one thread per pair (k, M-k)
  constexpr int half = M / 2 + 1;
  for (int t = threadIdx.x; !PAIRS && t < L * half; t += blockDim.x) {
    const int l = t / half, k = t - l * half;
    double2 *X = zb + l * ls;
    if (k == 0) {
      const double a = X[0].x, b = X[M].x;
      X[0] = make_double2(0.5 * (a + b), 0.5 * (a - b));
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
  const double sc = 1.0 / M;
  const int J = j + 1;
  const bool row_edge = (J == 1) | (J >= g.ny - 1);
  auto line_edge = [&](int l) {
    const int K = k0 + l + 1;
    return row_edge | (K == 1) | (K == g.nz);
  };
  auto store = [&](int l, int m, double2 z) {
        if (l >= Lv) return;
        const double x0 = z.x * sc, x1 = z.y * sc;
        const int K = k0 + l + 1;
        if (OUTMODE == ROUT_REAL) {
          double *row = out + (long long)g.nx * (j + (long long)g.ny * (K - 1));
          *reinterpret_cast<double2 *>(row + 2 * m) = make_double2(x0, x1);
        } else if (OUTMODE == ROUT_INTERIOR) {
          const int c0 = gidx(g, 2 * m + 1, J, K);
          out[c0] = x0;
          out[c0 + 1] = x1;
        } else {
          // ghost images only on edge lines and at the two ends of a line
          const int c0 = gidx(g, 2 * m + 1, J, K);
          out[c0] = x0;
          out[c0 + 1] = x1;
          if (line_edge(l) | (m == 0) | (m == M - 1)) {
            store_images_core(out, g.nx, g.ny, g.nz, g.NX, g.NY, g.wall, 2 * m + 1, J, K, x0, STAG_P);
            store_images_core(out, g.nx, g.ny, g.nz, g.NX, g.NY, g.wall, 2 * m + 2, J, K, x1, STAG_P);
          }
        }
      };
  if (!PAIRS) {
    __syncthreads();
    fft4_lines<N1, N2, true>([&](int l, int e) { return zb[l * ls + e]; }, store, buf, L, tw);
    return;
  }
  static_assert(!PAIRS || N2 % 4 == 0, "columns in pairs, 4 per warp");
  constexpr int P = fft4_pitch<N2>();
  constexpr int LS1 = N1 * P + 1;
  // step 1: 8 lines x 4 columns per warp, L/8 groups of N2/4 warps
  for (int it = threadIdx.x; it < 8 * N2 * (L / 8); it += blockDim.x) {
    const int lane = it & 31, w = it >> 5;
    const int grp = w / (N2 / 4), wg = w - grp * (N2 / 4);
    const int l = grp * 8 + (lane & 7), qd = lane >> 3;
    const int a = 2 * wg + (qd >> 1);
    const int j2 = (wg == 0 && qd == 1) ? N2 / 2 : ((qd & 1) ? N2 - a : a);
    const bool self0 = j2 == 0, selfh = j2 == N2 / 2;
    const double2 *X = zb + l * ls;
    double2 x[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) x[j1] = X[j1 * N2 + j2];
    const double2 xM = X[M];
    double2 v[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) {
      const double2 mine = x[N1 - 1 - j1];
      double2 other;
      other.x = __shfl_xor_sync(0xffffffffu, mine.x, 8);
      other.y = __shfl_xor_sync(0xffffffffu, mine.y, 8);
      const int k = j1 * N2 + j2;
      const double2 a0 = x[j1];
      if (self0 && j1 == 0) {  // k = 0 pairs with X[M]
        v[0] = make_double2(0.5 * (a0.x + xM.x), 0.5 * (a0.x - xM.x));
        continue;
      }
      const double2 b = self0 ? x[(N1 - j1) % N1] : (selfh ? mine : other);
      const double2 bc = cconj(b);
      const double2 e = cscale(cadd(a0, bc), 0.5);
      const double2 o = cmul(cscale(csub(a0, bc), 0.5), cconj(tn[k]));
      v[j1] = make_double2(e.x - o.y, e.y + o.x);
    }
    reg_fft<N1, true>(v, tw, N2);
    double2 *row = buf + l * LS1 + j2;
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) row[k1 * P] = k1 == 0 ? v[0] : cmul(v[k1], cconj(tw[j2 * k1]));
  }
  __syncthreads();
  // step 2 as in fft4_lines
  for (int it = threadIdx.x; it < L * N1; it += blockDim.x) {
    const int l = it / N1, k1 = it - l * N1;
    double2 v[N2];
    const double2 *col = buf + l * LS1 + k1 * P;
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++) v[j2] = col[j2];
    reg_fft<N2, true>(v, tw, N1);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) store(l, k1 + N1 * k2, v[k2]);
  }
  __syncthreads();
}

// Inverse real FFT along x, one tile of L lines per CTA.
// PAIRS: the pair pre-processing inside the first FFT pass (irfftx4_tile),
// where N2 % 4 == 0 and L % 8 == 0; elsewhere the separate pass.
template <int N1, int N2, int L, int OUTMODE, bool PAIRS = false>
__global__ void __launch_bounds__(F4_THREADS, 2) k_irfftx4(Geo g, const double2 *__restrict__ S,
                                                           double *__restrict__ out,
                                                           const double2 *__restrict__ twM,
                                                           const double2 *__restrict__ twN) {
  constexpr int M = N1 * N2;
  constexpr int ls = M + 2;
  extern __shared__ double2 smem[];
  double2 *zb = smem;
  double2 *buf = zb + L * ls;
  double2 *tw = buf + L * (N1 * fft4_pitch<N2>() + 1);
  double2 *tn = tw + M;
  const int ngrp = (g.nz + L - 1) / L;
  const int grp = blockIdx.x % ngrp;
  const int j = blockIdx.x / ngrp;
  const int k0 = grp * L;
  const int Lv = min(L, g.nz - k0);
  for (int t = threadIdx.x; t < M; t += blockDim.x) tw[t] = twM[t];
  for (int t = threadIdx.x; t <= M; t += blockDim.x) tn[t] = twN[t];
  batched_copy<16>(  // one round of loads for L = 16 lines of 193
      L * (M + 1),
      [&](int t) {
        const int kx = t / L, l = t - kx * L;
        return l < Lv ? S[sidx(g, kx, j, k0 + l)] : make_double2(0.0, 0.0);
      },
      [&](int t, double2 v) {
        const int kx = t / L, l = t - kx * L;
        zb[l * ls + kx] = v;
      });
  __syncthreads();
  irfftx4_tile<N1, N2, OUTMODE, PAIRS && N2 % 4 == 0 && L % 8 == 0>(g, zb, L, Lv, j, k0, out,
                                                                      buf, tw, tn);
}

}  // namespace dnsb
