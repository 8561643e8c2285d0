// zyz.cuh -- the spectral core of the wall-bounded Poisson solve in one
// kernel per kx plane: forward z-FFT, Thomas solve along y, inverse z-FFT.
//
// poisson! (src/poisson.jl:122-146) runs, between the x transforms,
//   fft along z (:131), thomas_kernel! along y for every (kx, kz) line
//   (:14-41, :133), ifft along z (:135)
// and each of the three reads and writes the whole half spectrum.  A kx
// plane (ny x nz complex values, 1.5 MB at 256 x 384) is too large for one
// SM but fits a thread-block cluster: CTA c of the cluster holds y rows
// [32c, 32c+32) of the plane in shared memory (204.8 KB at nz = 384), and
//   1. transforms its 32 z-lines with the four-step scheme of fft4.cuh,
//      reading them from HBM in step 1 and leaving the spectrum in place in
//      the transposed order (position k1*P + k2 of a row holds
//      X[k1 + N1*k2]; P = N2 + 1 keeps the runs on distinct banks);
//   2. solves every line kz over its 32 rows as one chunk of the chunked
//      Thomas algorithm of ysolve.cuh: the c' entering the chunk comes from
//      the per-context table (sequential recurrence, k_ythomas_entries with
//      32-row chunks), the forward and backward affine carries (Z, G) and
//      (Y, H) of the lower / upper chunks are read from the peer CTAs'
//      shared memory (distributed shared memory) after a cluster barrier,
//      and the sweeps are rerun from the true carries; 1/beta of the 32
//      rows stays in registers;
//   3. runs the four-step inverse from the transposed order back to the
//      natural one, writing the lines to HBM in its last step (x 1/nz).
// The plane is read from and written to HBM once: 2 passes of the half
// spectrum instead of 6.  Algebraically this is the reference's sequence
// (the same transforms and the same Thomas recurrences).
#pragma once
#include <cooperative_groups.h>

#include "fft4.cuh"
#include "ysolve.cuh"

namespace dnsb {

constexpr int ZYZ_ROWS = 32;     // y rows per CTA (one Thomas chunk)
constexpr int ZYZ_MAXC = 8;      // CTAs per cluster (the portable limit)
constexpr int ZYZ_THREADS = 384; // one z-line per thread in the Thomas phase (nz <= 384)

// dynamic shared memory: the rows, nz twiddles, the forward and backward
// chunk maps (3 doubles per line each)
template <int N1, int N2>
constexpr size_t zyz_smem() {
  return sizeof(double2) * ((size_t)ZYZ_ROWS * N1 * fft4_pitch<N2>() + (size_t)N1 * N2) +
         sizeof(double) * 6 * (size_t)N1 * N2;
}

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// One cluster of C = ny / 32 CTAs per kx plane (grid = nkx * C); rows of S
// are nz contiguous values (sidx: kz + nz (j + ny kx)).  cin = the c'
// entering each 32-row chunk of every (kx, kz) line (TY_CHUNKS per line).
template <int N1, int N2>
__global__ void __launch_bounds__(ZYZ_THREADS, 1)
    k_zyz(Geo g, double2 *__restrict__ S, const double *__restrict__ cin,
          const double *__restrict__ ay, const double *__restrict__ by,
          const double *__restrict__ cy, const double *__restrict__ lam1,
          const double *__restrict__ lam3, const double2 *__restrict__ twz) {
  namespace cg = cooperative_groups;
  constexpr int N = N1 * N2;  // nz
  constexpr int P = fft4_pitch<N2>();
  constexpr int RP = N1 * P;  // row pitch (complex) in shared memory
  constexpr int R = ZYZ_ROWS;
  static_assert(N <= ZYZ_THREADS, "one line per thread in the Thomas phase");
  extern __shared__ __align__(16) double2 zsm[];
  double2 *pl = zsm;                                 // [R][RP]
  double2 *tw = pl + R * RP;                         // [N]
  double *zg = reinterpret_cast<double *>(tw + N);   // [3][N] forward maps (Z.re, Z.im, G)
  double *yh = zg + 3 * N;                           // [3][N] backward maps (Y.re, Y.im, H)
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks();
  const int c = (int)cl.block_rank();
  const int kx = blockIdx.x / C;
  const int j0 = c * R;
  double2 *src = S + ((long long)kx * g.ny + j0) * N;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = twz[t];
  __syncthreads();

  // ---- forward z-FFT: step 1 from HBM, step 2 in place (transposed order)
  for (int it = threadIdx.x; it < R * N2; it += blockDim.x) {
    const int l = it / N2, j2 = it - l * N2;
    const double2 *line = src + (long long)l * N;
    double2 v[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) v[j1] = line[j1 * N2 + j2];
    reg_fft<N1, false>(v, tw, N2);
    double2 *row = pl + l * RP + j2;
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) row[k1 * P] = k1 == 0 ? v[0] : cmul(v[k1], tw[j2 * k1]);
  }
  __syncthreads();
  for (int it = threadIdx.x; it < R * N1; it += blockDim.x) {
    const int l = it / N1, k1 = it - l * N1;
    double2 *col = pl + l * RP + k1 * P;
    double2 v[N2];
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++) v[j2] = col[j2];
    reg_fft<N2, false>(v, tw, N1);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) col[k2] = v[k2];
  }
  __syncthreads();

  // ---- Thomas along y: this CTA is chunk c of every line
  {
    const int t = threadIdx.x;
    const bool act = t < N;
    const int k1 = act ? t / N2 : 0, k2 = act ? t - k1 * N2 : 0;
    const int kz = k1 + N1 * k2;
    double2 *x = pl + k1 * P + k2;  // row r of this line at x[r * RP]
    const double lam = __ldg(lam1 + kx) + __ldg(lam3 + kz);
    const bool pin = lam == 0.0;
    double cprev = act ? __ldg(cin + ((long long)kx * N + kz) * TY_CHUNKS + c) : 0.0;
    double ib[R];
    // forward, local map d'_end = Z + G d'_in; 1/beta of the rows kept
    {
      double2 z = make_double2(0.0, 0.0);
      double G = 1.0;
#pragma unroll
      for (int r = 0; r < R; r++) {
        const int j = j0 + r;
        const bool p0 = pin && j == 0;
        const double a = p0 ? 0.0 : __ldg(ay + j);
        const double b = p0 ? 1.0 : __ldg(by + j) + lam;
        const double cc = p0 ? 0.0 : __ldg(cy + j);
        const double rb = 1.0 / (b - a * cprev);
        cprev = cc * rb;
        ib[r] = rb;
        const double2 d = p0 ? make_double2(0.0, 0.0) : x[r * RP];
        z = make_double2((d.x - a * z.x) * rb, (d.y - a * z.y) * rb);
        G *= -a * rb;
      }
      if (act) {
        zg[t] = z.x;
        zg[N + t] = z.y;
        zg[2 * N + t] = G;
      }
    }
    cl.sync();
    // the true d' entering this chunk: maps of chunks 0..c-1 applied to 0
    double2 dp = make_double2(0.0, 0.0);
    if (act) {
      for (int i = 0; i < c; i++) {
        const double *m = cl.map_shared_rank(zg, i);
        const double gi = m[2 * N + t];
        dp = make_double2(fma(gi, dp.x, m[t]), fma(gi, dp.y, m[N + t]));
      }
    }
    // forward rerun from the true carry (d' in place)
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int j = j0 + r;
      const bool p0 = pin && j == 0;
      const double a = p0 ? 0.0 : __ldg(ay + j);
      const double2 d = p0 ? make_double2(0.0, 0.0) : x[r * RP];
      dp = make_double2((d.x - a * dp.x) * ib[r], (d.y - a * dp.y) * ib[r]);
      if (act) x[r * RP] = dp;
    }
    // backward, local map x_start = Y + H x_above
    {
      double2 y = make_double2(0.0, 0.0);
      double H = 1.0;
#pragma unroll
      for (int r = R - 1; r >= 0; r--) {
        const int j = j0 + r;
        const double cpr = ((pin && j == 0) ? 0.0 : __ldg(cy + j)) * ib[r];
        const double2 d = x[r * RP];
        y = make_double2(d.x - cpr * y.x, d.y - cpr * y.y);
        H *= -cpr;
      }
      if (act) {
        yh[t] = y.x;
        yh[N + t] = y.y;
        yh[2 * N + t] = H;
      }
    }
    cl.sync();
    // the true x above this chunk: maps of chunks C-1..c+1 applied to 0
    double2 xn = make_double2(0.0, 0.0);
    if (act) {
      for (int i = C - 1; i > c; i--) {
        const double *m = cl.map_shared_rank(yh, i);
        const double hi = m[2 * N + t];
        xn = make_double2(fma(hi, xn.x, m[t]), fma(hi, xn.y, m[N + t]));
      }
    }
    cluster_arrive();  // peers' maps read: they may exit once everyone has arrived
#pragma unroll
    for (int r = R - 1; r >= 0; r--) {
      const int j = j0 + r;
      const double cpr = ((pin && j == 0) ? 0.0 : __ldg(cy + j)) * ib[r];
      const double2 d = x[r * RP];
      xn = make_double2(d.x - cpr * xn.x, d.y - cpr * xn.y);
      if (act) x[r * RP] = xn;
    }
  }
  __syncthreads();

  // ---- inverse z-FFT: step 1 in place from the transposed order, step 2 to HBM
  for (int it = threadIdx.x; it < R * N1; it += blockDim.x) {
    const int l = it / N1, k1 = it - l * N1;
    double2 *col = pl + l * RP + k1 * P;
    double2 v[N2];
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) v[k2] = col[k2];
    reg_fft<N2, true>(v, tw, N1);
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++) col[j2] = (k1 == 0 || j2 == 0) ? v[j2] : cmul(v[j2], cconj(tw[j2 * k1]));
  }
  __syncthreads();
  const double sc = 1.0 / N;
  for (int it = threadIdx.x; it < R * N2; it += blockDim.x) {
    const int l = it / N2, j2 = it - l * N2;
    const double2 *row = pl + l * RP + j2;
    double2 v[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) v[k1] = row[k1 * P];
    reg_fft<N1, true>(v, tw, N2);
    double2 *line = src + (long long)l * N;
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) line[j1 * N2 + j2] = cscale(v[j1], sc);
  }
  cluster_wait();
}


// ---- two CTAs per SM: 16-row chunks, clusters of ny/16 (up to 16, the
// non-portable size), 192 threads.  The rows are stored without padding
// (16 x nz complex = 96 KB at nz = 384) under a rotation swizzle: element
// (k1, k2) of a row sits at k1 N2 + (k2 + k1) mod N2, which keeps the runs
// of the second four-step pass on distinct banks; the twiddles are read
// from global memory (L1-resident) and the forward and backward chunk maps
// share one buffer behind an extra cluster barrier, so that two CTAs fit in
// one SM's shared memory and their load, transform and solve phases
// overlap.  Same algorithm and results as k_zyz.
constexpr int ZYZ2_ROWS = 16;
constexpr int ZYZ2_THREADS = 192;  // two z-lines per thread in the Thomas phase
constexpr int ZYZ2_MAXC = 16;

template <int N1, int N2>
constexpr size_t zyz2_smem() {
  return sizeof(double2) * (size_t)ZYZ2_ROWS * N1 * N2 + sizeof(double) * 3 * (size_t)N1 * N2;
}

template <int N1, int N2>
__global__ void __launch_bounds__(ZYZ2_THREADS, 2)
    k_zyz2(Geo g, double2 *__restrict__ S, const double *__restrict__ cin,
           const double *__restrict__ ay, const double *__restrict__ by,
           const double *__restrict__ cy, const double *__restrict__ lam1,
           const double *__restrict__ lam3, const double2 *__restrict__ tw) {
  namespace cg = cooperative_groups;
  constexpr int N = N1 * N2;  // nz
  constexpr int R = ZYZ2_ROWS;
  constexpr int LPT = (N + ZYZ2_THREADS - 1) / ZYZ2_THREADS;  // lines per thread (2 at 384)
  static_assert(LPT <= 2, "at most two lines per thread");
  extern __shared__ __align__(16) double2 zsm2[];
  double2 *pl = zsm2;                               // [R][N], swizzled
  double *mp = reinterpret_cast<double *>(pl + R * N);  // [3][N] chunk maps
  auto pos = [](int k1, int k2) { int r = k2 + k1; r -= r >= N2 ? N2 : 0; return k1 * N2 + r; };
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks();
  const int c = (int)cl.block_rank();
  const int kx = blockIdx.x / C;
  const int j0 = c * R;
  double2 *src = S + ((long long)kx * g.ny + j0) * N;

  // forward z-FFT step 1: N1-point transforms from HBM into the swizzled rows
  for (int it = threadIdx.x; it < R * N2; it += blockDim.x) {
    const int l = it / N2, j2 = it - l * N2;
    const double2 *line = src + (long long)l * N;
    double2 v[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) v[j1] = line[j1 * N2 + j2];
    reg_fft<N1, false>(v, tw, N2);
    double2 *row = pl + l * N;
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) row[pos(k1, j2)] = k1 == 0 ? v[0] : cmul(v[k1], __ldg(tw + j2 * k1));
  }
  __syncthreads();
  // step 2 in place: pos(k1, k2) of a row holds X[k1 + N1 k2]
  for (int it = threadIdx.x; it < R * N1; it += blockDim.x) {
    const int l = it / N1, k1 = it - l * N1;
    double2 *row = pl + l * N;
    double2 v[N2];
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++) v[j2] = row[pos(k1, j2)];
    reg_fft<N2, false>(v, tw, N1);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) row[pos(k1, k2)] = v[k2];
  }
  __syncthreads();

  // Thomas along y: this CTA is chunk c of every line; thread t owns the
  // lines at row positions t and t + blockDim.x
  {
    int p[LPT], kz[LPT];
    bool act[LPT];
    double lam[LPT], cprev[LPT];
    bool pin[LPT];
#pragma unroll
    for (int q = 0; q < LPT; q++) {
      p[q] = threadIdx.x + q * ZYZ2_THREADS;
      act[q] = p[q] < N;
      const int pp = act[q] ? p[q] : 0;
      const int k1 = pp / N2;
      int k2 = pp - k1 * N2 - k1;
      while (k2 < 0) k2 += N2;
      kz[q] = k1 + N1 * k2;
      lam[q] = __ldg(lam1 + kx) + __ldg(lam3 + kz[q]);
      pin[q] = lam[q] == 0.0;
      cprev[q] = act[q] ? __ldg(cin + ((long long)kx * N + kz[q]) * TY_CHUNKS + c) : 0.0;
    }
    double ib[LPT][R];
    double2 z[LPT];
    double G[LPT];
#pragma unroll
    for (int q = 0; q < LPT; q++) { z[q] = make_double2(0.0, 0.0); G[q] = 1.0; }
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int j = j0 + r;
      const double a0 = __ldg(ay + j), b0 = __ldg(by + j), c0 = __ldg(cy + j);
#pragma unroll
      for (int q = 0; q < LPT; q++) {
        const bool p0 = pin[q] && j == 0;
        const double a = p0 ? 0.0 : a0, b = p0 ? 1.0 : b0 + lam[q], cc = p0 ? 0.0 : c0;
        const double rb = 1.0 / (b - a * cprev[q]);
        cprev[q] = cc * rb;
        ib[q][r] = rb;
        const double2 d = p0 ? make_double2(0.0, 0.0) : pl[r * N + (act[q] ? p[q] : 0)];
        z[q] = make_double2((d.x - a * z[q].x) * rb, (d.y - a * z[q].y) * rb);
        G[q] *= -a * rb;
      }
    }
#pragma unroll
    for (int q = 0; q < LPT; q++)
      if (act[q]) { mp[p[q]] = z[q].x; mp[N + p[q]] = z[q].y; mp[2 * N + p[q]] = G[q]; }
    cl.sync();
    double2 dp[LPT];
#pragma unroll
    for (int q = 0; q < LPT; q++) {
      dp[q] = make_double2(0.0, 0.0);
      if (act[q])
        for (int i = 0; i < c; i++) {
          const double *m = cl.map_shared_rank(mp, i);
          const double gi = m[2 * N + p[q]];
          dp[q] = make_double2(fma(gi, dp[q].x, m[p[q]]), fma(gi, dp[q].y, m[N + p[q]]));
        }
    }
    cluster_arrive();  // forward maps read; the buffer is reused below
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int j = j0 + r;
      const double a0 = __ldg(ay + j);
#pragma unroll
      for (int q = 0; q < LPT; q++) {
        const bool p0 = pin[q] && j == 0;
        const double a = p0 ? 0.0 : a0;
        double2 *x = pl + r * N + (act[q] ? p[q] : 0);
        const double2 d = p0 ? make_double2(0.0, 0.0) : *x;
        dp[q] = make_double2((d.x - a * dp[q].x) * ib[q][r], (d.y - a * dp[q].y) * ib[q][r]);
        if (act[q]) *x = dp[q];
      }
    }
    double2 y[LPT];
    double Hh[LPT];
#pragma unroll
    for (int q = 0; q < LPT; q++) { y[q] = make_double2(0.0, 0.0); Hh[q] = 1.0; }
#pragma unroll
    for (int r = R - 1; r >= 0; r--) {
      const int j = j0 + r;
      const double c0 = __ldg(cy + j);
#pragma unroll
      for (int q = 0; q < LPT; q++) {
        const double cpr = ((pin[q] && j == 0) ? 0.0 : c0) * ib[q][r];
        const double2 d = pl[r * N + (act[q] ? p[q] : 0)];
        y[q] = make_double2(d.x - cpr * y[q].x, d.y - cpr * y[q].y);
        Hh[q] *= -cpr;
      }
    }
    cluster_wait();  // every peer has read the forward maps
#pragma unroll
    for (int q = 0; q < LPT; q++)
      if (act[q]) { mp[p[q]] = y[q].x; mp[N + p[q]] = y[q].y; mp[2 * N + p[q]] = Hh[q]; }
    cl.sync();
    double2 xn[LPT];
#pragma unroll
    for (int q = 0; q < LPT; q++) {
      xn[q] = make_double2(0.0, 0.0);
      if (act[q])
        for (int i = C - 1; i > c; i--) {
          const double *m = cl.map_shared_rank(mp, i);
          const double hi = m[2 * N + p[q]];
          xn[q] = make_double2(fma(hi, xn[q].x, m[p[q]]), fma(hi, xn[q].y, m[N + p[q]]));
        }
    }
    cluster_arrive();  // peers' maps read: they may exit once everyone has arrived
#pragma unroll
    for (int r = R - 1; r >= 0; r--) {
      const int j = j0 + r;
      const double c0 = __ldg(cy + j);
#pragma unroll
      for (int q = 0; q < LPT; q++) {
        const double cpr = ((pin[q] && j == 0) ? 0.0 : c0) * ib[q][r];
        double2 *x = pl + r * N + (act[q] ? p[q] : 0);
        const double2 d = *x;
        xn[q] = make_double2(d.x - cpr * xn[q].x, d.y - cpr * xn[q].y);
        if (act[q]) *x = xn[q];
      }
    }
  }
  __syncthreads();

  // inverse z-FFT: step 1 in place per row run, step 2 to HBM (x 1/nz)
  for (int it = threadIdx.x; it < R * N1; it += blockDim.x) {
    const int l = it / N1, k1 = it - l * N1;
    double2 *row = pl + l * N;
    double2 v[N2];
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) v[k2] = row[pos(k1, k2)];
    reg_fft<N2, true>(v, tw, N1);
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++)
      row[pos(k1, j2)] = (k1 == 0 || j2 == 0) ? v[j2] : cmul(v[j2], cconj(__ldg(tw + j2 * k1)));
  }
  __syncthreads();
  const double sc = 1.0 / N;
  for (int it = threadIdx.x; it < R * N2; it += blockDim.x) {
    const int l = it / N2, j2 = it - l * N2;
    const double2 *row = pl + l * N;
    double2 v[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) v[k1] = row[pos(k1, j2)];
    reg_fft<N1, true>(v, tw, N2);
    double2 *line = src + (long long)l * N;
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) line[j1 * N2 + j2] = cscale(v[j1], sc);
  }
  cluster_wait();
}

}  // namespace dnsb
