// ysolve.cuh -- the wall-normal Poisson solve with every y-line split
// across 32 threads.
//
// thomas_kernel! (src/poisson.jl:14-41) solves, per (kx, kz) line,
//   a_j x_{j-1} + (b_j + lambda) x_j + c_j x_{j+1} = d_j,  j = 0..ny-1,
// with the mean mode (lambda == 0) pinned by replacing row 0 with x_0 = 0.
// One thread per line (k_thomas) leaves too few threads in flight and must
// park d' and c' in HBM.  Here a block holds TY_LINES lines (consecutive kz,
// so every row is one coalesced segment) x TY_CHUNKS chunks of MR rows; a
// thread keeps its chunk in registers:
//   c' recurrence  c'_j = c_j / beta_j, beta_j = b_j - a_j c'_{j-1}: it
//      depends on the line's lambda only, so the c' entering every chunk
//      is computed once per context by the sequential recurrence
//      (k_ythomas_entries) and read from a table of TY_CHUNKS values per
//      line.  (Carrying it across chunks as 2x2 matrix products instead
//      loses two digits on the nearly singular low modes.)
//   forward  d'_j = (d_j - a_j d'_{j-1}) / beta_j is affine in the carried
//      d'; the chunks' maps (Z, G) are composed by one warp per line (a
//      shuffle scan over shared memory), then the sweep is rerun from the
//      true carry;
//   backward  x_j = d'_j - c'_j x_{j+1}, the same way with (Y, H).
// Every element is read from and written to HBM once and no work array is
// needed.  Algebraically this is the reference's Thomas algorithm.
#pragma once
#include "common.cuh"

namespace dnsb {

constexpr int TY_CHUNKS = 32;
constexpr int TY_LINES = 8;

// Rows per chunk for ny rows (a value with an instantiated kernel), or 0
// when ny is beyond the register-resident range.
inline int ythomas_rows(int ny) {
  static const int mr[] = {1, 2, 3, 4, 6, 8, 12, 16};
  for (int m : mr)
    if (m * TY_CHUNKS >= ny) return m;
  return 0;
}

// Composes the per-chunk affine maps v -> A + B v (A complex, B real) of
// TY_LINES lines, in place: warp w scans line w with lane = chunk
// (Kogge-Stone over shuffles).  Forward (REV = false), m[k][w] becomes the
// value entering chunk k (maps 0..k-1 applied to 0); backward (REV = true)
// the value entering chunk k from above (maps TY_CHUNKS-1..k+1 applied to
// 0).  Call with all TY_LINES warps of the block, between barriers.
template <bool REV>
__device__ __forceinline__ void ythomas_scan(double4 (*m)[TY_LINES + 1]) {
  static_assert(TY_CHUNKS == 32, "one lane per chunk");
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int w = tid >> 5, lane = tid & 31;
  if (w >= TY_LINES) return;
  const double4 v = m[lane][w];
  double ar = v.x, ai = v.y, b = v.z;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double pr = REV ? __shfl_down_sync(0xffffffffu, ar, o) : __shfl_up_sync(0xffffffffu, ar, o);
    const double pi = REV ? __shfl_down_sync(0xffffffffu, ai, o) : __shfl_up_sync(0xffffffffu, ai, o);
    const double pb = REV ? __shfl_down_sync(0xffffffffu, b, o) : __shfl_up_sync(0xffffffffu, b, o);
    if (REV ? lane + o < 32 : lane >= o) {
      ar = fma(b, pr, ar);
      ai = fma(b, pi, ai);
      b *= pb;
    }
  }
  // exclusive: the value from the neighbouring chunk's inclusive result
  double er = REV ? __shfl_down_sync(0xffffffffu, ar, 1) : __shfl_up_sync(0xffffffffu, ar, 1);
  double ei = REV ? __shfl_down_sync(0xffffffffu, ai, 1) : __shfl_up_sync(0xffffffffu, ai, 1);
  if (REV ? lane == 31 : lane == 0) er = ei = 0.0;
  m[lane][w] = make_double4(er, ei, 0.0, 0.0);
}

// The c' entering each chunk of MR rows, for every line: one thread per
// line runs the reference's sequential recurrence (poisson.jl:20-30).
// cin[line * TY_CHUNKS + k] = c'_{k MR - 1} (0 for k = 0).
__global__ void k_ythomas_entries(Geo g, int mr, double *__restrict__ cin,
                                  const double *__restrict__ ay, const double *__restrict__ by,
                                  const double *__restrict__ cy, const double *__restrict__ lam1,
                                  const double *__restrict__ lam3) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)g.nz * g.nkx) return;
  const int kz = (int)(t % g.nz), kx = (int)(t / g.nz);
  const double lam = lam1[kx] + lam3[kz];
  const bool pin = lam == 0.0;
  double *out = cin + t * TY_CHUNKS;
  double cprev = 0.0;
  for (int k = 0; k < TY_CHUNKS; k++) {
    out[k] = cprev;
    for (int j = k * mr; j < min(g.ny, (k + 1) * mr); j++) {
      if (pin && j == 0) {
        cprev = 0.0;
      } else {
        const double beta = (by[j] + lam) - ay[j] * cprev;
        cprev = cy[j] / beta;
      }
    }
  }
}

// dynamic shared memory of k_ythomas<MR>
constexpr size_t ythomas_smem(int mr) { return sizeof(double) * (size_t)mr * TY_LINES * TY_CHUNKS; }

template <int MR>
__global__ void __launch_bounds__(TY_LINES *TY_CHUNKS, MR <= 8 ? 3 : 1)
    k_ythomas(Geo g, double2 *__restrict__ S, const double *__restrict__ cin,
              const double *__restrict__ ay, const double *__restrict__ by,
              const double *__restrict__ cy, const double *__restrict__ lam1,
              const double *__restrict__ lam3) {
  // chunk maps, one row of lines per chunk padded by one entry so that the
  // scan's lane-per-chunk reads spread over all banks
  __shared__ double4 za[TY_CHUNKS][TY_LINES + 1];  // forward (Z.re, Z.im, G)
  __shared__ double4 yb[TY_CHUNKS][TY_LINES + 1];  // backward (Y.re, Y.im, H)
  const int i = threadIdx.x, ck = threadIdx.y;
  const int ny = g.ny, nz = g.nz;
  const long long nl = (long long)nz * g.nkx;
  const long long t = (long long)blockIdx.x * TY_LINES + i;
  const bool act = t < nl;
  const int kz = act ? (int)(t % nz) : 0, kx = act ? (int)(t / nz) : 0;
  const double lam = __ldg(lam1 + kx) + __ldg(lam3 + kz);
  const bool pin = lam == 0.0;
  const long long st = nz;
  double2 *x = S + sidx(g, kx, 0, kz);
  const int s0 = ck * MR;
  // row j of the (pinned) system: a, b + lambda, c
  auto coefs = [&](int j, double &a, double &b, double &c) {
    if (pin && j == 0) {
      a = 0.0;
      b = 1.0;
      c = 0.0;
    } else {
      a = __ldg(ay + j);
      b = __ldg(by + j) + lam;
      c = __ldg(cy + j);
    }
  };
  double2 d[MR];
#pragma unroll
  for (int r = 0; r < MR; r++) {
    const int j = s0 + r;
    d[r] = (act && j < ny) ? x[j * st] : make_double2(0.0, 0.0);
  }
  if (pin && s0 == 0) d[0] = make_double2(0.0, 0.0);
  double cprev = act ? __ldg(cin + t * TY_CHUNKS + ck) : 0.0;
  // forward: 1/beta_j of the chunk (kept in shared memory, one column per
  // thread; c'_j = c_j / beta_j is re-formed where needed), its affine map
  // d'_e = Z + G d'_{s-1}
  extern __shared__ double ibs[];  // [MR][TY_LINES * TY_CHUNKS] (dynamic: ythomas_smem)
  const int tid = i + TY_LINES * ck;
  constexpr int NT = TY_LINES * TY_CHUNKS;
  auto cpj = [&](int r) {  // c'_j of row j = s0 + r from the stored 1/beta_j
    const int j = s0 + r;
    const double c = (pin && j == 0) ? 0.0 : __ldg(cy + j);
    return c * ibs[r * NT + tid];
  };
  {
    double2 z = make_double2(0.0, 0.0);
    double G = 1.0;
#pragma unroll
    for (int r = 0; r < MR; r++) {
      const int j = s0 + r;
      if (j < ny) {
        double a, b, c;
        coefs(j, a, b, c);
        const double beta = b - a * cprev;
        const double rb = 1.0 / beta;
        cprev = c * rb;
        ibs[r * NT + tid] = rb;
        z = make_double2((d[r].x - a * z.x) * rb, (d[r].y - a * z.y) * rb);
        G *= -a * rb;
      } else {
        ibs[r * NT + tid] = 0.0;
      }
    }
    za[ck][i] = make_double4(z.x, z.y, G, 0.0);
  }
  __syncthreads();
  ythomas_scan<false>(za);
  __syncthreads();
  {
    const double4 m = za[ck][i];
    double2 dp = make_double2(m.x, m.y);  // true d'_{s-1}
#pragma unroll
    for (int r = 0; r < MR; r++) {
      const int j = s0 + r;
      if (j < ny) {
        const double a = (pin && j == 0) ? 0.0 : __ldg(ay + j);
        const double rb = ibs[r * NT + tid];
        dp = make_double2((d[r].x - a * dp.x) * rb, (d[r].y - a * dp.y) * rb);
        d[r] = dp;
      }
    }
  }
  // backward: the chunk's map x_s = Y + H x_{e+1}
  {
    double2 y = make_double2(0.0, 0.0);
    double H = 1.0;
#pragma unroll
    for (int r = MR - 1; r >= 0; r--) {
      const int j = s0 + r;
      if (j < ny) {
        const double cpr = cpj(r);
        y = make_double2(d[r].x - cpr * y.x, d[r].y - cpr * y.y);
        H *= -cpr;
      }
    }
    yb[ck][i] = make_double4(y.x, y.y, H, 0.0);
  }
  __syncthreads();
  ythomas_scan<true>(yb);
  __syncthreads();
  const double4 mb = yb[ck][i];
  double2 xn = make_double2(mb.x, mb.y);  // true x_{e+1}
#pragma unroll
  for (int r = MR - 1; r >= 0; r--) {
    const int j = s0 + r;
    if (j < ny) {
      const double cpr = cpj(r);
      xn = make_double2(d[r].x - cpr * xn.x, d[r].y - cpr * xn.y);
      if (act) x[j * st] = xn;
    }
  }
}

}  // namespace dnsb
