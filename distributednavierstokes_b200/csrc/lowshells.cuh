// lowshells.cuh -- the shell-clamp forcing of a periodic FV box for the
// lowest shells by direct partial Fourier sums instead of 3-D FFTs.
//
// shellforcing (src/spectral/forcing.jl:37-56) only touches the modes with
// floor(|k|) < nb, nb <= 4: at most 4 x 7 x 7 of the half spectrum.  Their
// coefficients u_hat(k) = sum_x u(x) e^{-i k.x} (the unnormalised FFT of the
// interior, as the transform path computes them) are formed separably:
//   1. per (y, z) line, the x-sums for kx = 0..KM (one read of the field;
//      a warp per line, lanes striding x, shuffle reduction in a fixed order);
//   2. the y-sums (ky = -KM..KM) and z-sums (kz = -KM..KM), a block per
//      output row with fixed-order tree reductions;
//   3. one block: the shell energies (1/2 w |u_hat|^2 / N^2, w the rfft
//      double count), the clamp factors f = sqrt(eref / E), the corrections
//      G(k) = (f(shell) - 1) u_hat(k) / N and their z-sums back to physical z;
//   4. per (y, z) line, u += Re sum_k w G(k) e^{i k.x} (the y-sum of 2KM+1
//      terms per line, then the x-sum per point) and the periodic ghost
//      images are rewritten.
// Two passes over each component instead of three forward and three
// inverse 3-D transforms.  KM = nb - 1 <= 3 and 2 KM < n in every direction.
#pragma once
#include "common.cuh"
#include "fft.cuh"

namespace dnsb {

constexpr int LS_KX = 4;             // kx = 0..3
constexpr int LS_KY = 7;             // ky, kz = -3..3
constexpr int LS_LINES = 8;          // (y, z) lines per CTA of 256 threads

// the phases e^{+2 pi i r / n} = (cos, sin) for r = 0..n-1 of one direction,
// formed once per context (the expression the partial sums evaluated per
// point before)
__global__ void k_ls_phases(int n, double2 *__restrict__ ph) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    double sn, cs;
    sincospi(2.0 * (double)i / (double)n, &sn, &cs);
    ph[i] = make_double2(cs, sn);
  }
}

// e^{-2 pi i m / n} (sign -1) or e^{+2 pi i m / n} (sign +1) for integer m
// (|m| < 2^31, 32-bit reduction) from the direction's table
__device__ __forceinline__ double2 ls_phase_tab(int m, int n, double sign, const double2 *__restrict__ ph) {
  int r = m % n;
  if (r < 0) r += n;
  const double2 e = ph[r];
  return make_double2(e.x, sign * e.y);
}

// A[((c * (KM+1) + kx) * nz + (K-1)) * ny + (J-1)] = sum_i u_c(i, J, K) e^{-2 pi i kx i / nx}
__global__ void __launch_bounds__(256) k_ls_xsums(Geo g, CFields3 u, int KM, const double2 *__restrict__ xph,
                                                  double2 *__restrict__ A) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long line = (long long)blockIdx.x * LS_LINES + warp;
  if (line >= (long long)g.ny * g.nz) return;
  const int J = (int)(line % g.ny) + 1, K = (int)(line / g.ny) + 1;
  double2 acc[3][LS_KX];
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int kx = 0; kx < LS_KX; kx++) acc[c][kx] = make_double2(0.0, 0.0);
  const int row = gidx(g, 1, J, K);
  for (int i = lane; i < g.nx; i += 32) {
    const double2 e = xph[i];
    const double2 z1 = make_double2(e.x, -e.y);
    const double v[3] = {u.x[row + i], u.y[row + i], u.z[row + i]};
    double2 zk = make_double2(1.0, 0.0);
#pragma unroll
    for (int kx = 0; kx < LS_KX; kx++) {
      if (kx <= KM) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
          acc[c][kx].x = fma(v[c], zk.x, acc[c][kx].x);
          acc[c][kx].y = fma(v[c], zk.y, acc[c][kx].y);
        }
      }
      zk = cmul(zk, z1);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int kx = 0; kx < LS_KX; kx++) {
      double2 a = acc[c][kx];
      for (int o = 16; o > 0; o >>= 1) {
        a.x += __shfl_xor_sync(0xffffffffu, a.x, o);
        a.y += __shfl_xor_sync(0xffffffffu, a.y, o);
      }
      if (lane == 0 && kx <= KM) A[((long long)(c * (KM + 1) + kx) * g.nz + (K - 1)) * g.ny + (J - 1)] = a;
    }
}

// y-sums, one block of 128 per (c, kx, z-row): B[((c H + kx) nz + k) W + ky + KM]
// = sum_j A[...][j] e^{-2 pi i ky j / ny}, each thread over a stride of j,
// then a fixed-order tree reduction
__global__ void __launch_bounds__(128) k_ls_ysums(Geo g, const double2 *__restrict__ A, int KM,
                                                  const double2 *__restrict__ yph, double2 *__restrict__ B) {
  const int W = 2 * KM + 1;
  const long long r = blockIdx.x;  // (c H + kx) nz + k
  const double2 *a = A + r * g.ny;
  double2 acc[LS_KY];
#pragma unroll
  for (int q = 0; q < LS_KY; q++) acc[q] = make_double2(0.0, 0.0);
  for (int j = threadIdx.x; j < g.ny; j += blockDim.x) {
    const double2 v = a[j];
    const double2 e = yph[j];
    const double2 z1 = make_double2(e.x, -e.y);  // e^{-2 pi i j / ny}
    double2 zp = v, zm = v;                      // v e^{-+2 pi i ky j / ny}, ky = 0, 1, ..
    acc[KM] = cadd(acc[KM], v);
#pragma unroll
    for (int ky = 1; ky < LS_KX; ky++) {
      if (ky <= KM) {
        zp = cmul(zp, z1);
        zm = cmul(zm, cconj(z1));
        acc[KM + ky] = cadd(acc[KM + ky], zp);
        acc[KM - ky] = cadd(acc[KM - ky], zm);
      }
    }
  }
  __shared__ double2 red[LS_KY][128];
#pragma unroll
  for (int q = 0; q < LS_KY; q++) red[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int o = 64; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
#pragma unroll
      for (int q = 0; q < LS_KY; q++) red[q][threadIdx.x] = cadd(red[q][threadIdx.x], red[q][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if ((int)threadIdx.x < W) B[r * W + threadIdx.x] = red[threadIdx.x][0];
}

// z-sums, one block of 128 per (c, kx, ky): Gm[((c H + kx) W + ky + KM) W + kz + KM]
// = sum_k B[...][k] e^{-2 pi i kz k / nz} (the modes u_hat), fixed-order tree
__global__ void __launch_bounds__(128) k_ls_zsums(Geo g, const double2 *__restrict__ B, int KM,
                                                  const double2 *__restrict__ zph, double2 *__restrict__ Gm) {
  const int W = 2 * KM + 1;
  const int r = blockIdx.x;  // (c H + kx) W + ky + KM
  const int ckx = r / W, kyi = r % W;
  double2 acc[LS_KY];
#pragma unroll
  for (int q = 0; q < LS_KY; q++) acc[q] = make_double2(0.0, 0.0);
  for (int k = threadIdx.x; k < g.nz; k += blockDim.x) {
    const double2 v = B[((long long)ckx * g.nz + k) * W + kyi];
    const double2 e = zph[k];
    const double2 z1 = make_double2(e.x, -e.y);  // e^{-2 pi i k / nz}
    double2 zp = v, zm = v;
    acc[KM] = cadd(acc[KM], v);
#pragma unroll
    for (int kz = 1; kz < LS_KX; kz++) {
      if (kz <= KM) {
        zp = cmul(zp, z1);
        zm = cmul(zm, cconj(z1));
        acc[KM + kz] = cadd(acc[KM + kz], zp);
        acc[KM - kz] = cadd(acc[KM - kz], zm);
      }
    }
  }
  __shared__ double2 red[LS_KY][128];
#pragma unroll
  for (int q = 0; q < LS_KY; q++) red[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int o = 64; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
#pragma unroll
      for (int q = 0; q < LS_KY; q++) red[q][threadIdx.x] = cadd(red[q][threadIdx.x], red[q][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if ((int)threadIdx.x < W) Gm[(long long)r * W + threadIdx.x] = red[threadIdx.x][0];
}

// One block: the shell energies of the modes in Gm into E[0..nb), clamp
// factors into f, the corrections G = (f(shell) - 1) u_hat / N in place, and
// Hz[((c H + kx) W + ky + KM) nz + k] = sum_kz G e^{+2 pi i kz k / nz};
// eref[s] < 0 leaves shell s unforced.
__global__ void __launch_bounds__(1024) k_ls_modes(Geo g, int KM, double2 *__restrict__ Gm,
                                                   double2 *__restrict__ Hz, double *__restrict__ E,
                                                   const double *__restrict__ eref,
                                                   double *__restrict__ f, int nb,
                                                   const double2 *__restrict__ zph) {
  const int W = 2 * KM + 1, H = KM + 1;
  const double N = (double)g.nx * g.ny * g.nz;
  const int nM = 3 * H * W * W;
  // per-mode energies in shared memory (shell in the low bits), then the
  // shell sums by one thread in a fixed order, the factors, the corrections
  __shared__ double em[3 * LS_KX * LS_KY * LS_KY];
  __shared__ int sm[3 * LS_KX * LS_KY * LS_KY];
  for (int t = threadIdx.x; t < nM; t += blockDim.x) {
    const int kzi = t % W;
    const int r = t / W;
    const int kyi = r % W, kx = (r / W) % H;
    const int ky = kyi - KM, kz = kzi - KM;
    const int k2 = kx * kx + ky * ky + kz * kz;
    int sh = (int)sqrt((double)k2);
    while (sh * sh > k2) sh--;
    while ((sh + 1) * (sh + 1) <= k2) sh++;
    const double2 a = Gm[t];
    em[t] = (kx > 0 ? 2.0 : 1.0) * (a.x * a.x + a.y * a.y) / 2 / (N * N);
    sm[t] = sh;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double acc[LS_KX] = {0.0, 0.0, 0.0, 0.0};
    for (int t = 0; t < nM; t++) {
      const int sh = sm[t];
#pragma unroll
      for (int q = 0; q < LS_KX; q++) acc[q] += (sh == q) ? em[t] : 0.0;
    }
    for (int q = 0; q < nb; q++) {
      E[q] = acc[q];
      f[q] = (eref[q] >= 0 && acc[q] > 0) ? sqrt(eref[q] / acc[q]) : 1.0;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nM; t += blockDim.x) {
    const int kzi = t % W;
    const int r = t / W;
    const int kyi = r % W, kx = (r / W) % H;
    const int ky = kyi - KM, kz = kzi - KM;
    const int k2 = kx * kx + ky * ky + kz * kz;
    int sh = (int)sqrt((double)k2);
    while (sh * sh > k2) sh--;
    while ((sh + 1) * (sh + 1) <= k2) sh++;
    const double fac = sh < nb ? f[sh] - 1.0 : 0.0;
    Gm[t] = cscale(Gm[t], fac / N);
  }
  __syncthreads();
  const int nH = 3 * H * W * g.nz;
  for (int t = threadIdx.x; t < nH; t += blockDim.x) {
    const int k = t % g.nz, r = t / g.nz;  // r = (c H + kx) W + ky + KM
    double2 sacc = make_double2(0.0, 0.0);
    for (int kzi = 0; kzi < W; kzi++)
      sacc = cadd(sacc, cmul(Gm[r * W + kzi], ls_phase_tab((kzi - KM) * k, g.nz, 1.0, zph)));
    Hz[t] = sacc;
  }
}

// u_c(i, J, K) += Re sum_{kx, ky, kz} w(kx) G e^{+2 pi i (kx i/nx + ky j/ny + kz k/nz)},
// then the periodic ghost images of the updated cells
__global__ void __launch_bounds__(256) k_ls_correct(Geo g, Fields3 u, int KM,
                                                    const double2 *__restrict__ Hz,
                                                    const double2 *__restrict__ xph,
                                                    const double2 *__restrict__ yph) {
  const int W = 2 * KM + 1, H = KM + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long line = (long long)blockIdx.x * LS_LINES + warp;
  if (line >= (long long)g.ny * g.nz) return;
  const int j = (int)(line % g.ny), k = (int)(line / g.ny);
  const int J = j + 1, K = k + 1;
  // P[c][kx] = sum_{ky, kz} G e^{i (ky j / ny + kz k / nz)}: lane t < 3 H forms one
  double2 P = make_double2(0.0, 0.0);
  if (lane < 3 * H) {
    const int c = lane / H, kx = lane % H;
    for (int kyi = 0; kyi < W; kyi++)
      P = cadd(P, cmul(Hz[((long long)(c * H + kx) * W + kyi) * g.nz + k],
                       ls_phase_tab((kyi - KM) * j, g.ny, 1.0, yph)));
    if (kx > 0) P = cscale(P, 2.0);
  }
  double2 Pc[3][LS_KX];
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int kx = 0; kx < LS_KX; kx++) {
      const int src = c * H + kx;
      const double px = __shfl_sync(0xffffffffu, P.x, src < 32 ? src : 0);
      const double py = __shfl_sync(0xffffffffu, P.y, src < 32 ? src : 0);
      Pc[c][kx] = kx <= KM ? make_double2(px, py) : make_double2(0.0, 0.0);
    }
  double *fc[3] = {u.x, u.y, u.z};
  const int row = gidx(g, 1, J, K);
  for (int i = lane; i < g.nx; i += 32) {
    const double2 z1 = xph[i];
    double d[3] = {0.0, 0.0, 0.0};
    double2 zk = make_double2(1.0, 0.0);
#pragma unroll
    for (int kx = 0; kx < LS_KX; kx++) {
#pragma unroll
      for (int c = 0; c < 3; c++) d[c] += Pc[c][kx].x * zk.x - Pc[c][kx].y * zk.y;
      zk = cmul(zk, z1);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      store_img(fc[c], g, i + 1, J, K, fc[c][row + i] + d[c], STAG_P);
    }
  }
}

}  // namespace dnsb
