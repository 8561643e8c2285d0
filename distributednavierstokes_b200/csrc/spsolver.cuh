// spsolver.cuh -- pointwise kernels of the pseudo-spectral solver for a
// periodic cube (src/spectral/operators.jl, src/spectral/step.jl).
//
// The state is the reference's compact truncated spectrum: per component
// (kcut+1) x m x m complex values, m = 2 kcut + 1, kx fastest
// (q = i + (kcut+1) (j + m k); kx = i, ky / kz = compactfreq(j / k)),
// u_hat = F[u] / n^3.  The transforms run on the finite-volume context's
// FFT kernels over the full half spectrum S[kz + n (ky + n kx)] of the
// n^3 transform grid: scatter (zero padding) before the inverse, gather
// (truncation) after the forward transform.
#pragma once
#include "common.cuh"
#include "fft.cuh"

namespace dnsb {

// splitmix64 (src/spectral/ic.jl:31-36): one step of the published
// SplitMix64 generator from state x
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  unsigned long long z = x + 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

struct SpGeo {
  int n, kcut, m;
  long long nc;  // compact values per component
  double kfac;   // 2 pi / l
};

// compact index -> (integer kx, ky, kz) and the full-spectrum index
__device__ __forceinline__ void sp_modes(const SpGeo &s, long long q, int &kx, int &ky, int &kz) {
  const int h = s.kcut + 1;
  kx = (int)(q % h);
  const long long r = q / h;
  const int j = (int)(r % s.m), k = (int)(r / s.m);
  ky = j <= s.kcut ? j : j - s.m;  // compactfreq (src/spectral/operators.jl:7)
  kz = k <= s.kcut ? k : k - s.m;
}
__device__ __forceinline__ long long sp_full(const SpGeo &s, int kx, int ky, int kz) {
  const int j = ky >= 0 ? ky : ky + s.n, k = kz >= 0 ? kz : kz + s.n;
  return (long long)k + (long long)s.n * ((long long)j + (long long)s.n * kx);
}

#define SP_LOOP(q, n)                                                                   \
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (n); \
       q += (long long)gridDim.x * blockDim.x)

// S (already zeroed) <- the retained modes of one state component x scale
__global__ void k_sp_scatter(SpGeo s, const double2 *__restrict__ uh, double2 *__restrict__ S,
                             double scale) {
  SP_LOOP(q, s.nc) {
    int kx, ky, kz;
    sp_modes(s, q, kx, ky, kz);
    S[sp_full(s, kx, ky, kz)] = cscale(uh[q], scale);
  }
}

// the retained modes of S x sc into one state component (truncation)
__global__ void k_sp_gather(SpGeo s, const double2 *__restrict__ S, double2 *__restrict__ uh,
                            double sc) {
  SP_LOOP(q, s.nc) {
    int kx, ky, kz;
    sp_modes(s, q, kx, ky, kz);
    uh[q] = cscale(S[sp_full(s, kx, ky, kz)], sc);
  }
}

// The convective right-hand side -i k_j sigma_hat_ij from the transformed
// product a*b in S (times sc = 1/n^3), divdiag_kernel! / divoffdiag_kernel!
// (src/spectral/operators.jl:31-52): a == b sets du_a = -i k_a sigma;
// a != b subtracts i k_b sigma from du_a and i k_a sigma from du_b.
__global__ void k_sp_div(SpGeo s, const double2 *__restrict__ S, double2 *__restrict__ du, int a,
                         int b, double sc) {
  SP_LOOP(q, s.nc) {
    int kk[3];
    sp_modes(s, q, kk[0], kk[1], kk[2]);
    const double2 sg = cscale(S[sp_full(s, kk[0], kk[1], kk[2])], sc);
    const double ka = s.kfac * kk[a], kb = s.kfac * kk[b];
    double2 *da = du + a * s.nc, *db = du + b * s.nc;
    if (a == b) {
      da[q] = make_double2(ka * sg.y, -ka * sg.x);  // -i k sigma
    } else {
      const double2 x = da[q], y = db[q];
      da[q] = make_double2(x.x + kb * sg.y, x.y - kb * sg.x);  // - i k_b sigma
      db[q] = make_double2(y.x + ka * sg.y, y.y - ka * sg.x);  // - i k_a sigma
    }
  }
}

// r = va * vb on the n^3 transform grid
__global__ void k_sp_product(long long n3, const double *__restrict__ va,
                             const double *__restrict__ vb, double *__restrict__ r) {
  SP_LOOP(t, n3) r[t] = va[t] * vb[t];
}

// ifstage_kernel! (src/spectral/step.jl:22-43): one Wray stage with the
// integrating factor phi = exp(-nu dc dt k^2)
__global__ void k_sp_ifstage(SpGeo s, double2 *__restrict__ uh, double2 *__restrict__ ustart,
                             const double2 *__restrict__ du, double a, double b, double nudcdt,
                             double dt) {
  SP_LOOP(q, s.nc) {
    int kx, ky, kz;
    sp_modes(s, q, kx, ky, kz);
    const double k1 = s.kfac * kx, k2 = s.kfac * ky, k3 = s.kfac * kz;
    const double kk = k1 * k1 + k2 * k2 + k3 * k3;
    const double phi = exp(-nudcdt * kk);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const long long i = c * s.nc + q;
      const double2 st = ustart[i], d = du[i];
      uh[i] = make_double2(phi * (st.x + a * dt * d.x), phi * (st.y + a * dt * d.y));
      ustart[i] = make_double2(phi * (st.x + b * dt * d.x), phi * (st.y + b * dt * d.y));
    }
  }
}

// project_kernel! (src/spectral/operators.jl:10-23)
__global__ void k_sp_project(SpGeo s, double2 *__restrict__ uh) {
  SP_LOOP(q, s.nc) {
    int kx, ky, kz;
    sp_modes(s, q, kx, ky, kz);
    const double k1 = s.kfac * kx, k2 = s.kfac * ky, k3 = s.kfac * kz;
    const double kk = k1 * k1 + k2 * k2 + k3 * k3;
    const double2 ux = uh[q], uy = uh[s.nc + q], uz = uh[2 * s.nc + q];
    double2 p = make_double2((k1 * ux.x + k2 * uy.x + k3 * uz.x) / kk,
                             (k1 * ux.y + k2 * uy.y + k3 * uz.y) / kk);
    if (kk == 0) p = make_double2(0.0, 0.0);
    uh[q] = make_double2(ux.x - k1 * p.x, ux.y - k1 * p.y);
    uh[s.nc + q] = make_double2(uy.x - k2 * p.x, uy.y - k2 * p.y);
    uh[2 * s.nc + q] = make_double2(uz.x - k3 * p.x, uz.y - k3 * p.y);
  }
}

// Per-block partial sums over the compact state with the rfft
// double-counting weight (kx > 0 twice; kx <= kcut < n/2 has no Nyquist):
// mode 0 = |u_hat|^2 / 2 (spectral_energy), mode 1 = k^2 |u_hat|^2
// (spectral_dissipation without nu), src/spectral/operators.jl:60-102
__global__ void k_sp_sum(SpGeo s, const double2 *__restrict__ uh, int mode, double *partial) {
  double acc = 0.0;
  SP_LOOP(q, s.nc) {
    int kx, ky, kz;
    sp_modes(s, q, kx, ky, kz);
    double a2 = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 v = uh[c * s.nc + q];
      a2 += v.x * v.x + v.y * v.y;
    }
    const double k1 = s.kfac * kx, k2 = s.kfac * ky, k3 = s.kfac * kz;
    const double w = kx > 0 ? 2.0 : 1.0;
    acc += w * (mode == 0 ? a2 / 2 : a2 * (k1 * k1 + k2 * k2 + k3 * k3));
  }
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__device__ __forceinline__ unsigned long long sp_bits(double v) {
  return (unsigned long long)__double_as_longlong(v);
}

// max |k . u_hat| (spectral_maxdiv, src/spectral/operators.jl:104-110)
__global__ void k_sp_maxdiv(SpGeo s, const double2 *__restrict__ uh, unsigned long long *out) {
  double m = 0.0;
  SP_LOOP(q, s.nc) {
    int kx, ky, kz;
    sp_modes(s, q, kx, ky, kz);
    const double k1 = s.kfac * kx, k2 = s.kfac * ky, k3 = s.kfac * kz;
    const double2 ux = uh[q], uy = uh[s.nc + q], uz = uh[2 * s.nc + q];
    const double re = k1 * ux.x + k2 * uy.x + k3 * uz.x, im = k1 * ux.y + k2 * uy.y + k3 * uz.y;
    m = fmax(m, sqrt(re * re + im * im));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, sp_bits(m));
}

// vsummax (src/spectral/step.jl:45-58): max over the grid of |v1|+|v2|+|v3|
__global__ void k_sp_vsummax(long long n3, const double *__restrict__ v0,
                             const double *__restrict__ v1, const double *__restrict__ v2,
                             unsigned long long *out) {
  double m = 0.0;
  SP_LOOP(t, n3) m = fmax(m, fabs(v0[t]) + fabs(v1[t]) + fabs(v2[t]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, sp_bits(m));
}

// The LES cube |k_i| <= M/2 (M/2 <= kcut) of one state component in the
// coarse rfft layout cube[(kc M + jc)(M/2+1) + kx] (jc, kc wrapped: 0..M/2-1
// then -M/2..-1), straight from the compact state (lesboxes,
// src/spectral/les.jl:146-168: the cube of u_hat is a plain truncation)
__global__ void k_sp_cube(SpGeo s, const double2 *__restrict__ uh, int M, double2 *__restrict__ cube) {
  const int h = M / 2 + 1;
  const long long n = (long long)h * M * M;
  SP_LOOP(t, n) {
    const int kx = (int)(t % h);
    const long long r = t / h;
    const int jc = (int)(r % M), kc = (int)(r / M);
    const int ky = jc < M / 2 ? jc : jc - M, kz = kc < M / 2 ? kc : kc - M;
    const int j = ky >= 0 ? ky : ky + s.m, k = kz >= 0 ? kz : kz + s.m;  // compact index
    cube[t] = uh[kx + (long long)(s.kcut + 1) * (j + (long long)s.m * k)];
  }
}

// noise_kernel! (src/spectral/ic.jl:37-51) on the n^3 grid of component c
// (one rank: offsets 0): Box-Muller of two splitmix64 uniforms,
// key = ((c n + k) n + j) n + i
__global__ void k_sp_noise(int n, double *__restrict__ v, int c, unsigned long long seed) {
  const long long n3 = (long long)n * n * n;
  SP_LOOP(t, n3) {
    const unsigned long long key = (unsigned long long)c * (unsigned long long)n3 + (unsigned long long)t;
    const unsigned long long r1 = splitmix64(seed + 2 * key), r2 = splitmix64(seed + 2 * key + 1);
    const double u1 = ((double)(r1 >> 11) + 0.5) * 0x1p-53;
    const double u2 = ((double)(r2 >> 11) + 0.5) * 0x1p-53;
    v[t] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
}

// integer shell floor(sqrt(kx^2 + ky^2 + kz^2)) of a compact mode
// (src/spectral/forcing.jl:17) and its rfft weight
__device__ __forceinline__ int sp_shell(const SpGeo &s, long long q, double &w) {
  int kx, ky, kz;
  sp_modes(s, q, kx, ky, kz);
  const long long k2 = (long long)kx * kx + (long long)ky * ky + (long long)kz * kz;
  long long r = (long long)sqrt((double)k2);
  while (r * r > k2) r--;
  while ((r + 1) * (r + 1) <= k2) r++;
  w = kx > 0 ? 2.0 : 1.0;
  return (int)r;
}

// shell_energies (src/spectral/forcing.jl:12-24), fixed summation order:
// per-block partial sums of the lowest SP_SHELLS shells ...
constexpr int SP_SHELLS = 8;
__global__ void __launch_bounds__(256) k_sp_shells_det(SpGeo s, const double2 *__restrict__ uh,
                                                       double *partial) {
  double acc[SP_SHELLS];
#pragma unroll
  for (int i = 0; i < SP_SHELLS; i++) acc[i] = 0.0;
  SP_LOOP(q, s.nc) {
    double w;
    const int sh = sp_shell(s, q, w);
    if (sh >= SP_SHELLS) continue;
    double a2 = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 v = uh[c * s.nc + q];
      a2 += v.x * v.x + v.y * v.y;
    }
    const double e = w * a2 / 2;
#pragma unroll
    for (int i = 0; i < SP_SHELLS; i++) acc[i] += sh == i ? e : 0.0;
  }
  __shared__ double red[SP_SHELLS][256];
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < SP_SHELLS; i++) red[i][tid] = acc[i];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (tid < o) {
#pragma unroll
      for (int i = 0; i < SP_SHELLS; i++) red[i][tid] += red[i][tid + o];
    }
    __syncthreads();
  }
  if (tid < SP_SHELLS) partial[blockIdx.x * SP_SHELLS + tid] = red[tid][0];
}
__global__ void k_sp_shells_fold(const double *partial, int nblocks, int nb, double *E) {
  const int sh = threadIdx.x;
  if (sh >= nb) return;
  double a = 0.0;
  for (int b = 0; b < nblocks; b++) a += partial[b * SP_SHELLS + sh];
  E[sh] = a;
}
// ... or one block per shell for any number of shells (set-up time)
__global__ void __launch_bounds__(256) k_sp_shells_byshell(SpGeo s, const double2 *__restrict__ uh,
                                                           double *E) {
  const int target = blockIdx.x;
  double acc = 0.0;
  for (long long q = threadIdx.x; q < s.nc; q += blockDim.x) {
    double w;
    if (sp_shell(s, q, w) != target) continue;
    double a2 = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 v = uh[c * s.nc + q];
      a2 += v.x * v.x + v.y * v.y;
    }
    acc += w * a2 / 2;
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) E[target] = red[0];
}

// rescale_shell! (src/spectral/forcing.jl:26-35) for all shells < nb at once
__global__ void k_sp_scale_shells(SpGeo s, double2 *__restrict__ uh, const double *__restrict__ f,
                                  int nb) {
  SP_LOOP(q, s.nc) {
    double w;
    const int sh = sp_shell(s, q, w);
    if (sh >= nb) continue;
    const double fs = f[sh];
#pragma unroll
    for (int c = 0; c < 3; c++) uh[c * s.nc + q] = cscale(uh[c * s.nc + q], fs);
  }
}

// shellforcing's closure: f = sqrt(eref / E) for forced shells with E > 0
__global__ void k_sp_clamp_factors(const double *E, const double *eref, double *f, int nb) {
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    f[i] = (eref[i] >= 0 && E[i] > 0) ? sqrt(eref[i] / E[i]) : 1.0;
}

// phaserand_kernel! (src/spectral/ic.jl:108-128): every retained mode but
// the mean times a unit-modulus phase from splitmix64 of the mode's key;
// in the kx = 0 plane (0, k2, k3) and (0, -k2, -k3) share the canonical
// member's phase and the other member takes its conjugate
__global__ void k_sp_phaserand(SpGeo s, double2 *__restrict__ uh, unsigned long long seed) {
  SP_LOOP(q, s.nc) {
    int k1, k2, k3;
    sp_modes(s, q, k1, k2, k3);
    if (k1 == 0 && k2 == 0 && k3 == 0) continue;
    const bool canon = k1 > 0 || k2 > 0 || (k2 == 0 && k3 > 0);
    const long long c2 = canon ? k2 : -k2, c3 = canon ? k3 : -k3;
    const unsigned long long w = 2ULL * s.kcut + 2ULL;
    const unsigned long long key =
        ((unsigned long long)k1 * w + (unsigned long long)(c2 + s.kcut)) * w +
        (unsigned long long)(c3 + s.kcut);
    const double u = ((double)(splitmix64(seed + key) >> 11) + 0.5) * 0x1p-53;
    double sn, cs;
    sincospi(2.0 * u, &sn, &cs);
    const double2 ph = make_double2(cs, canon ? sn : -sn);
#pragma unroll
    for (int c = 0; c < 3; c++) uh[c * s.nc + q] = cmul(uh[c * s.nc + q], ph);
  }
}

#undef SP_LOOP

}  // namespace dnsb
