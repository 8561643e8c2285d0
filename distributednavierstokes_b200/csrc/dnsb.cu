// dnsb.cu -- context, plans and the C ABI of libdnsb.so (see include/dnsb.h).
//
// One RK3 stage (step!, src/timestep.jl:41-63) is, on the default path,
//   explicit: k_momentum<EXPLICIT>  q, W = u + B q            (+ W halos)
//             k_rfftx<DIVERGENCE>   S = rfft_x(div W)
//             k_fftz                S = fft_z(S)
//             k_thomas | k_yfourier solve in y
//             k_fftz<inv>, k_irfftx psi (+ halos)
//             k_grad<EXPLICIT>      u = W - grad psi          (+ u halos)
//   implicit: k_momentum<IMPLICIT>  q, V = u + B q - a dt grad p + th Dy u
//             k_cn                  u = (I - th Dy)^-1 V      (+ halos)
//             Poisson as above      delta (+ halos)
//             k_grad<IMPLICIT>      u -= grad delta, p += delta/(a dt) (+ halos)
// so that no separate halo, copy or transpose kernel runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dnsb.h"
#include "../../include/dnsb_cnn.h"
#include "cnn_host.h"
#include "common.cuh"
#include "fft.cuh"
#include "spectral.cuh"
#include "spectral4.cuh"
#include "ysolve.cuh"
#include "stencil.cuh"
#include "gradmom.cuh"
#include "zyz.cuh"
#include "spsolver.cuh"
#include "lowshells.cuh"

using namespace dnsb;

namespace {

const double RK_A[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
const double RK_B[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
const double RK_AL[3] = {1.0 / 3.0, 5.0 / 12.0, 1.0 / 4.0};

char g_create_err[512] = "";

// exp(-2 pi i t / n) evaluated in long double and rounded once, with exact
// values at the quarter turns.
double2 unit_root(long t, long n) {
  t %= n;
  if (t < 0) t += n;
  const long double pi = 3.141592653589793238462643383279502884L;
  long double x = (long double)t / (long double)n;
  long double c = cosl(2.0L * pi * x), s = sinl(2.0L * pi * x);
  if (t == 0) { c = 1; s = 0; }
  else if (4 * t == n) { c = 0; s = 1; }
  else if (2 * t == n) { c = -1; s = 0; }
  else if (4 * t == 3 * n) { c = 0; s = -1; }
  return make_double2((double)c, -(double)s);
}

// modλ (src/poisson.jl:12): 2 (cospi(2(k-1)/n) - 1) / Δ^2, k = 1-based
double modlam(int k1, int n, double d) {
  const long double pi = 3.141592653589793238462643383279502884L;
  double x = (double)(2 * (k1 - 1)) / (double)n;
  double c = (double)cosl((long double)x * pi);
  if (k1 - 1 == 0) c = 1.0;
  else if (4 * (k1 - 1) == n || 4 * (k1 - 1) == 3 * n) c = 0.0;
  else if (2 * (k1 - 1) == n) c = -1.0;
  return 2 * (c - 1) / (d * d);
}

}  // namespace

struct dnsb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  Geo g{};
  int implicit = 0;
  double dymin = 0;
  // device tables
  double *dy = nullptr, *dyu = nullptr, *rdy = nullptr, *rdyu = nullptr;
  double *lam1 = nullptr, *lam2 = nullptr, *lam3 = nullptr;
  double *ay = nullptr, *by = nullptr, *cy = nullptr;
  double *ycoef = nullptr;  // [at bt ct an bn cn] x ny
  double2 *ymet = nullptr;  // YMET packed per-row metrics of the momentum stencil
  double *ytab = nullptr;   // [3 stages][2 sets][ta cp ib] x ny
  double2 *twM = nullptr, *twN = nullptr, *twz = nullptr, *twy = nullptr;
  FFTPlan pM{}, pz{}, py{};
  int Lx = 1, Lz = 1, Ly = 1;
  size_t smem_rx = 0, smem_ix = 0, smem_z = 0, smem_y = 0, smem_cn = 0;
  int cn_mr = 1;      // rows per chunk of the CN solve
  int mom_tile = 1;   // z-marching momentum kernel with staged planes
  int fuse = 1;       // fused projection + momentum between implicit stages
  double *pn = nullptr;  // pressure after stage 1 when fused
  dim3 tgrid, tblock;
  // z-planes per CTA of the fused projection + momentum: 32 measured 1.5 %
  // faster than 16 and 64 at 384x256x384 (its prologue projects two planes)
  int gm_planes = 32;
  std::map<const void *, CUtensorMap> gm_maps;  // TMA maps of the fused kernel's staged fields
  int mom_planes = MC_Z;  // z planes per CTA of k_momentum_march
  // while a CUDA graph of LES steps is captured: the device word holding
  // the step size, read by the kernels that take dt (else nullptr)
  const double *dtp = nullptr;
  cudaStream_t les_cap = nullptr;  // capture stream of dnsb_les_advance's graph
  double *les_state = nullptr;     // its device state: t, dt, steps, t1, the loop threshold
  // dnsb_les_advance's instantiated graphs, one per argument set (the eight
  // fields, the closure and its creation serial, the CFL number, the shell
  // count, graph_gen), reused by later calls with other intervals; least
  // recently used out beyond LES_GRAPHS
  struct LesGraph {
    const void *ptr[9];
    unsigned long long serial;
    double cfl;
    int nb;
    unsigned gen;
    unsigned long long used;
    cudaGraphExec_t exec;
  };
  std::vector<LesGraph> les_graphs;
  unsigned long long les_uses = 0;
  unsigned graph_gen = 0;  // bumped by every setter whose value a captured kernel takes as an argument
  // one-barrier pipelined variant of the fused kernel: 2.5 % faster than
  // the two-barrier k_gradmom_march at 384x256x384
  int gm_pipe = 1;
  dim3 gmgrid;

  dim3 cgrid, cblock;  // launch shape of the per-cell step kernels
  // scratch
  double2 *S = nullptr;
  double2 *Sx[2] = {nullptr, nullptr};  // spectra of u.y, u.z during a shell clamp
  double2 *lsA = nullptr, *lsB = nullptr, *lsG = nullptr, *lsH = nullptr;  // low-shell clamp scratch
  // e^{2 pi i r / n}, r = 0..n-1, per direction, for the clamp's partial sums
  double2 *lsX = nullptr, *lsY = nullptr, *lsZ = nullptr;
  double *work = nullptr;
  double *ycin = nullptr;  // c' entering each y-chunk, per (kx, kz) line
  double *r = nullptr;
  double *W[3] = {nullptr, nullptr, nullptr};
  double *V[3] = {nullptr, nullptr, nullptr};
  unsigned long long *umax = nullptr;  // [3] max |u_c| of the last step; [3] scratch
  double *partial = nullptr;           // reduction partials
  double *shellbuf = nullptr;          // periodic boxes: [E | factors | eref] x nshell_max
  int nshell_max = 0;                  // floor(|k|max) + 1
  double *shellpart = nullptr;         // per-block partial shell sums (fixed-order path)
  std::vector<double> eref_host;       // shell-clamp reference energies on the device
  double *hostsolve = nullptr;         // device fields of dnsb_solve_host (first call on)
  double2 *cube = nullptr;             // LES cubes of the filtered-field sampler
  size_t cube_cap = 0;
  int *deverr = nullptr;               // device-side error word (bounded waits)
  unsigned wait_limit = DNSB_WAIT_LIMIT;  // polls per device-side wait
  int use_tma = 1;                     // persistent TMA-pipelined z-FFT
  int zyz_c = 0;                       // CTAs per cluster of k_zyz (0: three kernels)
  int zyz_mode = 1;                    // 1: k_zyz (32-row chunks), 2: k_zyz2 (16-row chunks)
  int nkx_active = 0;                  // z-FFTs on kx < nkx_active only (0: all; spectral solver)
  int x1 = 0, x2 = 0, z1 = 0, z2 = 0;  // four-step splits of nx/2 and nz (0: generic kernels)
  int L4z = 8;                         // lines per CTA of the z-FFT
  // divergence x-FFT with its output pass in registers (3 % faster at
  // 384x256x384 than the separate shared-memory pass)
  int rx_post = 1;
  int ix_pairs = 0;  // inverse x-FFT with the pair pre-processing in its first pass
  size_t smem_rx4 = 0, smem_ix4 = 0, smem_z4 = 0;
  int nsm = 148;
  size_t smem_zt = 0;
  double *hostred = nullptr;           // pinned, 8 doubles
  unsigned long long *hostumax = nullptr;  // pinned, 3 * UMAX_SLOTS
  const double *umax_for[3] = {nullptr, nullptr, nullptr};
  // launch counting and per-kind CUDA-event timing (dnsb_profile)
  long launches = 0;
  bool prof_on = false;
  std::vector<cudaEvent_t> evpool;
  size_t evused = 0;
  std::vector<std::pair<int, size_t>> recs;  // (kind, index of the start event)
  double prof_ms[DNSB_NKINDS] = {};
  long prof_n[DNSB_NKINDS] = {};
  std::vector<void *> allocs;
  std::string err;
};

namespace {

constexpr int RED_BLOCKS = 1184;

// integer knob from the environment (launch-shape tuning), default if unset
int envint(const char *name, int dflt) {
  const char *e = getenv(name);
  return (e && *e) ? atoi(e) : dflt;
}

int fail(dnsb_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  else snprintf(g_create_err, sizeof g_create_err, "%s", buf);
  return code;
}

#define CK(ctx, call)                                                                        \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(ctx, DNSB_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                  __LINE__);                                                                 \
  } while (0)

#define CKL(ctx) CK(ctx, cudaGetLastError())

const char *KIND_NAMES[DNSB_NKINDS] = {"momentum", "cn_solve", "div_rfft_x", "fft_z", "y_solve",
                                       "ifft_z", "irfft_x", "grad_update", "other",
                                       "grad_momentum", "fft_z_y_solve"};

int prof_harvest(dnsb_ctx *c) {
  if (c->recs.empty()) { c->evused = 0; return 0; }
  CK(c, cudaEventSynchronize(c->evpool[c->recs.back().second + 1]));
  for (auto &r : c->recs) {
    float ms = 0;
    CK(c, cudaEventElapsedTime(&ms, c->evpool[r.second], c->evpool[r.second + 1]));
    c->prof_ms[r.first] += ms;
    c->prof_n[r.first] += 1;
  }
  c->recs.clear();
  c->evused = 0;
  return 0;
}

int prof_begin(dnsb_ctx *c, int kind) {
  (void)kind;
  c->launches++;
  if (!c->prof_on) return 0;
  if (c->evused + 2 > c->evpool.size()) {
    int rc = prof_harvest(c);
    if (rc) return rc;
  }
  CK(c, cudaEventRecord(c->evpool[c->evused], c->stream));
  return 0;
}

int prof_end(dnsb_ctx *c, int kind) {
  if (!c->prof_on) return 0;
  CK(c, cudaEventRecord(c->evpool[c->evused + 1], c->stream));
  c->recs.push_back({kind, c->evused});
  c->evused += 2;
  return 0;
}

// Launch with counting and (when enabled) event timing of its kind.
#define LAUNCH(ctx, kind, ...)                       \
  do {                                               \
    int rc_ = prof_begin(ctx, kind);                 \
    if (rc_) return rc_;                             \
    __VA_ARGS__;                                     \
    CKL(ctx);                                        \
    rc_ = prof_end(ctx, kind);                       \
    if (rc_) return rc_;                             \
  } while (0)

template <class T>
int dalloc(dnsb_ctx *c, T **p, size_t n) {
  void *v = nullptr;
  cudaError_t e = cudaMalloc(&v, n * sizeof(T) > 0 ? n * sizeof(T) : 16);
  if (e != cudaSuccess)
    return fail(c, DNSB_ENOMEM, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
  c->allocs.push_back(v);
  *p = (T *)v;
  return 0;
}

template <class T>
int upload(dnsb_ctx *c, T **p, const std::vector<T> &h) {
  int rc = dalloc(c, p, h.size());
  if (rc) return rc;
  CK(c, cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

dim3 cell_grid(const Geo &g) { return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz); }
dim3 cn_grid(const Geo &g) { return dim3((g.nx + CN_LINES - 1) / CN_LINES, g.nz, 3); }
const dim3 cell_block(32, 8, 1);

CFields3 cf(const double *x, const double *y, const double *z) { return CFields3{x, y, z}; }
Fields3 ff(double *x, double *y, double *z) { return Fields3{x, y, z}; }

// opt in to the dynamic shared memory a kernel launches with (needed whenever
// static + dynamic shared memory exceeds 48 KB; requested unconditionally).
// The attribute belongs to the kernel function (per device), not to the
// context, so contexts of different sizes in one process may only ever raise
// it: the largest request per (device, kernel) is kept.
template <class K>
cudaError_t raise_smem(int device, K kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> granted;
  std::lock_guard<std::mutex> lock(mu);
  size_t &cur = granted[{device, reinterpret_cast<const void *>(kernel)}];
  if (bytes <= cur && cur != 0) return cudaSuccess;
  const size_t want = std::max(bytes, cur);
  const cudaError_t e =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want);
  if (e == cudaSuccess) cur = want;
  return e;
}

template <class K>
int allow_smem(dnsb_ctx *c, K kernel, size_t bytes) {
  CK(c, raise_smem(c->device, kernel, bytes));
  return 0;
}

// ----------------------------------------------------------- reductions --

// out[0..2]: max |u_c| over the interior (as ordered bits); with deverr,
// out[3] also receives the device error word (read after every earlier
// kernel of the stream has finished), so that one copy brings both back.
// max |u_c| over the interior cells (dbits order = value order for x >= 0).
// Warps walk the (J, K) rows and their lanes stride along x: one 32-bit
// division per row instead of 64-bit divisions per cell, coalesced loads;
// the block's maxima meet in shared memory and leave in one atomic per
// component (a maximum does not depend on the order).  Grid: maxabs_blocks.
__global__ void __launch_bounds__(256) k_maxabs3(Geo g, CFields3 u, unsigned long long *out,
                                                 const int *deverr) {
  if (deverr && blockIdx.x == 0 && threadIdx.x == 0) out[3] = (unsigned long long)(unsigned)*deverr;
  __shared__ double wm[3][8];
  double m0 = 0, m1 = 0, m2 = 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int rows = g.ny * g.nz;
  for (int r = blockIdx.x * nw + w; r < rows; r += gridDim.x * nw) {
    const int K = r / g.ny, J = r - K * g.ny;
    const int row = gidx(g, 0, J + 1, K + 1);
    for (int I = lane + 1; I <= g.nx; I += 32) {
      m0 = fmax(m0, fabs(u.x[row + I]));
      m1 = fmax(m1, fabs(u.y[row + I]));
      m2 = fmax(m2, fabs(u.z[row + I]));
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
    m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
  }
  if (lane == 0) wm[0][w] = m0, wm[1][w] = m1, wm[2][w] = m2;
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0;
    for (int k = 0; k < nw; k++) v = fmax(v, wm[threadIdx.x][k]);
    atomicMax(out + threadIdx.x, dbits(v));
  }
}

// blocks of k_maxabs3: four rows per warp, at most RED_BLOCKS
inline unsigned maxabs_blocks(const Geo &g) {
  const long long rows = (long long)g.ny * g.nz;
  return (unsigned)std::max(1LL, std::min<long long>(RED_BLOCKS, (rows + 31) / 32));
}

__global__ void k_maxdiv(Geo g, CFields3 u, unsigned long long *out) {
  double m = 0;
  const long long n = (long long)g.nx * g.ny * g.nz;
  const long long sy = g.NX, sz = (long long)g.NX * g.NY;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int I = (int)(t % g.nx) + 1;
    const long long r = t / g.nx;
    const int J = (int)(r % g.ny) + 1, K = (int)(r / g.ny) + 1;
    const long long c0 = gidx(g, I, J, K);
    const double d = (u.x[c0] - u.x[c0 - 1]) * g.rdx + (u.y[c0] - u.y[c0 - sy]) * g.rdy[J] +
                     (u.z[c0] - u.z[c0 - sz]) * g.rdz;
    m = fmax(m, fabs(d));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, dbits(m));
}

__device__ double block_sum(double v) {
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  v = 0;
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = l < nw ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;  // valid in thread 0
}

// kinetic energy partials: sum of u_c^2 dx D2[J] dz / 2 over ranges[c]
__global__ void k_ke_partial(Geo g, CFields3 u, double *partial) {
  double s = 0;
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int I = (int)(t % g.nx) + 1;
    const long long r = t / g.nx;
    const int J = (int)(r % g.ny) + 1, K = (int)(r / g.ny) + 1;
    const long long c0 = gidx(g, I, J, K);
    const double vx = u.x[c0], vz = u.z[c0];
    s += vx * vx * g.dx * g.dy[J] * g.dz / 2;
    s += vz * vz * g.dx * g.dy[J] * g.dz / 2;
    if (J <= g.jymax) {
      const double vy = u.y[c0];
      s += vy * vy * g.dx * g.dyu[J] * g.dz / 2;
    }
  }
  s = block_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void k_sum_final(const double *partial, int n, double *out) {
  double s = 0;
  for (int t = threadIdx.x; t < n; t += blockDim.x) s += partial[t];
  s = block_sum(s);
  if (threadIdx.x == 0) *out = s;
}

// channel plane sums (sample_channelstats!, src/stats.jl:39-58): one block
// per y row; rows 0..ny-1 cell quantities, rows ny..ny+nf-1 face quantities
__global__ void k_channel(Geo g, CFields3 u, double *acc, int nf) {
  const int row = blockIdx.x;
  const bool face = row >= g.ny;
  const int J = (face ? row - g.ny : row) + 1;
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  const long long n = (long long)g.nx * g.nz;
  const long long sy = g.NX;
  for (long long t = threadIdx.x; t < n; t += blockDim.x) {
    const int I = (int)(t % g.nx) + 1, K = (int)(t / g.nx) + 1;
    const long long c0 = gidx(g, I, J, K);
    if (!face) {
      const double x = u.x[c0], z = u.z[c0];
      s0 += x; s1 += z; s2 += x * x; s3 += z * z;
    } else {
      const double v = u.y[c0];
      const double uf = (u.x[c0] + u.x[c0 + sy]) / 2;
      const double vf = (u.y[c0] + u.y[c0 + 1]) / 2;
      s0 += v; s1 += v * v; s2 += uf; s3 += uf * vf;
    }
  }
  s0 = block_sum(s0);
  s1 = block_sum(s1);
  s2 = block_sum(s2);
  s3 = block_sum(s3);
  if (threadIdx.x == 0) {
    if (!face) {
      const int j = J - 1;
      acc[j] += s0; acc[g.ny + j] += s1; acc[2 * g.ny + j] += s2; acc[3 * g.ny + j] += s3;
    } else {
      double *f = acc + 4 * g.ny;
      const int j = J - 1;
      f[j] += s0; f[nf + j] += s1; f[2 * nf + j] += s2; f[3 * nf + j] += s3;
    }
  }
}

// Integer shell of the spectrum entry t (S layout): round(|k|) for the
// statistics of stats.jl:152, floor(|k|) for the shell operations of
// src/spectral/forcing.jl:12-35; w = rfft double-counting weight.
template <bool FLOORED>
__device__ __forceinline__ int shell_of(const Geo &g, long long t, double &w) {
  const int kz0 = (int)(t % g.nz);
  const long long r = t / g.nz;
  const int j = (int)(r % g.ny), kx = (int)(r / g.ny);
  const int ky = j > g.ny / 2 ? j - g.ny : j;
  const int kz = kz0 > g.nz / 2 ? kz0 - g.nz : kz0;
  const long long k2 = (long long)kx * kx + (long long)ky * ky + (long long)kz * kz;
  w = (0 < kx && 2 * kx < g.nx) ? 2.0 : 1.0;
  if (FLOORED) {
    long long s = (long long)sqrt((double)k2);  // integer square root, corrected
    while (s * s > k2) s--;
    while ((s + 1) * (s + 1) <= k2) s++;
    return (int)s;
  }
  return (int)llrint(sqrt((double)k2));
}

// binshells! (src/stats.jl:143-157): 1/2 |u_hat|^2 / N^2 into integer
// shells round(|k|) (FLOORED: floor(|k|), shell_energies of
// src/spectral/forcing.jl:12-24), conjugate modes 0 < kx < nx/2 counted twice
template <bool FLOORED>
__global__ void k_binshells(Geo g, const double2 *S, double *E, int nbins) {
  const long long n = (long long)g.nkx * g.ny * g.nz;
  const double N = (double)g.nx * g.ny * g.nz;
  const double N2 = N * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    double wgt;
    const int kap = shell_of<FLOORED>(g, t, wgt);
    const double2 a = S[t];
    const double a2 = a.x * a.x + a.y * a.y;
    if (kap < nbins) atomicAdd(E + kap, wgt * a2 / 2 / N2);
  }
}

// Shell energies of the lowest SHELL_DET shells in a fixed summation order
// (bit-reproducible from run to run, which the atomics of k_binshells are
// not): every thread sums its grid-stride entries in order, the block
// reduces them in a fixed tree, k_sum_shells adds the blocks in order.
constexpr int SHELL_DET = 8;
__global__ void __launch_bounds__(256) k_binshells_det(Geo g, const double2 *S, double *partial) {
  const long long n = (long long)g.nkx * g.ny * g.nz;
  const double N = (double)g.nx * g.ny * g.nz;
  const double N2 = N * N;
  double acc[SHELL_DET];
#pragma unroll
  for (int s = 0; s < SHELL_DET; s++) acc[s] = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    double wgt;
    const int kap = shell_of<true>(g, t, wgt);
    if (kap >= SHELL_DET) continue;
    const double2 a = S[t];
    const double v = wgt * (a.x * a.x + a.y * a.y) / 2 / N2;
#pragma unroll
    for (int s = 0; s < SHELL_DET; s++) acc[s] += kap == s ? v : 0.0;
  }
  __shared__ double red[SHELL_DET][256];
  const int tid = threadIdx.x;
#pragma unroll
  for (int s = 0; s < SHELL_DET; s++) red[s][tid] = acc[s];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (tid < o) {
#pragma unroll
      for (int s = 0; s < SHELL_DET; s++) red[s][tid] += red[s][tid + o];
    }
    __syncthreads();
  }
  if (tid < SHELL_DET) partial[blockIdx.x * SHELL_DET + tid] = red[tid][0];
}

// The same for any number of shells (set-up time: the random initial
// field): block s sums shell s over the whole spectrum in a fixed order.
__global__ void __launch_bounds__(256) k_binshells_byshell(Geo g, const double2 *S, double *E) {
  const long long n = (long long)g.nkx * g.ny * g.nz;
  const double N = (double)g.nx * g.ny * g.nz;
  const double N2 = N * N;
  const int sh = blockIdx.x;
  double acc = 0.0;
  for (long long t = threadIdx.x; t < n; t += blockDim.x) {
    double wgt;
    if (shell_of<true>(g, t, wgt) != sh) continue;
    const double2 a = S[t];
    acc += wgt * (a.x * a.x + a.y * a.y) / 2 / N2;
  }
  __shared__ double red[256];
  const int tid = threadIdx.x;
  red[tid] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (tid < o) red[tid] += red[tid + o];
    __syncthreads();
  }
  if (tid == 0) E[sh] += red[0];
}

// E[s] += the block partials of shell s, in block order
__global__ void k_sum_shells(const double *partial, int nblocks, int nb, double *E) {
  const int s = threadIdx.x;
  if (s >= nb) return;
  double a = 0.0;
  for (int b = 0; b < nblocks; b++) a += partial[b * SHELL_DET + s];
  E[s] += a;
}

// rescale_shell! (src/spectral/forcing.jl:26-35) for every shell at once:
// entry t of S times f[floor(|k|)] (shells >= nbins unchanged)
__global__ void k_scaleshells(Geo g, double2 *S, const double *__restrict__ f, int nbins) {
  const long long n = (long long)g.nkx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    double w;
    const int sh = shell_of<true>(g, t, w);
    if (sh < nbins) S[t] = cscale(S[t], f[sh]);
  }
}


__global__ void k_noise(Geo g, double *phi, int c, unsigned long long seed, double amp) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  const int jh = c == STAG_Y ? g.jymax : g.ny;
  if (I > g.nx || J > jh) return;
  const unsigned long long key =
      (((unsigned long long)c * g.nz + (K - 1)) * g.ny + (J - 1)) * g.nx + (I - 1);
  const unsigned long long rr = splitmix64(seed + key);
  const double U = ((double)(rr >> 11) + 0.5) * 0x1p-53;
  const long long c0 = gidx(g, I, J, K);
  // explicit roundings (no FMA contraction) so that the field is bit-identical
  // to a host evaluation of phi + amp*(2U - 1)
  phi[c0] = __dadd_rn(phi[c0], __dmul_rn(amp, __dsub_rn(2 * U, 1.0)));
}

// noise_kernel! (src/spectral/ic.jl:37-51) on the interior of component c:
// standard normal values from two counter-based uniforms (Box-Muller),
// key = ((c*nz + K-1)*ny + J-1)*nx + I-1 (the reference's key on its cube)
__global__ void k_gauss_noise(Geo g, double *phi, int c, unsigned long long seed) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  if (I > g.nx || J > g.ny) return;
  const unsigned long long key =
      (((unsigned long long)c * g.nz + (K - 1)) * g.ny + (J - 1)) * g.nx + (I - 1);
  const unsigned long long r1 = splitmix64(seed + 2 * key), r2 = splitmix64(seed + 2 * key + 1);
  const double u1 = ((double)(r1 >> 11) + 0.5) * 0x1p-53;
  const double u2 = ((double)(r2 >> 11) + 0.5) * 0x1p-53;
  phi[gidx(g, I, J, K)] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// Cell-centred velocity products for the filtered-field sampler: out = v_a
// (b < 0) or v_a v_b on the interior, v_c the average of the two faces of
// the cell along c (the cell-centre interpolation of operators.jl:71-72).
__global__ void k_cellprod(Geo g, CFields3 u, int a, int b, double *out) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  if (I > g.nx || J > g.ny) return;
  const int c0 = gidx(g, I, J, K);
  auto vc = [&](int c) {
    const double *f = c == 0 ? u.x : c == 1 ? u.y : u.z;
    const int o = c == 0 ? 1 : c == 1 ? g.NX : g.NX * g.NY;
    return (f[c0 - o] + f[c0]) / 2;
  };
  const double va = vc(a);
  out[c0] = b < 0 ? va : va * vc(b);
}

// The LES cube |k_i| <= M/2 of a transformed field (S, unnormalised) into
// the coarse rfft layout cube[(kc*M + jc)*(M/2+1) + kx] (kx = 0..M/2; jc, kc
// wrapped: 0..M/2-1 then -M/2..-1), times sc (1/N: u_hat = F[u]/N), after
// lesboxes / lescoarse (src/spectral/les.jl:146-168).
__global__ void k_lescube(Geo g, const double2 *__restrict__ S, int M, double sc,
                          double2 *__restrict__ cube) {
  const int h = M / 2 + 1;
  const long long n = (long long)h * M * M;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(t % h);
    const long long r = t / h;
    const int jc = (int)(r % M), kc = (int)(r / M);
    const int ky = jc < M / 2 ? jc : jc - M, kz = kc < M / 2 ? kc : kc - M;
    const int j = ky >= 0 ? ky : ky + g.ny, k = kz >= 0 ? kz : kz + g.nz;
    cube[t] = cscale(S[sidx(g, kx, j, k)], sc);
  }
}

// ------------------------------------------------------------- pipeline --

int ensure_device(dnsb_ctx *c) {
  CK(c, cudaSetDevice(c->device));
  return 0;
}

#define FFT4_SPLITS(X) X(16, 24) X(16, 16) X(16, 12) X(16, 8) X(8, 12) X(8, 8) X(8, 6) X(8, 4)
constexpr int IRX_L = 16;  // lines per CTA of the four-step inverse x-FFT
constexpr int RFX_L = 8;   // lines per CTA of the four-step forward x-FFT

// four-step kernel launches for the split chosen at create time
int launch_rfftx4(dnsb_ctx *c, int mode, const double *a, const double *b, const double *cc) {
  const Geo &g = c->g;
  dim3 grid(g.ny * ((g.nz + RFX_L - 1) / RFX_L));
#define RF4(A, B)                                                                                  \
  if (c->x1 == A && c->x2 == B) {                                                                  \
    if (mode == RIN_DIVERGENCE && c->rx_post)                                                      \
      LAUNCH(c, DNSB_KIND_RFFTX, k_rfftx4<A, B, RFX_L, RIN_DIVERGENCE, true><<<grid, F4_THREADS, c->smem_rx4, c->stream>>>(g, c->S, a, b, cc, c->twM, c->twN)); \
    else if (mode == RIN_DIVERGENCE)                                                               \
      LAUNCH(c, DNSB_KIND_RFFTX, k_rfftx4<A, B, RFX_L, RIN_DIVERGENCE><<<grid, F4_THREADS, c->smem_rx4, c->stream>>>(g, c->S, a, b, cc, c->twM, c->twN)); \
    else if (mode == RIN_REAL)                                                                     \
      LAUNCH(c, DNSB_KIND_RFFTX, k_rfftx4<A, B, RFX_L, RIN_REAL><<<grid, F4_THREADS, c->smem_rx4, c->stream>>>(g, c->S, a, b, cc, c->twM, c->twN)); \
    else if (mode == RIN_PRODUCT)                                                                  \
      LAUNCH(c, DNSB_KIND_RFFTX, k_rfftx4<A, B, RFX_L, RIN_PRODUCT><<<grid, F4_THREADS, c->smem_rx4, c->stream>>>(g, c->S, a, b, cc, c->twM, c->twN)); \
    else                                                                                           \
      LAUNCH(c, DNSB_KIND_RFFTX, k_rfftx4<A, B, RFX_L, RIN_FIELD><<<grid, F4_THREADS, c->smem_rx4, c->stream>>>(g, c->S, a, b, cc, c->twM, c->twN)); \
    return 0;                                                                                      \
  }
  FFT4_SPLITS(RF4)
#undef RF4
  return fail(c, DNSB_EUNSUP, "no four-step x kernel for %d x %d", c->x1, c->x2);
}

int launch_irfftx4(dnsb_ctx *c, int mode, double *out) {
  const Geo &g = c->g;
  dim3 grid(g.ny * ((g.nz + IRX_L - 1) / IRX_L));
#define IF4(A, B)                                                                                  \
  if (c->x1 == A && c->x2 == B) {                                                                  \
    if (mode == ROUT_INTERIOR)                                                                     \
      LAUNCH(c, DNSB_KIND_IRFFTX, k_irfftx4<A, B, IRX_L, ROUT_INTERIOR><<<grid, F4_THREADS, c->smem_ix4, c->stream>>>(g, c->S, out, c->twM, c->twN)); \
    else if (mode == ROUT_IMAGES)                                                                  \
      { if (c->ix_pairs) LAUNCH(c, DNSB_KIND_IRFFTX, k_irfftx4<A, B, IRX_L, ROUT_IMAGES, true><<<grid, F4_THREADS, c->smem_ix4, c->stream>>>(g, c->S, out, c->twM, c->twN)); \
        else LAUNCH(c, DNSB_KIND_IRFFTX, k_irfftx4<A, B, IRX_L, ROUT_IMAGES><<<grid, F4_THREADS, c->smem_ix4, c->stream>>>(g, c->S, out, c->twM, c->twN)); } \
    else                                                                                           \
      LAUNCH(c, DNSB_KIND_IRFFTX, k_irfftx4<A, B, IRX_L, ROUT_REAL><<<grid, F4_THREADS, c->smem_ix4, c->stream>>>(g, c->S, out, c->twM, c->twN)); \
    return 0;                                                                                      \
  }
  FFT4_SPLITS(IF4)
#undef IF4
  return fail(c, DNSB_EUNSUP, "no four-step x kernel for %d x %d", c->x1, c->x2);
}

int launch_fftz4(dnsb_ctx *c, bool inv) {
  const Geo &g = c->g;
  const long long nlines = (long long)g.ny * (c->nkx_active ? c->nkx_active : g.nkx);
  dim3 grid((unsigned)((nlines + c->L4z - 1) / c->L4z));
#define ZF4(A, B)                                                                                  \
  if (c->z1 == A && c->z2 == B) {                                                                  \
    if (inv) LAUNCH(c, DNSB_KIND_IFFTZ, k_fftz4<A, B, true><<<grid, F4_THREADS, c->smem_z4, c->stream>>>(g, c->S, c->L4z, c->twz)); \
    else LAUNCH(c, DNSB_KIND_FFTZ, k_fftz4<A, B, false><<<grid, F4_THREADS, c->smem_z4, c->stream>>>(g, c->S, c->L4z, c->twz)); \
    return 0;                                                                                      \
  }
  FFT4_SPLITS(ZF4)
#undef ZF4
  return fail(c, DNSB_EUNSUP, "no four-step z kernel for %d x %d", c->z1, c->z2);
}

// shared-memory opt-in of the four-step kernels of one split
template <int A, int B>
int allow_fft4(dnsb_ctx *c) {
  int rc;
  if ((rc = allow_smem(c, k_rfftx4<A, B, RFX_L, RIN_DIVERGENCE>, c->smem_rx4)) ||
      (rc = allow_smem(c, k_rfftx4<A, B, RFX_L, RIN_DIVERGENCE, true>, c->smem_rx4)) ||
      (rc = allow_smem(c, k_rfftx4<A, B, RFX_L, RIN_REAL>, c->smem_rx4)) ||
      (rc = allow_smem(c, k_rfftx4<A, B, RFX_L, RIN_FIELD>, c->smem_rx4)) ||
      (rc = allow_smem(c, k_rfftx4<A, B, RFX_L, RIN_PRODUCT>, c->smem_rx4)) ||
      (rc = allow_smem(c, k_irfftx4<A, B, IRX_L, ROUT_INTERIOR>, c->smem_ix4)) ||
      (rc = allow_smem(c, k_irfftx4<A, B, IRX_L, ROUT_IMAGES>, c->smem_ix4)) ||
      (rc = allow_smem(c, k_irfftx4<A, B, IRX_L, ROUT_IMAGES, true>, c->smem_ix4)) ||
      (rc = allow_smem(c, k_irfftx4<A, B, IRX_L, ROUT_REAL>, c->smem_ix4)) ||
      (rc = allow_smem(c, k_fftz4<A, B, false>, c->smem_z4)) ||
      (rc = allow_smem(c, k_fftz4<A, B, true>, c->smem_z4)))
    return rc;
  return 0;
}

int allow_fft4_split(dnsb_ctx *c, int a, int b) {
#define AF4(A, B) \
  if (a == A && b == B) return allow_fft4<A, B>(c);
  FFT4_SPLITS(AF4)
#undef AF4
  return 0;
}

// rfft_x of the divergence of (a, b, cc) (mode RIN_DIVERGENCE), of the
// ghost-free real a (RIN_REAL) or of the interior of field a (RIN_FIELD)
int launch_rfftx(dnsb_ctx *c, int mode, const double *a, const double *b, const double *cc) {
  const Geo &g = c->g;
  if (c->x1) return launch_rfftx4(c, mode, a, b, cc);
  dim3 grid(g.ny * ((g.nz + c->Lx - 1) / c->Lx));
  if (mode == RIN_DIVERGENCE)
    LAUNCH(c, DNSB_KIND_RFFTX, k_rfftx<RIN_DIVERGENCE><<<grid, SPEC_THREADS, c->smem_rx, c->stream>>>(g, c->S, a, b, cc, c->pM, c->Lx, c->twM, c->twN));
  else if (mode == RIN_REAL)
    LAUNCH(c, DNSB_KIND_RFFTX, k_rfftx<RIN_REAL><<<grid, SPEC_THREADS, c->smem_rx, c->stream>>>(g, c->S, a, b, cc, c->pM, c->Lx, c->twM, c->twN));
  else
    LAUNCH(c, DNSB_KIND_RFFTX, k_rfftx<RIN_FIELD><<<grid, SPEC_THREADS, c->smem_rx, c->stream>>>(g, c->S, a, b, cc, c->pM, c->Lx, c->twM, c->twN));
  return 0;
}

int launch_fftz(dnsb_ctx *c, bool inv) {
  const Geo &g = c->g;
  if (c->z1 && !c->use_tma) return launch_fftz4(c, inv);
  long long nlines = (long long)g.ny * (c->nkx_active && !c->use_tma ? c->nkx_active : g.nkx);
  if (c->use_tma) {
    const long long ngroups = (nlines + c->Lz - 1) / c->Lz;
    dim3 grid((unsigned)std::min<long long>(ngroups, 2LL * c->nsm));
    if (inv) LAUNCH(c, DNSB_KIND_IFFTZ, k_fftz_tma<true><<<grid, SPEC_THREADS, c->smem_zt, c->stream>>>(g, c->S, c->pz, c->Lz, c->twz, c->deverr, c->wait_limit));
    else LAUNCH(c, DNSB_KIND_FFTZ, k_fftz_tma<false><<<grid, SPEC_THREADS, c->smem_zt, c->stream>>>(g, c->S, c->pz, c->Lz, c->twz, c->deverr, c->wait_limit));
    return 0;
  }
  dim3 grid((unsigned)((nlines + c->Lz - 1) / c->Lz));
  if (inv) LAUNCH(c, DNSB_KIND_IFFTZ, k_fftz<true><<<grid, SPEC_THREADS, c->smem_z, c->stream>>>(g, c->S, c->pz, c->Lz, c->twz));
  else LAUNCH(c, DNSB_KIND_FFTZ, k_fftz<false><<<grid, SPEC_THREADS, c->smem_z, c->stream>>>(g, c->S, c->pz, c->Lz, c->twz));
  return 0;
}

int launch_ysolve(dnsb_ctx *c) {
  const Geo &g = c->g;
  if (g.wall) {
    const long long n = (long long)g.nkx * g.nz;
    const dim3 grid((unsigned)((n + TY_LINES - 1) / TY_LINES)), block(TY_LINES, TY_CHUNKS);
#define YT(MR)                                                                                    \
  case MR:                                                                                        \
    LAUNCH(c, DNSB_KIND_YSOLVE,                                                                   \
           k_ythomas<MR><<<grid, block, ythomas_smem(MR), c->stream>>>(g, c->S, c->ycin, c->ay,   \
                                                        c->by, c->cy, c->lam1, c->lam3));         \
    break;
    switch (ythomas_rows(g.ny)) {
      YT(1) YT(2) YT(3) YT(4) YT(6) YT(8) YT(12) YT(16)
      default:
        LAUNCH(c, DNSB_KIND_YSOLVE,
               k_thomas<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(
                   g, c->S, c->work, c->ay, c->by, c->cy, c->lam1, c->lam3));
    }
#undef YT
  } else {
    dim3 grid(g.nkx * ((g.nz + c->Ly - 1) / c->Ly));
    LAUNCH(c, DNSB_KIND_YSOLVE, k_yfourier<YF_SOLVE><<<grid, SPEC_THREADS, c->smem_y, c->stream>>>(g, c->S, c->py, c->Ly, c->twy, c->lam1, c->lam2, c->lam3));
  }
  return 0;
}

int launch_irfftx(dnsb_ctx *c, int mode, double *out) {
  const Geo &g = c->g;
  if (c->x1) return launch_irfftx4(c, mode, out);
  dim3 grid(g.ny * ((g.nz + c->Lx - 1) / c->Lx));
  if (mode == ROUT_INTERIOR)
    LAUNCH(c, DNSB_KIND_IRFFTX, k_irfftx<ROUT_INTERIOR><<<grid, SPEC_THREADS, c->smem_ix, c->stream>>>(g, c->S, out, c->pM, c->Lx, c->twM, c->twN));
  else if (mode == ROUT_IMAGES)
    LAUNCH(c, DNSB_KIND_IRFFTX, k_irfftx<ROUT_IMAGES><<<grid, SPEC_THREADS, c->smem_ix, c->stream>>>(g, c->S, out, c->pM, c->Lx, c->twM, c->twN));
  else
    LAUNCH(c, DNSB_KIND_IRFFTX, k_irfftx<ROUT_REAL><<<grid, SPEC_THREADS, c->smem_ix, c->stream>>>(g, c->S, out, c->pM, c->Lx, c->twM, c->twN));
  return 0;
}

// k_zyz (mode 1) or k_zyz2 (mode 2) for this context's z split: one cluster
// of zyz_c CTAs per kx plane
template <int N1, int N2>
cudaError_t launch_zyz_as(dnsb_ctx *c, bool query, int *nclusters) {
  const Geo &g = c->g;
  const bool two = c->zyz_mode == 2;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)c->zyz_c;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)(g.nkx * c->zyz_c));
  cfg.blockDim = dim3(two ? ZYZ2_THREADS : ZYZ_THREADS);
  cfg.dynamicSmemBytes = two ? zyz2_smem<N1, N2>() : zyz_smem<N1, N2>();
  cfg.stream = c->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  auto kern = two ? k_zyz2<N1, N2> : k_zyz<N1, N2>;
  if (query) return cudaOccupancyMaxActiveClusters(nclusters, kern, &cfg);
  return cudaLaunchKernelEx(&cfg, kern, g, c->S, (const double *)c->ycin, (const double *)c->ay,
                            (const double *)c->by, (const double *)c->cy, (const double *)c->lam1,
                            (const double *)c->lam3, (const double2 *)c->twz);
}

cudaError_t launch_zyz_split(dnsb_ctx *c, bool query, int *nclusters) {
  if (c->z1 == 16 && c->z2 == 24) return launch_zyz_as<16, 24>(c, query, nclusters);
  if (c->z1 == 16 && c->z2 == 16) return launch_zyz_as<16, 16>(c, query, nclusters);
  return cudaErrorInvalidValue;
}

template <class K>
int allow_cluster_kernel(dnsb_ctx *c, K kern, size_t smem, bool nonportable) {
  int rc = allow_smem(c, kern, smem);
  if (rc) return rc;
  if (nonportable &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return -1;  // not available: the caller falls back
  }
  return 0;
}

// Chooses the fused z-FFT / y-solve / inverse z-FFT kernel where it applies:
// walls, nz in {256, 384} (four-step 16 x 16 / 16 x 24), ny a multiple of
// the chunk rows (32 for mode 1, 16 for mode 2) with at most 8 (16) chunks,
// and a cluster of that size can be resident.
int setup_zyz(dnsb_ctx *c, int mode) {
  const Geo &g = c->g;
  c->zyz_c = 0;
  c->zyz_mode = mode == 2 ? 2 : 1;
  if (!(c->z1 == 16 && (c->z2 == 24 || c->z2 == 16))) return 0;
  const int rows = c->zyz_mode == 2 ? ZYZ2_ROWS : ZYZ_ROWS;
  const int maxc = c->zyz_mode == 2 ? ZYZ2_MAXC : ZYZ_MAXC;
  if (g.ny % rows != 0 || g.ny / rows > maxc) return 0;
  const int C = g.ny / rows;
  int rc;
  if (c->zyz_mode == 2) {
    rc = c->z2 == 24 ? allow_cluster_kernel(c, k_zyz2<16, 24>, zyz2_smem<16, 24>(), C > 8)
                     : allow_cluster_kernel(c, k_zyz2<16, 16>, zyz2_smem<16, 16>(), C > 8);
    if (rc < 0) return 0;
  } else {
    rc = c->z2 == 24 ? allow_smem(c, k_zyz<16, 24>, zyz_smem<16, 24>())
                     : allow_smem(c, k_zyz<16, 16>, zyz_smem<16, 16>());
  }
  if (rc) return rc;
  c->zyz_c = C;
  int n = 0;
  if (launch_zyz_split(c, true, &n) != cudaSuccess || n < 1) {
    cudaGetLastError();  // the query's error is not the context's
    c->zyz_c = 0;
  }
  return 0;
}

// S already holds rfft_x(rhs): finish the Poisson solve into out
int poisson_from_spectrum(dnsb_ctx *c, int outmode, double *out) {
  int rc;
  if (c->zyz_c) {
    LAUNCH(c, DNSB_KIND_ZYZ, CK(c, launch_zyz_split(c, false, nullptr)));
  } else {
    if ((rc = launch_fftz(c, false))) return rc;
    if ((rc = launch_ysolve(c))) return rc;
    if ((rc = launch_fftz(c, true))) return rc;
  }
  return launch_irfftx(c, outmode, out);
}

bool aligned16(const double *q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; }

// the z-marching momentum kernel copies 16-byte chunks of the velocity rows
typedef CUresult (*TmaEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

TmaEncodeFn tma_encoder() {
  static TmaEncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (TmaEncodeFn)p;
  });
  return fn;
}

// The five tensor maps (u*x, u*y, u*z, delta, p_in) of k_gradmom_tma: 3-D
// FP64 maps of the ghosted field, box GP_X x GP_Y x 1; cached per field
// pointer.  False (the caller runs k_gradmom_pipe) when a field is not
// 16-byte aligned, a row is not a multiple of 16 bytes, the last x tile
// has more wrap columns than the kernel's two registers per thread cover,
// or the driver has no encoder.
bool gm_tma_maps(dnsb_ctx *c, CFields3 us, const double *delta, const double *pin,
                 const CUtensorMap **out) {
  const Geo &g = c->g;
  const int nwrap = std::max(0, (int)(c->gmgrid.x - 1) * MC_X + GP_X - g.NX);
  if (g.NX % 2 || 5 * GP_Y * nwrap > 2 * MC_X * MC_Y) return false;
  const double *f[5] = {us.x, us.y, us.z, delta, pin};
  TmaEncodeFn enc = tma_encoder();
  if (!enc) return false;
  for (int i = 0; i < 5; i++) {
    if (!aligned16(f[i])) return false;
    auto it = c->gm_maps.find(f[i]);
    if (it == c->gm_maps.end()) {
      if (c->gm_maps.size() >= 64) c->gm_maps.clear();
      CUtensorMap m;
      const cuuint64_t dims[3] = {(cuuint64_t)g.NX, (cuuint64_t)g.NY, (cuuint64_t)g.NZ};
      const cuuint64_t strides[2] = {8ull * g.NX, 8ull * g.NX * g.NY};
      const cuuint32_t box[3] = {GP_X, GP_Y, 1}, es[3] = {1, 1, 1};
      if (enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(f[i]), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
      it = c->gm_maps.emplace(f[i], m).first;
    }
    out[i] = &it->second;
  }
  return true;
}

bool use_tile(const dnsb_ctx *c, const double *ux, const double *uy, const double *uz) {
  return c->mom_tile && aligned16(ux) && aligned16(uy) && aligned16(uz);
}

void launch_cn(dnsb_ctx *c, Fields3 out, CFields3 V, const double *tab) {
  const Geo &g = c->g;
  const dim3 grid = cn_grid(g), block(CN_LINES, CN_CHUNKS);
  switch (c->cn_mr) {
    case 1: k_cn<1><<<grid, block, c->smem_cn, c->stream>>>(g, out, V, tab); break;
    case 2: k_cn<2><<<grid, block, c->smem_cn, c->stream>>>(g, out, V, tab); break;
    case 4: k_cn<4><<<grid, block, c->smem_cn, c->stream>>>(g, out, V, tab); break;
    case 8: k_cn<8><<<grid, block, c->smem_cn, c->stream>>>(g, out, V, tab); break;
    case 16: k_cn<16><<<grid, block, c->smem_cn, c->stream>>>(g, out, V, tab); break;
    default: k_cn<32><<<grid, block, c->smem_cn, c->stream>>>(g, out, V, tab); break;
  }
}

int do_step(dnsb_ctx *c, double *ux, double *uy, double *uz, double *p, double *qx, double *qy,
            double *qz, double *delta, double dt) {
  const Geo &g = c->g;
  int rc;
  // projection + next momentum fused (needs 16-byte aligned planes to stage)
  const bool fused = c->implicit && c->fuse && c->pn && use_tile(c, ux, uy, uz) &&
                     aligned16(delta) && aligned16(p);
  CK(c, cudaMemsetAsync(c->umax, 0, 3 * UMAX_SLOTS * sizeof(unsigned long long), c->stream));
  if (c->implicit)
    LAUNCH(c, DNSB_KIND_OTHER,
           k_cn_tables<<<1, CN_TABLE_THREADS, 0, c->stream>>>(g.ny, c->cn_mr, CN_CHUNKS, c->ycoef, c->ytab, dt,
                                                g.visc, RK_AL[0], RK_AL[1], RK_AL[2]));
  for (int s = 0; s < 3; s++) {
    const double A = RK_A[s], B = RK_B[s], al = RK_AL[s];
    const int readq = A != 0.0;
    unsigned long long *um = s == 2 ? c->umax : nullptr;
    if (!c->implicit) {
      if (use_tile(c, ux, uy, uz))
        LAUNCH(c, DNSB_KIND_MOMENTUM,
               k_momentum_march<MOM_EXPLICIT><<<c->tgrid, c->tblock, 0, c->stream>>>(
                   g, ff(qx, qy, qz), cf(ux, uy, uz), ff(c->W[0], c->W[1], c->W[2]), nullptr, A,
                   dt, B, 0.0, readq, c->ymet, 0.0, c->mom_planes, c->dtp));
      else
        LAUNCH(c, DNSB_KIND_MOMENTUM,
               k_momentum<MOM_EXPLICIT><<<c->cgrid, c->cblock, 0, c->stream>>>(
                   g, ff(qx, qy, qz), cf(ux, uy, uz), ff(c->W[0], c->W[1], c->W[2]), nullptr, A,
                   dt, B, 0.0, readq, c->ymet, 0.0));
      if ((rc = launch_rfftx(c, RIN_DIVERGENCE, c->W[0], c->W[1], c->W[2]))) return rc;
      if ((rc = poisson_from_spectrum(c, ROUT_IMAGES, p))) return rc;
      LAUNCH(c, DNSB_KIND_GRAD,
             k_grad<GRAD_EXPLICIT><<<c->cgrid, c->cblock, 0, c->stream>>>(
                 g, ff(ux, uy, uz), cf(c->W[0], c->W[1], c->W[2]), p, nullptr, 0.0, um));
    } else {
      const double adt = al * dt;
      const double th = al * dt * g.visc / 2;
      if (s > 0 && fused) {
        // the momentum of this stage ran inside the previous stage's projection
      } else if (use_tile(c, ux, uy, uz))
        LAUNCH(c, DNSB_KIND_MOMENTUM,
               k_momentum_march<MOM_IMPLICIT><<<c->tgrid, c->tblock, 0, c->stream>>>(
                   g, ff(qx, qy, qz), cf(ux, uy, uz), ff(c->V[0], c->V[1], c->V[2]), p, A, dt, B,
                   adt, readq, c->ymet, th, c->mom_planes, c->dtp));
      else
        LAUNCH(c, DNSB_KIND_MOMENTUM,
               k_momentum<MOM_IMPLICIT><<<c->cgrid, c->cblock, 0, c->stream>>>(
                   g, ff(qx, qy, qz), cf(ux, uy, uz), ff(c->V[0], c->V[1], c->V[2]), p, A, dt, B,
                   adt, readq, c->ymet, th));
      LAUNCH(c, DNSB_KIND_CN,
             launch_cn(c, ff(ux, uy, uz), cf(c->V[0], c->V[1], c->V[2]),
                       c->ytab + (long long)s * 2 * cn_tab_stride(g.ny)));
      if ((rc = launch_rfftx(c, RIN_DIVERGENCE, ux, uy, uz))) return rc;
      if ((rc = poisson_from_spectrum(c, ROUT_IMAGES, delta))) return rc;
      if (s < 2 && fused) {
        // projection of this stage + momentum of the next; the pressure
        // goes p -> pn (stage 1) -> p (stage 2), never in place
        const double A1 = RK_A[s + 1], B1 = RK_B[s + 1], al1 = RK_AL[s + 1];
        const double *pin = s == 0 ? p : c->pn;
        double *pout = s == 0 ? c->pn : p;
        const CUtensorMap *mp[5];
        if (c->gm_pipe == 3 && gm_tma_maps(c, cf(ux, uy, uz), delta, pin, mp))
          LAUNCH(c, DNSB_KIND_GRADMOM,
                 k_gradmom_tma<<<c->gmgrid, c->tblock, GRADMOM_TMA_SMEM, c->stream>>>(
                     *mp[0], *mp[1], *mp[2], *mp[3], *mp[4], g, c->gm_planes, cf(ux, uy, uz), delta,
                     pin, pout, 1.0 / adt, ff(qx, qy, qz), ff(c->V[0], c->V[1], c->V[2]), A1, dt, B1,
                     al1 * dt, c->ymet, al1 * dt * g.visc / 2, c->deverr, c->wait_limit));
        else
        LAUNCH(c, DNSB_KIND_GRADMOM,
               (c->gm_pipe == 2 ? k_gradmom_deep : c->gm_pipe ? k_gradmom_pipe : k_gradmom_march)<<<
                   c->gmgrid, c->tblock,
                   c->gm_pipe == 2 ? GRADMOM_DEEP_SMEM : c->gm_pipe ? GRADMOM_PIPE_SMEM : GRADMOM_SMEM,
                   c->stream>>>(
                   g, c->gm_planes, cf(ux, uy, uz), delta, pin, pout, 1.0 / adt, ff(qx, qy, qz),
                   ff(c->V[0], c->V[1], c->V[2]), A1, dt, B1, al1 * dt, c->ymet,
                   al1 * dt * g.visc / 2));
      } else {
        LAUNCH(c, DNSB_KIND_GRAD,
               k_grad<GRAD_IMPLICIT><<<c->cgrid, c->cblock, 0, c->stream>>>(
                   g, ff(ux, uy, uz), cf(ux, uy, uz), delta, p, 1.0 / adt, um));
      }
    }
  }
  c->umax_for[0] = ux;
  c->umax_for[1] = uy;
  c->umax_for[2] = uz;
  return 0;
}

int do_project(dnsb_ctx *c, double *ux, double *uy, double *uz, double *psi) {
  const Geo &g = c->g;
  int rc;
  if ((rc = launch_rfftx(c, RIN_DIVERGENCE, ux, uy, uz))) return rc;
  if ((rc = poisson_from_spectrum(c, ROUT_IMAGES, psi))) return rc;
  LAUNCH(c, DNSB_KIND_GRAD,
         k_grad<GRAD_EXPLICIT><<<c->cgrid, c->cblock, 0, c->stream>>>(
             g, ff(ux, uy, uz), cf(ux, uy, uz), psi, nullptr, 0.0, nullptr));
  c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
  return 0;
}

int fill3(dnsb_ctx *c, double *ux, double *uy, double *uz) {
  const Geo &g = c->g;
  double *f[3] = {ux, uy, uz};
  for (int s = 0; s < 3; s++) {
    k_fill_ghosts<<<4 * 148, 256, 0, c->stream>>>(g, f[s], s);
    CKL(c);
  }
  return 0;
}

// reads the device error word (set by a kernel whose bounded wait ran out);
// the caller has synchronised the stream
int check_deverr(dnsb_ctx *c) {
  int e = 0;
  CK(c, cudaMemcpy(&e, c->deverr, sizeof(int), cudaMemcpyDeviceToHost));
  if (e != 0) {
    cudaMemset(c->deverr, 0, sizeof(int));
    return fail(c, DNSB_ECUDA, "a device-side wait ran out of its iteration limit (code %d)", e);
  }
  return 0;
}

int cfl_from_max(dnsb_ctx *c, double cfl, const unsigned long long *bits, double *dt_out) {
  const Geo &g = c->g;
  const double eps = 2.220446049250313e-16;
  double mx[3];
  for (int i = 0; i < 3; i++) {
    long long b = (long long)bits[i];
    memcpy(&mx[i], &b, sizeof(double));
  }
  const double c1 = g.dx / (mx[0] + eps), c2 = c->dymin / (mx[1] + eps), c3 = g.dz / (mx[2] + eps);
  const double conv = std::fmin(std::fmin(c1, c2), c3);
  const double invdy2 = c->implicit ? 0.0 : 1 / (c->dymin * c->dymin);
  const double diff = 1 / (2 * g.visc * (1 / (g.dx * g.dx) + invdy2 + 1 / (g.dz * g.dz)) + eps);
  *dt_out = std::fmin(cfl * conv, cfl * diff);
  return 0;
}

// --------------------------------------------- integer-wavenumber shells --
// Periodic boxes only.  Every velocity component is transformed on its own
// staggered grid; a real factor per shell |k| multiplies the same modes of
// all three components, so the discrete divergence stays zero.

int alloc_shells(dnsb_ctx *c) {
  const Geo &g = c->g;
  if (g.wall) return 0;
  const long long k2 = (long long)(g.nx / 2) * (g.nx / 2) + (long long)(g.ny / 2) * (g.ny / 2) +
                       (long long)(g.nz / 2) * (g.nz / 2);
  long long s = (long long)sqrt((double)k2);
  while (s * s > k2) s--;
  while ((s + 1) * (s + 1) <= k2) s++;
  c->nshell_max = (int)s + 1;
  int rc = dalloc(c, &c->shellpart, (size_t)RED_BLOCKS * SHELL_DET);
  if (rc) return rc;
  return dalloc(c, &c->shellbuf, 3 * (size_t)c->nshell_max);
}

// S = the 3-D transform of the interior of component u
int spectrum_of(dnsb_ctx *c, const double *u) {
  const Geo &g = c->g;
  int rc;
  if ((rc = launch_rfftx(c, RIN_FIELD, u, nullptr, nullptr))) return rc;
  if ((rc = launch_fftz(c, false))) return rc;
  dim3 grid(g.nkx * ((g.nz + c->Ly - 1) / c->Ly));
  k_yfourier<YF_FORWARD><<<grid, SPEC_THREADS, c->smem_y, c->stream>>>(g, c->S, c->py, c->Ly, c->twy,
                                                                       c->lam1, c->lam2, c->lam3);
  CKL(c);
  return 0;
}

// E[0..nb) (device) = energies of the floor shells, summed in a fixed order
// (bit-reproducible): per block and shell for nb <= SHELL_DET (the clamp
// forcing, every step), one block per shell otherwise
int shell_energies_dev(dnsb_ctx *c, const double *const u[3], double *E, int nb) {
  CK(c, cudaMemsetAsync(E, 0, nb * sizeof(double), c->stream));
  int rc;
  for (int comp = 0; comp < 3; comp++) {
    if ((rc = spectrum_of(c, u[comp]))) return rc;
    if (nb <= SHELL_DET) {
      k_binshells_det<<<RED_BLOCKS, 256, 0, c->stream>>>(c->g, c->S, c->shellpart);
      CKL(c);
      k_sum_shells<<<1, 32, 0, c->stream>>>(c->shellpart, RED_BLOCKS, nb, E);
    } else {
      k_binshells_byshell<<<nb, 256, 0, c->stream>>>(c->g, c->S, E);
    }
    CKL(c);
  }
  return 0;
}

// u <- u with shell s scaled by f[s] (device), s < nb; images rewritten
int shell_scale_dev(dnsb_ctx *c, double *const u[3], const double *f, int nb) {
  const Geo &g = c->g;
  int rc;
  for (int comp = 0; comp < 3; comp++) {
    if ((rc = spectrum_of(c, u[comp]))) return rc;
    k_scaleshells<<<RED_BLOCKS, 256, 0, c->stream>>>(g, c->S, f, nb);
    CKL(c);
    dim3 grid(g.nkx * ((g.nz + c->Ly - 1) / c->Ly));
    k_yfourier<YF_INVERSE><<<grid, SPEC_THREADS, c->smem_y, c->stream>>>(g, c->S, c->py, c->Ly, c->twy,
                                                                         c->lam1, c->lam2, c->lam3);
    CKL(c);
    if ((rc = launch_fftz(c, true))) return rc;
    if ((rc = launch_irfftx(c, ROUT_IMAGES, u[comp]))) return rc;
  }
  c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
  return 0;
}

// The clamp with the three spectra kept: each component is transformed
// once, its shell energies summed (fixed order), the factors formed, and
// the same spectra scaled and transformed back -- 6 transforms instead of
// the 9 of energies followed by rescale.  c->S is pointed at each
// component's buffer in turn and restored on every return.
struct SpecSwap {
  dnsb_ctx *c;
  double2 *s0;
  ~SpecSwap() { c->S = s0; }
};

__global__ void k_clamp_factors(const double *E, const double *eref, double *f, int nb);

int shell_clamp_dev(dnsb_ctx *c, double *const u[3], double *E, const double *er, double *f,
                    int nb) {
  const Geo &g = c->g;
  SpecSwap guard{c, c->S};
  double2 *Ss[3] = {c->S, c->Sx[0], c->Sx[1]};
  CK(c, cudaMemsetAsync(E, 0, nb * sizeof(double), c->stream));
  int rc;
  for (int comp = 0; comp < 3; comp++) {
    c->S = Ss[comp];
    if ((rc = spectrum_of(c, u[comp]))) return rc;
    if (nb <= SHELL_DET) {
      k_binshells_det<<<RED_BLOCKS, 256, 0, c->stream>>>(g, c->S, c->shellpart);
      CKL(c);
      k_sum_shells<<<1, 32, 0, c->stream>>>(c->shellpart, RED_BLOCKS, nb, E);
    } else {
      k_binshells_byshell<<<nb, 256, 0, c->stream>>>(g, c->S, E);
    }
    CKL(c);
  }
  k_clamp_factors<<<1, 256, 0, c->stream>>>(E, er, f, nb);
  CKL(c);
  for (int comp = 0; comp < 3; comp++) {
    c->S = Ss[comp];
    k_scaleshells<<<RED_BLOCKS, 256, 0, c->stream>>>(g, c->S, f, nb);
    CKL(c);
    dim3 grid(g.nkx * ((g.nz + c->Ly - 1) / c->Ly));
    k_yfourier<YF_INVERSE><<<grid, SPEC_THREADS, c->smem_y, c->stream>>>(g, c->S, c->py, c->Ly, c->twy,
                                                                         c->lam1, c->lam2, c->lam3);
    CKL(c);
    if ((rc = launch_fftz(c, true))) return rc;
    if ((rc = launch_irfftx(c, ROUT_IMAGES, u[comp]))) return rc;
  }
  c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
  return 0;
}

// shellforcing's closure (src/spectral/forcing.jl:50-55) on the device:
// f[s] = sqrt(eref[s] / E[s]) for forced shells (eref[s] >= 0) with E > 0, else 1
__global__ void k_clamp_factors(const double *E, const double *eref, double *f, int nb) {
  for (int s = threadIdx.x; s < nb; s += blockDim.x)
    f[s] = (eref[s] >= 0 && E[s] > 0) ? sqrt(eref[s] / E[s]) : 1.0;
}

// the shell-clamp reference table on the device (synchronous; skipped when
// it is already there, so that a captured clamp never synchronises)
// the clamp of shells 0..nb-1 by partial Fourier sums (lowshells.cuh)
bool clamp_direct(const dnsb_ctx *c, int nb) {
  const Geo &g = c->g;
  const int KM = nb - 1;
  return nb <= LS_KX && 2 * KM < g.nx && 2 * KM < g.ny && 2 * KM < g.nz;
}

int upload_eref(dnsb_ctx *c, const double *eref, int nb) {
  const Geo &g = c->g;
  int rc;
  if (clamp_direct(c, nb)) {
    if (!c->lsA) {  // scratch for the largest direct case and the x-phases (first clamp only)
      if ((rc = dalloc(c, &c->lsA, (size_t)3 * LS_KX * g.ny * g.nz)) ||
          (rc = dalloc(c, &c->lsB, (size_t)3 * LS_KX * g.nz * LS_KY)) ||
          (rc = dalloc(c, &c->lsG, (size_t)3 * LS_KX * LS_KY * LS_KY)) ||
          (rc = dalloc(c, &c->lsH, (size_t)3 * LS_KX * LS_KY * g.nz)) ||
          (rc = dalloc(c, &c->lsX, (size_t)g.nx)) || (rc = dalloc(c, &c->lsY, (size_t)g.ny)) ||
          (rc = dalloc(c, &c->lsZ, (size_t)g.nz)))
        return rc;
      k_ls_phases<<<(g.nx + 255) / 256, 256, 0, c->stream>>>(g.nx, c->lsX);
      k_ls_phases<<<(g.ny + 255) / 256, 256, 0, c->stream>>>(g.ny, c->lsY);
      k_ls_phases<<<(g.nz + 255) / 256, 256, 0, c->stream>>>(g.nz, c->lsZ);
      CKL(c);
    }
  } else if (!c->Sx[0]) {  // the transform clamp keeps all three spectra
    const size_t nspec = (size_t)g.nkx * g.ny * g.nz;
    if ((rc = dalloc(c, &c->Sx[0], nspec)) || (rc = dalloc(c, &c->Sx[1], nspec))) return rc;
  }
  if (c->eref_host.size() == (size_t)nb && std::equal(eref, eref + nb, c->eref_host.begin())) return 0;
  double *er = c->shellbuf + 2 * c->nshell_max;
  CK(c, cudaMemcpyAsync(er, eref, nb * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  c->eref_host.assign(eref, eref + nb);
  return 0;
}

int check_shells(dnsb_ctx *c, const void *ux, const void *uy, const void *uz) {
  if (!c) return DNSB_EINVAL;
  if (!ux || !uy || !uz) return fail(c, DNSB_EINVAL, "null field");
  if (c->g.wall) return fail(c, DNSB_EINVAL, "spectral operations require a fully periodic box");
  if (ensure_device(c)) return DNSB_ECUDA;
  return 0;
}

}  // namespace

// ================================================================== C ABI ==

extern "C" {

int dnsb_version(void) { return DNSB_VERSION; }

const char *dnsb_last_error(const dnsb_ctx *ctx) { return ctx ? ctx->err.c_str() : g_create_err; }

int dnsb_create(const dnsb_grid *gr, int device, void *stream, dnsb_ctx **out) {
  return dnsb_create_tuned(gr, nullptr, device, stream, out);
}

int dnsb_create_tuned(const dnsb_grid *gr, const dnsb_tuning *tun, int device, void *stream,
                      dnsb_ctx **out) {
  if (!gr || !out) return fail(nullptr, DNSB_EINVAL, "null argument");
  if (tun && (tun->lines_x < 0 || tun->lines_z < 0 || tun->lines_y < 0 || tun->lines_z4 < 0 ||
              tun->cell_bx < 0 || tun->cell_by < 0 || tun->gm_planes < 0))
    return fail(nullptr, DNSB_EINVAL, "tuning values must be >= 0 (0: default)");
  // an explicit tuning value wins over the DNSB_* environment default
  auto tuned = [&](int v, const char *env, int dflt) { return v > 0 ? v : envint(env, dflt); };
  *out = nullptr;
  const int nx = gr->nx, ny = gr->ny, nz = gr->nz;
  if (nx < 2 || ny < 2 || nz < 1 || nx % 2)
    return fail(nullptr, DNSB_EINVAL, "need nx >= 2 even, ny >= 2, nz >= 1 (got %d %d %d)", nx, ny, nz);
  if (gr->bc_y != DNSB_BC_PERIODIC && gr->bc_y != DNSB_BC_WALL)
    return fail(nullptr, DNSB_EINVAL, "bc[2] must be :periodic or :wall");
  if (gr->ydiffusion != DNSB_YDIFF_EXPLICIT && gr->ydiffusion != DNSB_YDIFF_IMPLICIT)
    return fail(nullptr, DNSB_EINVAL, "ydiffusion must be :explicit or :implicit");
  if (gr->ydiffusion == DNSB_YDIFF_IMPLICIT && gr->bc_y != DNSB_BC_WALL)
    return fail(nullptr, DNSB_EINVAL, "implicit y-diffusion requires bc[2] == :wall");
  if (!gr->dy || !gr->dyu) return fail(nullptr, DNSB_EINVAL, "dy/dyu missing");
  const int M = nx / 2;
  if (M > 4096 || nz > 4096 || ny > 4096)
    return fail(nullptr, DNSB_EUNSUP, "FFT lengths above 4096 are not supported");
  if ((long long)(nx + 2) * (ny + 2) * (nz + 2) >= (1LL << 31))
    return fail(nullptr, DNSB_EUNSUP, "ghosted fields of 2^31 or more values are not supported");
  dnsb_ctx *c = new dnsb_ctx();
  c->device = device;
  c->stream = (cudaStream_t)stream;
  c->implicit = gr->ydiffusion == DNSB_YDIFF_IMPLICIT;
  auto bail = [&](int rc) {
    g_create_err[0] = 0;
    snprintf(g_create_err, sizeof g_create_err, "%s", c->err.c_str());
    dnsb_destroy(c);
    return rc;
  };
  if (cudaSetDevice(device) != cudaSuccess) {
    fail(c, DNSB_ECUDA, "cudaSetDevice(%d) failed", device);
    return bail(DNSB_ECUDA);
  }
  if (!make_fft_plan(M, c->pM) || !make_fft_plan(nz, c->pz) ||
      (gr->bc_y == DNSB_BC_PERIODIC && !make_fft_plan(ny, c->py))) {
    fail(c, DNSB_EUNSUP, "FFT lengths nx/2=%d, nz=%d%s must factor into 2, 3, 5", M, nz,
         gr->bc_y == DNSB_BC_PERIODIC ? ", ny" : "");
    return bail(DNSB_EUNSUP);
  }
  Geo &g = c->g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.NX = nx + 2; g.NY = ny + 2; g.NZ = nz + 2;
  g.wall = gr->bc_y == DNSB_BC_WALL;
  g.jymax = g.wall ? ny - 1 : ny;
  g.nkx = M + 1;
  g.dx = gr->dx; g.dz = gr->dz;
  g.rdx = 1.0 / g.dx; g.rdz = 1.0 / g.dz;
  g.rdx2 = 1.0 / (g.dx * g.dx); g.rdz2 = 1.0 / (g.dz * g.dz);
  g.visc = gr->visc;
  g.fx = gr->bodyforce[0]; g.fy = gr->bodyforce[1]; g.fz = gr->bodyforce[2];
  g.epsy = c->implicit ? 0.0 : 1.0;  // src/setup.jl:108

  std::vector<double> dy(gr->dy, gr->dy + ny + 2), dyu(gr->dyu, gr->dyu + ny + 2);
  std::vector<double> rdy(ny + 2), rdyu(ny + 2);
  for (int J = 0; J < ny + 2; J++) { rdy[J] = 1.0 / dy[J]; rdyu[J] = 1.0 / dyu[J]; }
  c->dymin = dy[1];
  for (int J = 1; J <= ny; J++) c->dymin = std::fmin(c->dymin, dy[J]);
  int rc;
  if ((rc = upload(c, &c->dy, dy)) || (rc = upload(c, &c->dyu, dyu)) ||
      (rc = upload(c, &c->rdy, rdy)) || (rc = upload(c, &c->rdyu, rdyu)))
    return bail(rc);
  g.dy = c->dy; g.dyu = c->dyu; g.rdy = c->rdy; g.rdyu = c->rdyu;

  // plan_poisson (src/poisson.jl:56-120), w = 1: Julia's Δye[j+w] is dy[j]
  std::vector<double> lam1(g.nkx), lam3(nz), lam2(ny);
  for (int k = 1; k <= g.nkx; k++) lam1[k - 1] = modlam(k, nx, g.dx);
  for (int k = 1; k <= nz; k++) lam3[k - 1] = modlam(k, nz, g.dz);
  for (int k = 1; k <= ny; k++) lam2[k - 1] = modlam(k, ny, dy[1]);
  std::vector<double> ay(ny, 0.0), by(ny, 0.0), cy(ny, 0.0);
  if (g.wall) {
    for (int j = 1; j <= ny; j++) {
      double a = j == 1 ? 0.0 : 1 / (dy[j] * dyu[j - 1]);
      double cc = j == ny ? 0.0 : 1 / (dy[j] * dyu[j]);
      ay[j - 1] = a; cy[j - 1] = cc; by[j - 1] = -(a + cc);
    }
  } else {
    double mx = dy[1], mn = dy[1];
    for (int J = 1; J <= ny; J++) { mx = std::fmax(mx, dy[J]); mn = std::fmin(mn, dy[J]); }
    if (!(mx - mn < 1e-12 * mx)) {
      fail(c, DNSB_EINVAL, "periodic y requires a uniform grid (stretch = identity)");
      return bail(DNSB_EINVAL);
    }
  }
  // ydiffusion_coefficients (src/ydiffusion.jl:31-51)
  std::vector<double> yc(6 * (size_t)ny, 0.0);
  double *at = yc.data(), *bt = at + ny, *ct = bt + ny, *an = ct + ny, *bn = an + ny, *cn = bn + ny;
  for (int j = 1; j <= ny; j++) {
    double a = 1 / (dy[j] * dyu[j - 1]);
    double cc = 1 / (dy[j] * dyu[j]);
    at[j - 1] = j == 1 ? 0.0 : a;
    ct[j - 1] = j == ny ? 0.0 : cc;
    bt[j - 1] = j == 1 ? -(cc + 2 * a) : j == ny ? -(a + 2 * cc) : -(a + cc);
  }
  for (int j = 1; j <= ny - 1; j++) {
    double a = 1 / (dyu[j] * dy[j]);
    double cc = 1 / (dyu[j] * dy[j + 1]);
    an[j - 1] = j == 1 ? 0.0 : a;
    cn[j - 1] = j == ny - 1 ? 0.0 : cc;
    bn[j - 1] = -(a + cc);
  }
  std::vector<double2> ym((size_t)YMET * (ny + 2), make_double2(0.0, 0.0));
  for (int J = 1; J <= ny; J++) {
    const int j = J - 1;
    double2 *r = ym.data() + (size_t)YMET * J;
    r[0] = make_double2(dy[J], dy[J + 1]);
    r[1] = make_double2(1.0 / dy[J], 1.0 / dy[J + 1]);
    r[2] = make_double2(1.0 / dyu[J], 1.0 / dyu[J - 1]);
    r[3] = make_double2(at[j], bt[j]);
    r[4] = make_double2(ct[j], an[j]);
    r[5] = make_double2(bn[j], cn[j]);
  }
  std::vector<double2> twM(M), twN(M + 1), twz(nz), twy(ny);
  for (int t = 0; t < M; t++) twM[t] = unit_root(t, M);
  for (int t = 0; t <= M; t++) twN[t] = unit_root(t, nx);
  for (int t = 0; t < nz; t++) twz[t] = unit_root(t, nz);
  for (int t = 0; t < ny; t++) twy[t] = unit_root(t, ny);
  if ((rc = upload(c, &c->lam1, lam1)) || (rc = upload(c, &c->lam2, lam2)) ||
      (rc = upload(c, &c->lam3, lam3)) || (rc = upload(c, &c->ay, ay)) ||
      (rc = upload(c, &c->by, by)) || (rc = upload(c, &c->cy, cy)) ||
      (rc = upload(c, &c->ycoef, yc)) || (rc = upload(c, &c->ymet, ym)) ||
      (rc = upload(c, &c->twM, twM)) ||
      (rc = upload(c, &c->twN, twN)) || (rc = upload(c, &c->twz, twz)) ||
      (rc = upload(c, &c->twy, twy)))
    return bail(rc);
  if ((rc = dalloc(c, &c->ytab, 6 * (size_t)cn_tab_stride(ny)))) return bail(rc);
  c->cn_mr = 1;
  while (c->cn_mr * CN_CHUNKS < ny) c->cn_mr *= 2;
  c->smem_cn = sizeof(double) * (5 * (size_t)cn_skew_pitch(ny, c->cn_mr) + 2 * CN_CHUNKS + 2 * CN_CHUNKS * CN_LINES);
  if (c->implicit && c->cn_mr > 32) {
    fail(c, DNSB_EUNSUP, "semi-implicit y-diffusion supports ny <= %d", 32 * CN_CHUNKS);
    return bail(DNSB_EUNSUP);
  }
  if ((rc = allow_smem(c, k_cn<1>, c->smem_cn)) || (rc = allow_smem(c, k_cn<2>, c->smem_cn)) ||
      (rc = allow_smem(c, k_cn<4>, c->smem_cn)) || (rc = allow_smem(c, k_cn<8>, c->smem_cn)) ||
      (rc = allow_smem(c, k_cn<16>, c->smem_cn)) || (rc = allow_smem(c, k_cn<32>, c->smem_cn)))
    return bail(rc);

  // launch shapes: L lines per CTA, two line buffers each within ~100 KB;
  // DNSB_LX / DNSB_LZ / DNSB_LY / DNSB_CELL_BLOCK ("32x8") override them
  auto pow2floor = [](int v) { int p = 1; while (2 * p <= v) p *= 2; return p; };
  const int budget = 100 * 1024 / (2 * (int)sizeof(double2));  // complex per buffer
  c->Lx = pow2floor(std::max(1, std::min({std::max(1, tuned(tun ? tun->lines_x : 0, "DNSB_LX", 8)),
                                            nz, budget / (M + 2)})));
  c->Lz = std::max(1, std::min(std::max(1, tuned(tun ? tun->lines_z : 0, "DNSB_LZ", 4)), budget / (nz + 1)));
  c->Ly = pow2floor(std::max(1, std::min({std::max(1, tuned(tun ? tun->lines_y : 0, "DNSB_LY", 8)),
                                            nz, budget / ny})));
  {
    int bx = 64, by = 2;
    const char *e = getenv("DNSB_CELL_BLOCK");
    if (tun && tun->cell_bx > 0 && tun->cell_by > 0) {
      bx = tun->cell_bx;
      by = tun->cell_by;
      if (bx * by > 256 || bx % 32 != 0)
        return bail(fail(c, DNSB_EINVAL, "cell block %dx%d: need a multiple of 32 wide, <= 256 threads", bx, by));
    } else if (e && sscanf(e, "%dx%d", &bx, &by) == 2 && bx > 0 && by > 0 && bx * by <= 256 && bx % 32 == 0) {
    } else { bx = 64; by = 2; }
    c->cblock = dim3(bx, by, 1);
    c->cgrid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, nz);
    c->mom_tile = envint("DNSB_MOMTILE", 1) != 0;
    c->fuse = envint("DNSB_FUSE", 1) != 0;
    c->tblock = dim3(MC_X, MC_Y, 1);
    c->tgrid = dim3((nx + MC_X - 1) / MC_X, (ny + MC_Y - 1) / MC_Y, (nz + MC_Z - 1) / MC_Z);
    c->gm_planes = std::max(4, std::min(256, tuned(tun ? tun->gm_planes : 0, "DNSB_GMZ", c->gm_planes)));
    c->gm_pipe = std::max(0, std::min(3, envint("DNSB_GMPIPE", c->gm_pipe)));
    c->gmgrid = dim3(c->tgrid.x, c->tgrid.y, (nz + c->gm_planes - 1) / c->gm_planes);
  }
  c->smem_rx = sizeof(double2) * (2 * (size_t)c->Lx * (M + 1) + M + (M + 1));
  c->smem_ix = sizeof(double2) * (2 * (size_t)c->Lx * (M + 2) + M + (M + 1));
  c->smem_z = sizeof(double2) * (2 * (size_t)c->Lz * (nz + 1) + nz);
  c->smem_y = sizeof(double2) * (2 * (size_t)c->Ly * ny + ny);
  c->smem_zt = sizeof(double2) * (2 * (size_t)c->Lz * nz + 2 * (size_t)c->Lz * (nz + 1) + nz) + 16;
  // four-step kernels for the lengths with a register split (DNSB_FFT4=0: off)
  if (envint("DNSB_FFT4", 1) != 0) {
    int a = 0, b = 0;
    c->L4z = std::max(1, tuned(tun ? tun->lines_z4 : 0, "DNSB_L4Z", 8));
    c->rx_post = envint("DNSB_RXPOST", c->rx_post) != 0;
    c->ix_pairs = envint("DNSB_IXPAIRS", c->ix_pairs) != 0;
    if (fft4_split(M, a, b)) {
      c->x1 = a;
      c->x2 = b;
      const size_t pitch = b % 2 == 0 ? b + 1 : b;
      c->smem_rx4 = sizeof(double2) * ((size_t)RFX_L * (a * pitch + 1) + (size_t)RFX_L * (M + 1) + M + (M + 1));
      c->smem_ix4 = sizeof(double2) * ((size_t)IRX_L * (M + 2) + (size_t)IRX_L * (a * pitch + 1) + M + (M + 1));
    }
    if (fft4_split(nz, a, b)) {
      c->z1 = a;
      c->z2 = b;
      c->smem_z4 = sizeof(double2) * ((size_t)c->L4z * a * (b % 2 == 0 ? b + 1 : b) + nz);
    }
  }
  // the persistent TMA-pipelined z-FFT is opt-in: at the production size the
  // non-persistent kernel with more CTAs per SM is faster
  c->use_tma = envint("DNSB_TMA", 0) != 0 && c->smem_zt <= 200 * 1024;
  {
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && nsm > 0)
      c->nsm = nsm;
  }
  {
    // planes per momentum CTA: MC_Z, halved while the grid would give
    // fewer than two CTAs per SM (small boxes), DNSB_MOMZ overrides
    const long cols = (long)c->tgrid.x * c->tgrid.y;
    int mp = envint("DNSB_MOMZ", 0);
    if (mp <= 0) {
      mp = MC_Z;
      while (mp > 2 && cols * ((nz + mp - 1) / mp) < 2L * c->nsm) mp /= 2;
    }
    c->mom_planes = std::max(1, std::min(64, mp));
    c->tgrid.z = (nz + c->mom_planes - 1) / c->mom_planes;
  }
  if ((c->x1 && (rc = allow_fft4_split(c, c->x1, c->x2))) ||
      (c->z1 && (rc = allow_fft4_split(c, c->z1, c->z2))))
    return bail(rc);
  if ((rc = allow_smem(c, k_rfftx<RIN_DIVERGENCE>, c->smem_rx)) ||
      (rc = allow_smem(c, k_rfftx<RIN_REAL>, c->smem_rx)) ||
      (rc = allow_smem(c, k_rfftx<RIN_FIELD>, c->smem_rx)) ||
      (rc = allow_smem(c, k_irfftx<ROUT_INTERIOR>, c->smem_ix)) ||
      (rc = allow_smem(c, k_irfftx<ROUT_IMAGES>, c->smem_ix)) ||
      (rc = allow_smem(c, k_irfftx<ROUT_REAL>, c->smem_ix)) ||
      (rc = allow_smem(c, k_fftz<false>, c->smem_z)) ||
      (rc = allow_smem(c, k_fftz<true>, c->smem_z)) ||
      (rc = allow_smem(c, k_fftz_tma<false>, c->smem_zt)) ||
      (rc = allow_smem(c, k_fftz_tma<true>, c->smem_zt)) ||
      (rc = allow_smem(c, k_yfourier<YF_SOLVE>, c->smem_y)) ||
      (rc = allow_smem(c, k_yfourier<YF_FORWARD>, c->smem_y)) ||
      (rc = allow_smem(c, k_yfourier<YF_INVERSE>, c->smem_y)))
    return bail(rc);

  // scratch
  const size_t G = (size_t)g.NX * g.NY * g.NZ;
  const size_t nspec = (size_t)g.nkx * ny * nz;
  if ((rc = dalloc(c, &c->S, nspec)) || (rc = dalloc(c, &c->r, (size_t)nx * ny * nz)) ||
      (rc = dalloc(c, &c->umax, 3 * UMAX_SLOTS + 8)) || (rc = dalloc(c, &c->partial, RED_BLOCKS + 8)) ||
      (rc = alloc_shells(c)) ||
      (rc = dalloc(c, &c->deverr, 4)))
    return bail(rc);
  if (g.wall && ythomas_rows(ny) == 0 && (rc = dalloc(c, &c->work, nspec))) return bail(rc);
  // the fused z-FFT / y-solve / inverse z-FFT is opt-in: at 384 x 256 x 384
  // it measured 0.44-0.46 ms against 0.43 ms for the three kernels
  if (g.wall && !c->use_tma && envint("DNSB_ZYZ", 0) != 0 && (rc = setup_zyz(c, envint("DNSB_ZYZ", 0))))
    return bail(rc);
  if (g.wall && (c->zyz_c || ythomas_rows(ny) != 0)) {
#define YTS(MR)                                                                                    \
  if (ythomas_rows(ny) == MR && (rc = allow_smem(c, k_ythomas<MR>, ythomas_smem(MR)))) return bail(rc);
    YTS(1) YTS(2) YTS(3) YTS(4) YTS(6) YTS(8) YTS(12) YTS(16)
#undef YTS
    const long long nl = (long long)g.nkx * nz;
    if ((rc = dalloc(c, &c->ycin, (size_t)nl * TY_CHUNKS))) return bail(rc);
    k_ythomas_entries<<<(unsigned)((nl + 127) / 128), 128, 0, c->stream>>>(
        g, c->zyz_c ? (c->zyz_mode == 2 ? ZYZ2_ROWS : ZYZ_ROWS) : ythomas_rows(ny), c->ycin, c->ay,
        c->by, c->cy, c->lam1, c->lam3);
    if (cudaGetLastError() != cudaSuccess) {
      fail(c, DNSB_ECUDA, "launch of the y-solve table kernel failed");
      return bail(DNSB_ECUDA);
    }
  }
  for (int i = 0; i < 3; i++) {
    if (!c->implicit) {
      if ((rc = dalloc(c, &c->W[i], G))) return bail(rc);
      if (cudaMemset(c->W[i], 0, G * sizeof(double)) != cudaSuccess) {
        fail(c, DNSB_ECUDA, "cudaMemset failed");
        return bail(DNSB_ECUDA);
      }
    }
    if (c->implicit) {
      if ((rc = dalloc(c, &c->V[i], G))) return bail(rc);
    }
  }
  if (c->implicit && c->fuse) {
    if ((rc = dalloc(c, &c->pn, G))) return bail(rc);
    if ((rc = allow_smem(c, k_gradmom_march, GRADMOM_SMEM)) ||
        (rc = allow_smem(c, k_gradmom_pipe, GRADMOM_PIPE_SMEM)) ||
        (rc = allow_smem(c, k_gradmom_tma, GRADMOM_TMA_SMEM)) ||
        (rc = allow_smem(c, k_gradmom_deep, GRADMOM_DEEP_SMEM)))
      return bail(rc);
  }
  if (cudaMemset(c->deverr, 0, 4 * sizeof(int)) != cudaSuccess) {
    fail(c, DNSB_ECUDA, "cudaMemset failed");
    return bail(DNSB_ECUDA);
  }
  if (cudaMallocHost(&c->hostred, 8 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&c->hostumax, 3 * UMAX_SLOTS * sizeof(unsigned long long)) != cudaSuccess) {
    fail(c, DNSB_ENOMEM, "cudaMallocHost failed");
    return bail(DNSB_ENOMEM);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    fail(c, DNSB_ECUDA, "device synchronisation after setup failed");
    return bail(DNSB_ECUDA);
  }
  *out = c;
  return DNSB_OK;
}

void dnsb_destroy(dnsb_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  else cudaDeviceSynchronize();
  for (auto &e : c->evpool) cudaEventDestroy(e);
  for (void *p : c->allocs) cudaFree(p);
  if (c->hostred) cudaFreeHost(c->hostred);
  if (c->hostumax) cudaFreeHost(c->hostumax);
  for (auto &e : c->les_graphs) cudaGraphExecDestroy(e.exec);
  if (c->les_cap) cudaStreamDestroy(c->les_cap);
  delete c;
}

int dnsb_set_stream(dnsb_ctx *c, void *stream) {
  if (!c) return DNSB_EINVAL;
  c->stream = (cudaStream_t)stream;
  return 0;
}

int dnsb_get_tuning(const dnsb_ctx *c, dnsb_tuning *t) {
  if (!c || !t) return DNSB_EINVAL;
  t->lines_x = c->Lx;
  t->lines_z = c->Lz;
  t->lines_y = c->Ly;
  t->lines_z4 = c->L4z;
  t->cell_bx = (int)c->cblock.x;
  t->cell_by = (int)c->cblock.y;
  t->gm_planes = c->gm_planes;
  return 0;
}

int dnsb_set_wait_limit(dnsb_ctx *c, unsigned long polls) {
  if (!c) return DNSB_EINVAL;
  c->wait_limit = polls == 0 ? 0u : (unsigned)std::min<unsigned long>(polls, 0xffffffffUL);
  c->graph_gen++;
  return 0;
}

int dnsb_sync(dnsb_ctx *c) {
  if (!c) return DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  CK(c, cudaStreamSynchronize(c->stream));
  return check_deverr(c);
}

int dnsb_fill_ghosts(dnsb_ctx *c, double *phi, int stag) {
  if (!c || !phi || stag < 0 || stag > 3) return c ? fail(c, DNSB_EINVAL, "bad argument") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  k_fill_ghosts<<<4 * 148, 256, 0, c->stream>>>(c->g, phi, stag);
  CKL(c);
  c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
  return 0;
}

int dnsb_divergence(dnsb_ctx *c, double *r, const double *ux, const double *uy, const double *uz) {
  if (!c || !r || !ux || !uy || !uz) return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  k_divergence<<<cell_grid(c->g), cell_block, 0, c->stream>>>(c->g, r, cf(ux, uy, uz));
  CKL(c);
  return 0;
}

int dnsb_momentum(dnsb_ctx *c, double *qx, double *qy, double *qz, const double *ux,
                  const double *uy, const double *uz, double A, double dt) {
  if (!c || !qx || !qy || !qz || !ux || !uy || !uz)
    return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  if (use_tile(c, ux, uy, uz))
    k_momentum_march<MOM_ONLY><<<c->tgrid, c->tblock, 0, c->stream>>>(
        c->g, ff(qx, qy, qz), cf(ux, uy, uz), ff(nullptr, nullptr, nullptr), nullptr, A, dt, 0.0,
        0.0, 1, c->ymet, 0.0, c->mom_planes, c->dtp);
  else
    k_momentum<MOM_ONLY><<<cell_grid(c->g), cell_block, 0, c->stream>>>(
        c->g, ff(qx, qy, qz), cf(ux, uy, uz), ff(nullptr, nullptr, nullptr), nullptr, A, dt, 0.0,
        0.0, 1, c->ymet, 0.0);
  CKL(c);
  return 0;
}

int dnsb_pressuregrad(dnsb_ctx *c, double *phi, const double *p, int comp, double s) {
  if (!c || !phi || !p || comp < 0 || comp > 2)
    return c ? fail(c, DNSB_EINVAL, "bad argument") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  k_pgrad<<<cell_grid(c->g), cell_block, 0, c->stream>>>(c->g, phi, p, comp, s);
  CKL(c);
  c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
  return 0;
}

int dnsb_poisson(dnsb_ctx *c, const double *r, double *p) {
  if (!c || !r || !p) return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  int rc;
  if ((rc = launch_rfftx(c, RIN_REAL, r, nullptr, nullptr))) return rc;
  return poisson_from_spectrum(c, ROUT_INTERIOR, p);
}

// ---------------------------------------------- z-slab decomposition ---
// The pieces of poisson! between which a z-slab decomposition (the
// reference's (P,1) process grid: z split over ranks, transpose.jl:47-122)
// redistributes the spectrum: the real x-transform of a rank's planes into
// its context's spectrum ([kx][j][z], z fastest), the z-transform, y-solve
// and inverse z-transform of a kx-slab holding every z (on a context of the
// global grid, whose plans and tables it uses), and the inverse
// x-transform back into a rank's pressure.

__global__ void k_zblock_copy(double2 *__restrict__ dst, const double2 *__restrict__ src, int nkx,
                              int ny, int nz_dst, int z_dst, int nz_src, int z_src, int nz_copy) {
  const long long n = (long long)nkx * ny * nz_copy;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(t % nz_copy);
    const long long line = t / nz_copy;  // kx * ny + j
    dst[line * nz_dst + z_dst + z] = src[line * nz_src + z_src + z];
  }
}

__global__ void k_axpy_interior(Geo g, double *__restrict__ y, const double *__restrict__ x, double a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const int c0 = gidx(g, i + 1, j + 1, blockIdx.z + 1);
  y[c0] += a * x[c0];
}

int dnsb_axpy(dnsb_ctx *c, double *y, const double *x, double a) {
  if (!c || !y || !x) return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  k_axpy_interior<<<cell_grid(c->g), cell_block, 0, c->stream>>>(c->g, y, x, a);
  CKL(c);
  c->launches++;
  return 0;
}

int dnsb_poisson_x(dnsb_ctx *c, const double *r) {
  if (!c || !r) return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  return launch_rfftx(c, RIN_REAL, r, nullptr, nullptr);
}

int dnsb_poisson_xinv(dnsb_ctx *c, double *p) {
  if (!c || !p) return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  return launch_irfftx(c, ROUT_IMAGES, p);
}

int dnsb_poisson_zy(dnsb_ctx *c, void *S, int kx0, int nkx) {
  if (!c || !S) return c ? fail(c, DNSB_EINVAL, "null spectrum") : DNSB_EINVAL;
  if (kx0 < 0 || nkx < 1 || kx0 + nkx > c->g.nkx)
    return fail(c, DNSB_EINVAL, "kx-slab %d..%d outside 0..%d", kx0, kx0 + nkx - 1, c->g.nkx - 1);
  if (ensure_device(c)) return DNSB_ECUDA;
  // run the three launches on the caller's slab: the spectrum, the kx count
  // and the kx-indexed tables point at the slab for the duration
  double2 *S0 = c->S;
  const int nkx0 = c->g.nkx, act0 = c->nkx_active;
  double *lam1_0 = c->lam1, *ycin0 = c->ycin;
  c->S = (double2 *)S;
  c->g.nkx = nkx;
  c->nkx_active = 0;
  c->lam1 = lam1_0 + kx0;
  if (ycin0) c->ycin = ycin0 + (long long)kx0 * c->g.nz * TY_CHUNKS;
  int rc = launch_fftz(c, false);
  if (!rc) rc = launch_ysolve(c);
  if (!rc) rc = launch_fftz(c, true);
  c->S = S0;
  c->g.nkx = nkx0;
  c->nkx_active = act0;
  c->lam1 = lam1_0;
  c->ycin = ycin0;
  return rc;
}

int dnsb_spectrum(dnsb_ctx *c, void **S, int *nkx, int *ny, int *nz) {
  if (!c || !S) return DNSB_EINVAL;
  *S = c->S;
  if (nkx) *nkx = c->g.nkx;
  if (ny) *ny = c->g.ny;
  if (nz) *nz = c->g.nz;
  return 0;
}

int dnsb_zblock_copy(dnsb_ctx *c, void *dst, const void *src, int nkx, int ny, int nz_dst, int z_dst,
                     int nz_src, int z_src, int nz_copy) {
  if (!c || !dst || !src) return c ? fail(c, DNSB_EINVAL, "null buffer") : DNSB_EINVAL;
  if (nkx < 0 || ny < 0 || nz_copy < 0 || z_dst < 0 || z_src < 0 || z_dst + nz_copy > nz_dst ||
      z_src + nz_copy > nz_src)
    return fail(c, DNSB_EINVAL, "z-block outside its lines");
  if (ensure_device(c)) return DNSB_ECUDA;
  const long long n = (long long)nkx * ny * nz_copy;
  if (n == 0) return 0;
  const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 8LL * 148);
  k_zblock_copy<<<blocks, 256, 0, c->stream>>>((double2 *)dst, (const double2 *)src, nkx, ny, nz_dst,
                                               z_dst, nz_src, z_src, nz_copy);
  CKL(c);
  c->launches++;
  return 0;
}

int dnsb_project(dnsb_ctx *c, double *ux, double *uy, double *uz, double *psi) {
  if (!c || !ux || !uy || !uz || !psi) return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  return do_project(c, ux, uy, uz, psi);
}

// One explicit Runge-Kutta stage update with a sub-filter-stress closure on
// a periodic box (no counterpart in the reference): after momentum! has set
// q <- A q + dt F(u), add dt f_sfs to q, f_sfs = -div(tau) on the staggered
// faces, then u += B q (the explicit stage of step!, src/timestep.jl:52-57).
// tau holds 6 cell-centred components [xx, yy, zz, xy, yz, zx] of nx*ny*nz
// values (x fastest).  Normal stresses are differenced across the face
// (the two cells it separates); shear stresses are averaged onto the cell
// edges (four cells) and differenced across the face's cell in the
// transverse direction.  tau == NULL: the plain stage update.
__global__ void k_sfs_stage(Geo g, const double *__restrict__ tau, Fields3 q, Fields3 u, double dt,
                            double B, const double *__restrict__ dtp) {
  if (dtp) dt = *dtp;  // the step size from device memory (a step inside a CUDA graph)
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int I = i + 1, J = j + 1, K = k + 1;
  const long long n3 = (long long)g.nx * g.ny * g.nz;
  double f[3] = {0.0, 0.0, 0.0};
  if (tau) {
    // periodic neighbours, wrapped once per cell
    const int ip = i + 1 == g.nx ? 0 : i + 1, im = i == 0 ? g.nx - 1 : i - 1;
    const int jp = j + 1 == g.ny ? 0 : j + 1, jm = j == 0 ? g.ny - 1 : j - 1;
    const int kp = k + 1 == g.nz ? 0 : k + 1, km = k == 0 ? g.nz - 1 : k - 1;
    auto T = [&](int c, int a, int b, int d) {  // component c at cell (a, b, d), wrapped
      return __ldg(tau + c * n3 + ((long long)d * g.ny + b) * g.nx + a);
    };
    const double rdy = g.rdy[J], rdyu = g.rdyu[J];
    // x-face between cells i, i+1
    {
      const double dxx = (T(0, ip, j, k) - T(0, i, j, k)) * g.rdx;
      const double en = 0.25 * (T(3, i, j, k) + T(3, ip, j, k) + T(3, i, jp, k) + T(3, ip, jp, k));
      const double es = 0.25 * (T(3, i, j, k) + T(3, ip, j, k) + T(3, i, jm, k) + T(3, ip, jm, k));
      const double eu = 0.25 * (T(5, i, j, k) + T(5, ip, j, k) + T(5, i, j, kp) + T(5, ip, j, kp));
      const double ed = 0.25 * (T(5, i, j, k) + T(5, ip, j, k) + T(5, i, j, km) + T(5, ip, j, km));
      f[0] = -(dxx + (en - es) * rdy + (eu - ed) * g.rdz);
    }
    // y-face between cells j, j+1
    {
      const double dyy = (T(1, i, jp, k) - T(1, i, j, k)) * rdyu;
      const double ee = 0.25 * (T(3, i, j, k) + T(3, i, jp, k) + T(3, ip, j, k) + T(3, ip, jp, k));
      const double ew = 0.25 * (T(3, i, j, k) + T(3, i, jp, k) + T(3, im, j, k) + T(3, im, jp, k));
      const double eu = 0.25 * (T(4, i, j, k) + T(4, i, jp, k) + T(4, i, j, kp) + T(4, i, jp, kp));
      const double ed = 0.25 * (T(4, i, j, k) + T(4, i, jp, k) + T(4, i, j, km) + T(4, i, jp, km));
      f[1] = -((ee - ew) * g.rdx + dyy + (eu - ed) * g.rdz);
    }
    // z-face between cells k, k+1
    {
      const double dzz = (T(2, i, j, kp) - T(2, i, j, k)) * g.rdz;
      const double ee = 0.25 * (T(5, i, j, k) + T(5, i, j, kp) + T(5, ip, j, k) + T(5, ip, j, kp));
      const double ew = 0.25 * (T(5, i, j, k) + T(5, i, j, kp) + T(5, im, j, k) + T(5, im, j, kp));
      const double en = 0.25 * (T(4, i, j, k) + T(4, i, j, kp) + T(4, i, jp, k) + T(4, i, jp, kp));
      const double es = 0.25 * (T(4, i, j, k) + T(4, i, j, kp) + T(4, i, jm, k) + T(4, i, jm, kp));
      f[2] = -((ee - ew) * g.rdx + (en - es) * rdy + dzz);
    }
  }
  const int c0 = gidx(g, I, J, K);
  double *qs[3] = {q.x, q.y, q.z};
  double *us[3] = {u.x, u.y, u.z};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const double qn = qs[c][c0] + dt * f[c];
    qs[c][c0] = qn;
    store_img(us[c], g, I, J, K, us[c][c0] + B * qn, c);
  }
}

int dnsb_sfs_stage(dnsb_ctx *c, const double *tau, double *qx, double *qy, double *qz, double *ux,
                   double *uy, double *uz, double dt, double B) {
  if (!c || !qx || !qy || !qz || !ux || !uy || !uz)
    return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (c->g.wall && tau) return fail(c, DNSB_EINVAL, "the closure stage needs a periodic box");
  if (ensure_device(c)) return DNSB_ECUDA;
  k_sfs_stage<<<cell_grid(c->g), cell_block, 0, c->stream>>>(c->g, tau, ff(qx, qy, qz),
                                                             ff(ux, uy, uz), dt, B, c->dtp);
  CKL(c);
  c->launches++;
  c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
  return 0;
}

int dnsb_les_step(dnsb_ctx *c, dnsb_cnn *cnn, double *ux, double *uy, double *uz, double *p,
                  double *qx, double *qy, double *qz, double *tau, double dt) {
  if (!c || !ux || !uy || !uz || !p || !qx || !qy || !qz)
    return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (cnn && !tau) return fail(c, DNSB_EINVAL, "a closure needs the tau buffer");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(c, DNSB_EINVAL, "dt must be positive and finite");
  if (c->implicit) return fail(c, DNSB_EINVAL, "the LES step is explicit (ydiffusion = :explicit)");
  if (ensure_device(c)) return DNSB_ECUDA;
  if (cnn && dnsb_cnn_set_stream(cnn, c->stream))
    return fail(c, DNSB_ECUDA, "closure: %s", dnsb_cnn_last_error(cnn));
  for (int s = 0; s < 3; s++) {
    int rc;
    if (cnn && (rc = dnsb_cnn_infer(cnn, ux, uy, uz, tau)))
      return fail(c, rc, "closure: %s", dnsb_cnn_last_error(cnn));
    if ((rc = dnsb_momentum(c, qx, qy, qz, ux, uy, uz, RK_A[s], dt)) ||
        (rc = dnsb_sfs_stage(c, cnn ? tau : nullptr, qx, qy, qz, ux, uy, uz, dt, RK_B[s])) ||
        (rc = dnsb_project(c, ux, uy, uz, p)))
      return rc;
  }
  return 0;
}

// The CFL step of cfl_from_max on the device (the same correctly rounded
// operations in the same order, so the same bits as the host's), limited
// to t1 - t: st = {t, dt, steps, t1, threshold}; cfl_diff = cfl * the
// diffusive limit.
__global__ void k_les_dt(const unsigned long long *bits, double *st, double dx, double dymin, double dz,
                         double cfl, double cfl_diff) {
  const double eps = 2.220446049250313e-16;
  const double m0 = __longlong_as_double((long long)bits[0]);
  const double m1 = __longlong_as_double((long long)bits[1]);
  const double m2 = __longlong_as_double((long long)bits[2]);
  const double c1 = __ddiv_rn(dx, __dadd_rn(m0, eps)), c2 = __ddiv_rn(dymin, __dadd_rn(m1, eps));
  const double c3 = __ddiv_rn(dz, __dadd_rn(m2, eps));
  const double conv = fmin(fmin(c1, c2), c3);
  const double dt = fmin(__dmul_rn(cfl, conv), cfl_diff);
  const double left = __dsub_rn(st[3], st[0]);
  st[1] = left < dt ? left : dt;
}

// t += dt, one more step, and the loop condition t < st[4] for the next pass
__global__ void k_les_tick(double *st, cudaGraphConditionalHandle cond) {
  const double t = __dadd_rn(st[0], st[1]);
  st[0] = t;
  st[2] += 1.0;
  cudaGraphSetConditional(cond, t < st[4] ? 1u : 0u);
}

constexpr size_t LES_GRAPHS = 4;

// The graph of dnsb_les_advance: a conditional WHILE node whose body is one
// step (CFL maximum -> dt on the device -> the step with the kernels
// reading dt from device memory -> shell clamp -> t += dt and the loop
// condition).  The interval (t, t1, threshold) is device state, so one
// instantiation serves every later call with the same arguments.
int les_capture(dnsb_ctx *c, dnsb_cnn *cnn, double *ux, double *uy, double *uz, double *p, double *qx,
                double *qy, double *qz, double *tau, double cfl, const double *eref, int nshells, int nb,
                cudaGraphExec_t *out) {
  const Geo &g = c->g;
  int rc;
  // the diffusive limit exactly as cfl_from_max forms it
  const double eps = 2.220446049250313e-16;
  const double invdy2 = c->implicit ? 0.0 : 1 / (c->dymin * c->dymin);
  const double diff = 1 / (2 * g.visc * (1 / (g.dx * g.dx) + invdy2 + 1 / (g.dz * g.dz)) + eps);
  const double cfl_diff = cfl * diff;
  cudaGraph_t graph = nullptr, captured = nullptr;
  cudaGraphConditionalHandle cond;
  CK(c, cudaGraphCreate(&graph, 0));
  // (the captured graph is the WHILE node's body, owned by `graph`)
  auto drop = [&](int code) {
    cudaGraphDestroy(graph);
    return code;
  };
  if (cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess)
    return drop(fail(c, DNSB_ECUDA, "conditional handle creation failed"));
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = cond;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  if (cudaGraphAddNode(&wnode, graph, nullptr, 0, &wp) != cudaSuccess)
    return drop(fail(c, DNSB_ECUDA, "conditional node creation failed"));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  cudaStream_t orig = c->stream;
  {
    const cudaError_t se = cudaGetLastError();
    if (se != cudaSuccess) return drop(fail(c, DNSB_ECUDA, "error pending before the capture: %s", cudaGetErrorString(se)));
  }
  if (cudaStreamBeginCaptureToGraph(c->les_cap, body, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return drop(fail(c, DNSB_ECUDA, "stream capture could not start"));
  c->stream = c->les_cap;
  c->dtp = c->les_state + 1;
  unsigned long long *scratch = c->umax + 3 * UMAX_SLOTS;
  rc = 0;
  if (cudaMemsetAsync(scratch, 0, 3 * sizeof(unsigned long long), c->stream) != cudaSuccess)
    rc = fail(c, DNSB_ECUDA, "capture: memset failed");
  auto launched = [&](const char *what) {
    const cudaError_t le = cudaGetLastError();
    return le == cudaSuccess ? 0 : fail(c, DNSB_ECUDA, "capture: %s: %s", what, cudaGetErrorString(le));
  };
  if (!rc) {
    k_maxabs3<<<maxabs_blocks(g), 256, 0, c->stream>>>(g, cf(ux, uy, uz), scratch, nullptr);
    rc = launched("velocity maxima");
  }
  if (!rc) {
    k_les_dt<<<1, 1, 0, c->stream>>>(scratch, c->les_state, g.dx, c->dymin, g.dz, cfl, cfl_diff);
    rc = launched("step size");
  }
  // the dt argument only passes the host-side checks: the kernels read *dtp
  if (!rc)
    rc = cnn ? dnsb_les_step(c, cnn, ux, uy, uz, p, qx, qy, qz, tau, 1.0)
             : dnsb_step(c, ux, uy, uz, p, qx, qy, qz, nullptr, 1.0);
  if (!rc && nb) rc = dnsb_shell_clamp(c, ux, uy, uz, eref, nshells);
  if (!rc) {
    k_les_tick<<<1, 1, 0, c->stream>>>(c->les_state, cond);
    rc = launched("time advance");
  }
  const cudaError_t ce = cudaStreamEndCapture(c->les_cap, &captured);
  c->stream = orig;
  c->dtp = nullptr;
  if (cnn) dnsb_cnn_set_stream(cnn, orig);
  if (rc) return drop(rc);
  if (ce != cudaSuccess) return drop(fail(c, DNSB_ECUDA, "stream capture failed: %s", cudaGetErrorString(ce)));
  if (cudaGraphInstantiate(out, graph, 0) != cudaSuccess)
    return drop(fail(c, DNSB_ECUDA, "graph instantiation failed"));
  return drop(0);
}

// dnsb_les_advance as one graph launch, with no host synchronisation until
// the end; the graph is captured on the first call with these arguments.
int les_advance_graph(dnsb_ctx *c, dnsb_cnn *cnn, double *ux, double *uy, double *uz, double *p,
                      double *qx, double *qy, double *qz, double *tau, double t0, double t1, double cfl,
                      const double *eref, int nshells, double *t_out, long *n_out) {
  int rc;
  const double thr = t1 - 1e-12 * (std::fabs(t1) + 1);
  if (!(t0 < thr)) {
    if (t_out) *t_out = t1;
    if (n_out) *n_out = 0;
    return 0;
  }
  if (!c->les_cap) CK(c, cudaStreamCreateWithFlags(&c->les_cap, cudaStreamNonBlocking));
  if (!c->les_state && (rc = dalloc(c, &c->les_state, 8))) return rc;
  const int nb = eref && nshells > 0 ? std::min(nshells, c->nshell_max) : 0;
  if (nb && (rc = upload_eref(c, eref, nb))) return rc;  // the clamp's table (scratch before a capture)
  const void *key[9] = {ux, uy, uz, p, qx, qy, qz, tau, cnn};
  const unsigned long long serial = cnn ? dnsb_internal::cnn_serial(cnn) : 0;
  cudaGraphExec_t exec = nullptr;
  for (auto &e : c->les_graphs)
    if (std::equal(key, key + 9, e.ptr) && e.serial == serial && e.cfl == cfl && e.nb == nb &&
        e.gen == c->graph_gen) {
      exec = e.exec;
      e.used = ++c->les_uses;
      break;
    }
  if (!exec) {
    if ((rc = les_capture(c, cnn, ux, uy, uz, p, qx, qy, qz, tau, cfl, eref, nshells, nb, &exec))) return rc;
    if (c->les_graphs.size() >= LES_GRAPHS) {
      auto old = std::min_element(c->les_graphs.begin(), c->les_graphs.end(),
                                  [](const dnsb_ctx::LesGraph &a, const dnsb_ctx::LesGraph &b) {
                                    return a.used < b.used;
                                  });
      cudaGraphExecDestroy(old->exec);
      c->les_graphs.erase(old);
    }
    dnsb_ctx::LesGraph e{};
    std::copy(key, key + 9, e.ptr);
    e.serial = serial;
    e.cfl = cfl;
    e.nb = nb;
    e.gen = c->graph_gen;
    e.used = ++c->les_uses;
    e.exec = exec;
    c->les_graphs.push_back(e);
  }
  double *h = c->hostred;
  h[0] = t0;
  h[1] = 0.0;
  h[2] = 0.0;
  h[3] = t1;
  h[4] = thr;
  if (cudaMemcpyAsync(c->les_state, h, 5 * sizeof(double), cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
      cudaGraphLaunch(exec, c->stream) != cudaSuccess ||
      cudaMemcpyAsync(h, c->les_state, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return fail(c, DNSB_ECUDA, "graph launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  if ((rc = check_deverr(c))) return rc;
  c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
  if (t_out) *t_out = t1;
  if (n_out) *n_out = (long)h[2];
  return 0;
}

int dnsb_les_advance(dnsb_ctx *c, dnsb_cnn *cnn, double *ux, double *uy, double *uz, double *p,
                     double *qx, double *qy, double *qz, double *tau, double t0, double t1,
                     double cfl, const double *eref, int nshells, double *t_out, long *n_out) {
  if (!c || !ux || !uy || !uz || !p || !qx || !qy || !qz)
    return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (!(cfl > 0) || !std::isfinite(t0) || !std::isfinite(t1))
    return fail(c, DNSB_EINVAL, "cfl must be positive and the times finite");
  if (ensure_device(c)) return DNSB_ECUDA;
  // one graph launch for the whole run where every kernel of the step can
  // read dt from device memory (the z-marching momentum: aligned fields),
  // no per-launch timing is on (the context's or the closure's) and the box
  // is explicit; DNSB_LESGRAPH=0 keeps the host loop
  const bool direct_clamp = !eref || nshells <= 0 || (!c->g.wall && clamp_direct(c, std::min(nshells, c->nshell_max)));
  if (envint("DNSB_LESGRAPH", 1) != 0 && !c->implicit && !c->prof_on && use_tile(c, ux, uy, uz) &&
      direct_clamp && !(cnn && dnsb_internal::cnn_profiling(cnn)))
    return les_advance_graph(c, cnn, ux, uy, uz, p, qx, qy, qz, tau, t0, t1, cfl, eref, nshells, t_out,
                             n_out);
  double t = t0;
  long n = 0;
  while (t < t1 - 1e-12 * (std::fabs(t1) + 1)) {
    double dt = 0;
    int rc = dnsb_cfl(c, ux, uy, uz, cfl, 0, &dt);
    if (rc) return rc;
    dt = std::min(dt, t1 - t);
    rc = cnn ? dnsb_les_step(c, cnn, ux, uy, uz, p, qx, qy, qz, tau, dt)
             : dnsb_step(c, ux, uy, uz, p, qx, qy, qz, nullptr, dt);
    if (rc) return rc;
    if (eref && nshells > 0 && (rc = dnsb_shell_clamp(c, ux, uy, uz, eref, nshells))) return rc;
    t += dt;
    n++;
  }
  if (t_out) *t_out = t1;
  if (n_out) *n_out = n;
  return 0;
}

int dnsb_imex_update(dnsb_ctx *c, double *ux, double *uy, double *uz, const double *qx,
                     const double *qy, const double *qz, const double *p, double B, double alpha,
                     double dt) {
  if (!c) return DNSB_EINVAL;
  if (!c->implicit) return fail(c, DNSB_EINVAL, "implicit y-diffusion requires ydiffusion = :implicit");
  if (!ux || !uy || !uz || !qx || !qy || !qz || !p) return fail(c, DNSB_EINVAL, "null field");
  if (ensure_device(c)) return DNSB_ECUDA;
  const Geo &g = c->g;
  const double adt = alpha * dt;
  const double th = alpha * dt * g.visc / 2;
  k_vupdate<<<cell_grid(g), cell_block, 0, c->stream>>>(
      g, ff(c->V[0], c->V[1], c->V[2]), cf(ux, uy, uz), cf(qx, qy, qz), p, B, adt, c->ymet, th);
  CKL(c);
  // tables for this alpha in stage slot 0
  k_cn_tables<<<1, CN_TABLE_THREADS, 0, c->stream>>>(g.ny, c->cn_mr, CN_CHUNKS, c->ycoef, c->ytab, dt, g.visc,
                                       alpha, alpha, alpha);
  CKL(c);
  launch_cn(c, ff(ux, uy, uz), cf(c->V[0], c->V[1], c->V[2]), c->ytab);
  CKL(c);
  c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
  return 0;
}

int dnsb_step(dnsb_ctx *c, double *ux, double *uy, double *uz, double *p, double *qx, double *qy,
              double *qz, double *delta, double dt) {
  if (!c || !ux || !uy || !uz || !p || !qx || !qy || !qz)
    return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (c->implicit && (!delta || delta == p))
    return fail(c, DNSB_EINVAL, "semi-implicit mode needs a separate delta field");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(c, DNSB_EINVAL, "dt must be positive and finite");
  if (ensure_device(c)) return DNSB_ECUDA;
  return do_step(c, ux, uy, uz, p, qx, qy, qz, delta, dt);
}

int dnsb_cfl(dnsb_ctx *c, const double *ux, const double *uy, const double *uz, double cfl,
             int use_step_max, double *dt_out) {
  if (!c || !ux || !uy || !uz || !dt_out) return c ? fail(c, DNSB_EINVAL, "null argument") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  const bool cached = use_step_max && c->umax_for[0] == ux && c->umax_for[1] == uy && c->umax_for[2] == uz;
  unsigned long long bits[3] = {0, 0, 0};
  unsigned long long *scratch = c->umax + 3 * UMAX_SLOTS;
  if (!cached) {
    CK(c, cudaMemsetAsync(scratch, 0, 3 * sizeof(unsigned long long), c->stream));
    k_maxabs3<<<maxabs_blocks(c->g), 256, 0, c->stream>>>(c->g, cf(ux, uy, uz), scratch, c->deverr);
    CKL(c);
    CK(c, cudaMemcpyAsync(c->hostred, scratch, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    memcpy(bits, c->hostred, sizeof bits);
    unsigned long long e = 0;
    memcpy(&e, (const char *)c->hostred + 3 * sizeof(unsigned long long), sizeof e);
    if (e != 0) {
      cudaMemset(c->deverr, 0, sizeof(int));
      return fail(c, DNSB_ECUDA, "a device-side wait ran out of its iteration limit (code %d)", (int)e);
    }
    return cfl_from_max(c, cfl, bits, dt_out);
  } else {
    CK(c, cudaMemcpyAsync(c->hostumax, c->umax, 3 * UMAX_SLOTS * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 3; k++)
      for (int s = 0; s < UMAX_SLOTS; s++) bits[k] = std::max(bits[k], c->hostumax[k * UMAX_SLOTS + s]);
  }
  int rc = check_deverr(c);
  if (rc) return rc;
  return cfl_from_max(c, cfl, bits, dt_out);
}

int dnsb_maxdiv(dnsb_ctx *c, const double *ux, const double *uy, const double *uz, double *out) {
  if (!c || !ux || !uy || !uz || !out) return c ? fail(c, DNSB_EINVAL, "null argument") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  unsigned long long *scratch = c->umax + 3 * UMAX_SLOTS;
  CK(c, cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), c->stream));
  k_maxdiv<<<RED_BLOCKS, 256, 0, c->stream>>>(c->g, cf(ux, uy, uz), scratch);
  CKL(c);
  CK(c, cudaMemcpyAsync(c->hostred, scratch, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  *out = c->hostred[0];
  return 0;
}

int dnsb_kinetic_energy(dnsb_ctx *c, const double *ux, const double *uy, const double *uz, double *out) {
  if (!c || !ux || !uy || !uz || !out) return c ? fail(c, DNSB_EINVAL, "null argument") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  k_ke_partial<<<RED_BLOCKS, 256, 0, c->stream>>>(c->g, cf(ux, uy, uz), c->partial);
  CKL(c);
  k_sum_final<<<1, 1024, 0, c->stream>>>(c->partial, RED_BLOCKS, c->partial + RED_BLOCKS);
  CKL(c);
  CK(c, cudaMemcpyAsync(c->hostred, c->partial + RED_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  *out = c->hostred[0];
  return 0;
}

int dnsb_channel_sample(dnsb_ctx *c, const double *ux, const double *uy, const double *uz, double *acc) {
  if (!c || !ux || !uy || !uz || !acc) return c ? fail(c, DNSB_EINVAL, "null argument") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  const int nf = c->g.wall ? c->g.ny - 1 : c->g.ny;
  k_channel<<<c->g.ny + nf, 256, 0, c->stream>>>(c->g, cf(ux, uy, uz), acc, nf);
  CKL(c);
  return 0;
}

int dnsb_spectrum_sample(dnsb_ctx *c, const double *ux, const double *uy, const double *uz, double *E,
                         int nbins) {
  if (!c || !ux || !uy || !uz || !E || nbins < 1) return c ? fail(c, DNSB_EINVAL, "bad argument") : DNSB_EINVAL;
  if (c->g.wall) return fail(c, DNSB_EINVAL, "spectra require a fully periodic box");
  if (ensure_device(c)) return DNSB_ECUDA;
  const Geo &g = c->g;
  const double *u[3] = {ux, uy, uz};
  int rc;
  for (int comp = 0; comp < 3; comp++) {
    if ((rc = launch_rfftx(c, RIN_FIELD, u[comp], nullptr, nullptr))) return rc;
    if ((rc = launch_fftz(c, false))) return rc;
    dim3 grid(g.nkx * ((g.nz + c->Ly - 1) / c->Ly));
    k_yfourier<YF_FORWARD><<<grid, SPEC_THREADS, c->smem_y, c->stream>>>(g, c->S, c->py, c->Ly, c->twy,
                                                                  c->lam1, c->lam2, c->lam3);
    CKL(c);
    k_binshells<false><<<RED_BLOCKS, 256, 0, c->stream>>>(g, c->S, E, nbins);
    CKL(c);
  }
  return 0;
}

int dnsb_shell_count(const dnsb_ctx *c) { return c ? c->nshell_max : -1; }

int dnsb_shell_energies(dnsb_ctx *c, const double *ux, const double *uy, const double *uz, double *E,
                        int nshells) {
  int rc = check_shells(c, ux, uy, uz);
  if (rc) return rc;
  if (!E || nshells < 1) return fail(c, DNSB_EINVAL, "bad shell count");
  const int nb = std::min(nshells, c->nshell_max);
  const double *u[3] = {ux, uy, uz};
  if ((rc = shell_energies_dev(c, u, c->shellbuf, nb))) return rc;
  CK(c, cudaMemcpyAsync(E, c->shellbuf, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  for (int s = nb; s < nshells; s++) E[s] = 0;
  return 0;
}

int dnsb_shell_rescale(dnsb_ctx *c, double *ux, double *uy, double *uz, const double *factors,
                       int nshells) {
  int rc = check_shells(c, ux, uy, uz);
  if (rc) return rc;
  if (!factors || nshells < 1) return fail(c, DNSB_EINVAL, "bad shell count");
  const int nb = std::min(nshells, c->nshell_max);
  double *f = c->shellbuf + c->nshell_max;
  CK(c, cudaMemcpyAsync(f, factors, nb * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  double *u[3] = {ux, uy, uz};
  rc = shell_scale_dev(c, u, f, nb);
  if (rc) return rc;
  CK(c, cudaStreamSynchronize(c->stream));  // factors may be pageable host memory
  return 0;
}

int dnsb_random_field(dnsb_ctx *c, double *ux, double *uy, double *uz, double totalenergy,
                      double kpeak, unsigned long long seed, const double *profile, int nprofile) {
  int rc = check_shells(c, ux, uy, uz);
  if (rc) return rc;
  if (profile ? nprofile < 1 : !(kpeak > 0)) return fail(c, DNSB_EINVAL, "bad spectrum profile");
  const Geo &g = c->g;
  double *u[3] = {ux, uy, uz};
  for (int comp = 0; comp < 3; comp++) {
    k_gauss_noise<<<cell_grid(g), cell_block, 0, c->stream>>>(g, u[comp], comp, seed);
    CKL(c);
  }
  if ((rc = fill3(c, ux, uy, uz))) return rc;
  if ((rc = do_project(c, ux, uy, uz, c->implicit ? c->V[0] : c->W[0]))) return rc;
  const int nb = c->nshell_max;
  std::vector<double> E(nb), prof(nb), f(nb);
  if ((rc = dnsb_shell_energies(c, ux, uy, uz, E.data(), nb))) return rc;
  double tot = 0;
  for (int s = 0; s < nb; s++) {
    const double k = s;
    prof[s] = profile ? (s < nprofile ? profile[s] : 0.0) : k * k * k * k * exp(-2 * (k / kpeak) * (k / kpeak));
    tot += prof[s];
  }
  if (!(tot > 0)) return fail(c, DNSB_EINVAL, "spectrum profile sums to zero");
  for (int s = 0; s < nb; s++) {
    const double e0 = totalenergy * prof[s] / tot;
    f[s] = E[s] > 0 ? sqrt(e0 / E[s]) : 0.0;
  }
  return dnsb_shell_rescale(c, ux, uy, uz, f.data(), nb);
}

int dnsb_shell_clamp(dnsb_ctx *c, double *ux, double *uy, double *uz, const double *eref,
                     int nshells) {
  int rc = check_shells(c, ux, uy, uz);
  if (rc) return rc;
  if (!eref || nshells < 1) return fail(c, DNSB_EINVAL, "bad shell count");
  const int nb = std::min(nshells, c->nshell_max);
  double *E = c->shellbuf, *f = E + c->nshell_max, *er = f + c->nshell_max;
  if ((rc = upload_eref(c, eref, nb))) return rc;
  if (clamp_direct(c, nb)) {
    const Geo &g = c->g;
    const int KM = nb - 1;
    const unsigned lines = (unsigned)(((long long)g.ny * g.nz + LS_LINES - 1) / LS_LINES);
    k_ls_xsums<<<lines, 32 * LS_LINES, 0, c->stream>>>(g, cf(ux, uy, uz), KM, c->lsX, c->lsA);
    CKL(c);
    k_ls_ysums<<<(unsigned)(3 * (KM + 1) * g.nz), 128, 0, c->stream>>>(g, c->lsA, KM, c->lsY, c->lsB);
    CKL(c);
    k_ls_zsums<<<(unsigned)(3 * (KM + 1) * (2 * KM + 1)), 128, 0, c->stream>>>(g, c->lsB, KM, c->lsZ, c->lsG);
    CKL(c);
    k_ls_modes<<<1, 1024, 0, c->stream>>>(g, KM, c->lsG, c->lsH, E, er, f, nb, c->lsZ);
    CKL(c);
    k_ls_correct<<<lines, 32 * LS_LINES, 0, c->stream>>>(g, ff(ux, uy, uz), KM, c->lsH, c->lsX, c->lsY);
    CKL(c);
    c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
    return 0;
  }
  double *u[3] = {ux, uy, uz};
  return shell_clamp_dev(c, u, E, er, f, nb);
}

int dnsb_les_cube(dnsb_ctx *c, const double *ux, const double *uy, const double *uz, int M,
                  double *out) {
  int rc = check_shells(c, ux, uy, uz);
  if (rc) return rc;
  const Geo &g = c->g;
  if (!out || M < 2 || M % 2 || M / 2 > g.nx / 2 || M / 2 > g.ny / 2 || M / 2 > g.nz / 2)
    return fail(c, DNSB_EINVAL, "LES cube needs an even M with M/2 <= n/2 in every direction");
  const size_t per = (size_t)(M / 2 + 1) * M * M;
  if (c->cube_cap < 9 * per) {
    double2 *nb = nullptr;
    if ((rc = dalloc(c, &nb, 9 * per))) return rc;
    c->cube = nb;  // the previous, smaller buffer stays in the context's list until destroy
    c->cube_cap = 9 * per;
  }
  double *scr = c->implicit ? c->V[0] : c->W[0];
  const CFields3 u = cf(ux, uy, uz);
  static const int pa[9] = {0, 1, 2, 0, 1, 2, 0, 1, 2}, pb[9] = {-1, -1, -1, 0, 1, 2, 1, 2, 0};
  const double sc = 1.0 / ((double)g.nx * g.ny * g.nz);
  for (int f = 0; f < 9; f++) {
    k_cellprod<<<cell_grid(g), cell_block, 0, c->stream>>>(g, u, pa[f], pb[f], scr);
    CKL(c);
    if ((rc = spectrum_of(c, scr))) return rc;
    k_lescube<<<RED_BLOCKS, 256, 0, c->stream>>>(g, c->S, M, sc, c->cube + f * per);
    CKL(c);
  }
  CK(c, cudaMemcpyAsync(out, c->cube, 9 * per * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  return 0;
}

int dnsb_noise(dnsb_ctx *c, double *phi, int comp, unsigned long long seed, double amp) {
  if (!c || !phi || comp < 0 || comp > 2) return c ? fail(c, DNSB_EINVAL, "bad argument") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  k_noise<<<cell_grid(c->g), cell_block, 0, c->stream>>>(c->g, phi, comp, seed, amp);
  CKL(c);
  c->umax_for[0] = c->umax_for[1] = c->umax_for[2] = nullptr;
  return 0;
}

int dnsb_profile(dnsb_ctx *c, int enable) {
  if (!c) return DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  if (enable && c->evpool.empty()) {
    c->evpool.resize(4096);
    for (auto &e : c->evpool) CK(c, cudaEventCreate(&e));
  }
  int rc = prof_harvest(c);
  if (rc) return rc;
  for (int k = 0; k < DNSB_NKINDS; k++) { c->prof_ms[k] = 0; c->prof_n[k] = 0; }
  c->prof_on = enable != 0;
  return 0;
}

int dnsb_profile_read(dnsb_ctx *c, int kind, double *ms, long *launches) {
  if (!c || kind < 0 || kind >= DNSB_NKINDS) return c ? fail(c, DNSB_EINVAL, "bad kind") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  int rc = prof_harvest(c);
  if (rc) return rc;
  if (ms) *ms = c->prof_ms[kind];
  if (launches) *launches = c->prof_n[kind];
  return 0;
}

long dnsb_launch_count(const dnsb_ctx *c) { return c ? c->launches : -1; }

const char *dnsb_kind_name(int kind) {
  return (kind >= 0 && kind < DNSB_NKINDS) ? KIND_NAMES[kind] : "";
}

int dnsb_solve(dnsb_ctx *c, double *ux, double *uy, double *uz, double *p, double *qx, double *qy,
               double *qz, double *delta, double t0, double t1, double dt, double cfl,
               long max_steps, double *t_out, long *n_out) {
  if (!c || !ux || !uy || !uz || !p || !qx || !qy || !qz)
    return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (c->implicit && (!delta || delta == p))
    return fail(c, DNSB_EINVAL, "semi-implicit mode needs a separate delta field");
  if (ensure_device(c)) return DNSB_ECUDA;
  double *d = c->implicit ? delta : p;
  int rc;
  // solve! (src/timestep.jl:92-111): halo, projection, then the loop
  if ((rc = fill3(c, ux, uy, uz))) return rc;
  if ((rc = do_project(c, ux, uy, uz, d))) return rc;
  double t = t0;
  long n = 0;
  bool have_max = false;
  while (t < t1 - 1e-10 * (std::fabs(t1) + 1)) {
    if (max_steps >= 0 && n >= max_steps) break;
    double dtn = dt;
    if (!(dt > 0)) {
      if ((rc = dnsb_cfl(c, ux, uy, uz, cfl, have_max ? 1 : 0, &dtn))) return rc;
    }
    dtn = std::fmin(dtn, t1 - t);
    if ((rc = do_step(c, ux, uy, uz, p, qx, qy, qz, d, dtn))) return rc;
    have_max = true;
    t += dtn;
    n++;
  }
  CK(c, cudaStreamSynchronize(c->stream));
  if ((rc = check_deverr(c))) return rc;
  if (t_out) *t_out = t;
  if (n_out) *n_out = n;
  return 0;
}

int dnsb_solve_host(dnsb_ctx *c, double *ux, double *uy, double *uz, double *p, double t0, double t1,
                    double dt, double cfl, long max_steps, double *t_out, long *n_out) {
  if (!c || !ux || !uy || !uz) return c ? fail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  if (ensure_device(c)) return DNSB_ECUDA;
  const Geo &g = c->g;
  const size_t G = (size_t)g.NX * g.NY * g.NZ;
  const int nf = c->implicit ? 8 : 7;
  // the device fields persist in the context after the first call, so that
  // repeated calls neither map memory nor synchronise on an allocation
  if (!c->hostsolve) {
    int arc = dalloc(c, &c->hostsolve, nf * G);
    if (arc) return arc;
  }
  double *buf = c->hostsolve;
  double *f[8];
  for (int i = 0; i < nf; i++) f[i] = buf + i * G;
  int rc = 0;
  do {
    if (cudaMemsetAsync(buf, 0, nf * G * sizeof(double), c->stream) != cudaSuccess) { rc = fail(c, DNSB_ECUDA, "memset failed"); break; }
    double *hu[3] = {ux, uy, uz};
    for (int i = 0; i < 3 && !rc; i++)
      if (cudaMemcpyAsync(f[i], hu[i], G * sizeof(double), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        rc = fail(c, DNSB_ECUDA, "host to device copy failed");
    if (rc) break;
    rc = dnsb_solve(c, f[0], f[1], f[2], f[3], f[4], f[5], f[6], c->implicit ? f[7] : nullptr, t0, t1,
                    dt, cfl, max_steps, t_out, n_out);
    if (rc) break;
    for (int i = 0; i < 3 && !rc; i++)
      if (cudaMemcpyAsync(hu[i], f[i], G * sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
        rc = fail(c, DNSB_ECUDA, "device to host copy failed");
    if (!rc && p && cudaMemcpyAsync(p, f[3], G * sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
      rc = fail(c, DNSB_ECUDA, "device to host copy failed");
  } while (0);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (!rc && e != cudaSuccess) rc = fail(c, DNSB_ECUDA, "%s", cudaGetErrorString(e));
  return rc;
}

// ---------------------------------------------------------------- ensembles
// The last node of the ensemble's loop body: one step done; loop again
// while steps are left.
__global__ void k_ens_countdown(cudaGraphConditionalHandle cond, long long *left) {
  const long long n = --(*left);
  cudaGraphSetConditional(cond, n > 0 ? 1u : 0u);
}

// Members are ordinary contexts with their own streams.  One RK3 step of all
// members is captured from an internal origin stream (capture cannot start
// on the legacy default stream a caller may pass): fork event -> member
// streams -> join events; the executable graph is replayed on the origin
// stream, which is ordered after and before the caller's stream by events.

struct dnsb_ensemble {
  int n = 0, device = 0;
  cudaStream_t stream = nullptr;  // the caller's
  cudaStream_t origin = nullptr;
  std::vector<dnsb_ctx *> m;
  std::vector<cudaStream_t> ms;
  std::vector<cudaEvent_t> done;
  cudaEvent_t fork = nullptr, in = nullptr, out = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long *counter = nullptr;            // device: steps left in the while loop
  std::vector<double *> key_fields;
  std::vector<double> key_dts;
  std::vector<std::vector<double>> eref;  // per member: shell-clamp table (empty: no forcing)
  std::string err;
};

static int efail(dnsb_ensemble *e, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (e) e->err = buf;
  else snprintf(g_create_err, sizeof g_create_err, "%s", buf);
  return code;
}

static void ens_drop_graph(dnsb_ensemble *e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->exec = nullptr;
  e->graph = nullptr;
  e->key_fields.clear();
  e->key_dts.clear();
}

void dnsb_ensemble_destroy(dnsb_ensemble *e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->origin) cudaStreamSynchronize(e->origin);
  ens_drop_graph(e);
  for (dnsb_ctx *c : e->m) dnsb_destroy(c);
  for (cudaStream_t st : e->ms) cudaStreamDestroy(st);
  for (cudaEvent_t ev : e->done) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->in) cudaEventDestroy(e->in);
  if (e->out) cudaEventDestroy(e->out);
  if (e->counter) cudaFree(e->counter);
  if (e->origin) cudaStreamDestroy(e->origin);
  delete e;
}

int dnsb_ensemble_create(int n, const dnsb_grid *grids, int device, void *stream,
                         dnsb_ensemble **out) {
  return dnsb_ensemble_create_tuned(n, grids, nullptr, device, stream, out);
}

int dnsb_ensemble_create_tuned(int n, const dnsb_grid *grids, const dnsb_tuning *tunings,
                               int device, void *stream, dnsb_ensemble **out) {
  if (!out || !grids || n <= 0) return efail(nullptr, DNSB_EINVAL, "need n >= 1 grids and an output");
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess)
    return efail(nullptr, DNSB_ECUDA, "cudaSetDevice(%d) failed", device);
  dnsb_ensemble *e = new dnsb_ensemble();
  e->n = n;
  e->eref.resize(n);
  e->device = device;
  e->stream = (cudaStream_t)stream;
  auto bail = [&](int rc, const char *msg) {
    snprintf(g_create_err, sizeof g_create_err, "%.500s", msg);
    dnsb_ensemble_destroy(e);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&e->counter, sizeof(long long)) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->out, cudaEventDisableTiming) != cudaSuccess)
    return bail(DNSB_ECUDA, "stream or event creation failed");
  for (int i = 0; i < n; i++) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
      return bail(DNSB_ECUDA, "member stream creation failed");
    e->ms.push_back(st);
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
      return bail(DNSB_ECUDA, "member event creation failed");
    e->done.push_back(ev);
    dnsb_ctx *c = nullptr;
    const int rc = dnsb_create_tuned(&grids[i], tunings ? &tunings[i] : nullptr, device, st, &c);
    if (rc) {
      char msg[600];
      snprintf(msg, sizeof msg, "member %d: %.480s", i, g_create_err);
      return bail(rc, msg);
    }
    e->m.push_back(c);
  }
  *out = e;
  return 0;
}

const char *dnsb_ensemble_last_error(const dnsb_ensemble *e) { return e ? e->err.c_str() : g_create_err; }

dnsb_ctx *dnsb_ensemble_member(dnsb_ensemble *e, int i) {
  return (e && i >= 0 && i < e->n) ? e->m[i] : nullptr;
}

int dnsb_ensemble_forcing(dnsb_ensemble *e, int i, const double *eref, int nshells) {
  if (!e) return DNSB_EINVAL;
  if (i < 0 || i >= e->n) return efail(e, DNSB_EINVAL, "member %d out of range", i);
  if (cudaSetDevice(e->device) != cudaSuccess) return efail(e, DNSB_ECUDA, "cudaSetDevice failed");
  dnsb_ctx *c = e->m[i];
  std::vector<double> t;
  if (eref && nshells > 0) {
    if (c->g.wall) return efail(e, DNSB_EINVAL, "member %d: shell forcing needs a periodic box", i);
    t.assign(eref, eref + std::min(nshells, c->nshell_max));
    const int rc = upload_eref(c, t.data(), (int)t.size());
    if (rc) return efail(e, rc, "member %d: %s", i, dnsb_last_error(c));
  }
  if (t != e->eref[i]) {
    e->eref[i] = t;
    ens_drop_graph(e);
  }
  return 0;
}

int dnsb_ensemble_run(dnsb_ensemble *e, double *const *fields, const double *dts, long nsteps) {
  if (!e) return DNSB_EINVAL;
  if (!fields || !dts || nsteps < 0) return efail(e, DNSB_EINVAL, "null fields/dts or nsteps < 0");
  if (cudaSetDevice(e->device) != cudaSuccess) return efail(e, DNSB_ECUDA, "cudaSetDevice failed");
  const int n = e->n;
  std::vector<double *> f(fields, fields + 8 * (size_t)n);
  std::vector<double> d(dts, dts + n);
  for (int i = 0; i < n; i++) {
    if (!(d[i] > 0.0)) return efail(e, DNSB_EINVAL, "member %d: dt must be positive", i);
    for (int k = 0; k < 7; k++)
      if (!f[8 * i + k]) return efail(e, DNSB_EINVAL, "member %d: null field %d", i, k);
  }
  if (nsteps == 0) return 0;
  if (!e->exec || f != e->key_fields || d != e->key_dts) {
    ens_drop_graph(e);
    // The executable graph is [while (steps left) { one RK3 step of every
    // member (fork/join over the member streams, each followed by its
    // forcing); count down }]: one graph launch runs all nsteps steps.
    cudaGraph_t graph = nullptr;
    cudaGraphConditionalHandle cond;
    cudaGraphNode_t wnode;
    cudaGraphNodeParams wp = {};
    if (cudaGraphCreate(&graph, 0) != cudaSuccess)
      return efail(e, DNSB_ECUDA, "graph creation failed");
    e->graph = graph;
    // the loop condition starts at 1 on every launch: a launch runs >= 1 step
    if (cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
      ens_drop_graph(e);
      return efail(e, DNSB_ECUDA, "conditional handle creation failed");
    }
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = cond;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    if (cudaGraphAddNode(&wnode, graph, nullptr, 0, &wp) != cudaSuccess) {
      ens_drop_graph(e);
      return efail(e, DNSB_ECUDA, "conditional node creation failed");
    }
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(e->origin, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      ens_drop_graph(e);
      return efail(e, DNSB_ECUDA, "stream capture could not start");
    }
    int rc = 0;
    cudaEventRecord(e->fork, e->origin);
    for (int i = 0; i < n && !rc; i++) {
      cudaStreamWaitEvent(e->ms[i], e->fork, 0);
      double *const *fi = f.data() + 8 * (size_t)i;
      rc = dnsb_step(e->m[i], fi[0], fi[1], fi[2], fi[3], fi[4], fi[5], fi[6], fi[7], d[i]);
      if (rc) {
        efail(e, rc, "member %d: %s", i, dnsb_last_error(e->m[i]));
        break;
      }
      if (!e->eref[i].empty()) {
        rc = dnsb_shell_clamp(e->m[i], fi[0], fi[1], fi[2], e->eref[i].data(), (int)e->eref[i].size());
        if (rc) {
          efail(e, rc, "member %d forcing: %s", i, dnsb_last_error(e->m[i]));
          break;
        }
      }
      cudaEventRecord(e->done[i], e->ms[i]);
      cudaStreamWaitEvent(e->origin, e->done[i], 0);
    }
    if (!rc) k_ens_countdown<<<1, 1, 0, e->origin>>>(cond, e->counter);
    cudaGraph_t captured = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e->origin, &captured);
    if (rc) {
      ens_drop_graph(e);
      return rc;
    }
    if (ce != cudaSuccess) {
      ens_drop_graph(e);
      return efail(e, DNSB_ECUDA, "stream capture failed: %s", cudaGetErrorString(ce));
    }
    if (cudaGraphInstantiate(&e->exec, e->graph, 0) != cudaSuccess) {
      ens_drop_graph(e);
      return efail(e, DNSB_ECUDA, "graph instantiation failed");
    }
    e->key_fields = f;
    e->key_dts = d;
  }
  cudaEventRecord(e->in, e->stream);
  cudaStreamWaitEvent(e->origin, e->in, 0);
  // steps for the loop (the counter is read by the graph's countdown kernel)
  const long long steps = nsteps;
  if (cudaMemcpyAsync(e->counter, &steps, sizeof steps, cudaMemcpyHostToDevice, e->origin) != cudaSuccess)
    return efail(e, DNSB_ECUDA, "step count upload failed");
  if (cudaGraphLaunch(e->exec, e->origin) != cudaSuccess)
    return efail(e, DNSB_ECUDA, "graph launch failed");
  cudaEventRecord(e->out, e->origin);
  cudaStreamWaitEvent(e->stream, e->out, 0);
  // (a copy from pageable memory is staged before cudaMemcpyAsync returns)
  const cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess) return efail(e, DNSB_ECUDA, "%s", cudaGetErrorString(le));
  return 0;
}

}  // extern "C"

// ================================================ pseudo-spectral solver ==
//
// The reference's second solver (src/spectral/*.jl) on a periodic cube:
// state = the compact truncated spectrum (spsolver.cuh), transforms on a
// finite-volume context of the n^3 transform grid (its FFT plans and
// spectrum buffer), the nonlinear term in divergence form from the six
// velocity products (spectral_rhs!, operators.jl:66-96), Wray RK3 with the
// integrating-factor viscosity (spectral_step!, step.jl:60-92).
struct dnsb_spectral {
  dnsb_ctx *c = nullptr;
  SpGeo s{};
  double visc = 0, l = 0;
  double *v[3] = {nullptr, nullptr, nullptr};  // physical velocity, n^3 each (x fastest)
  double *r = nullptr;                         // one product, n^3
  double2 *ustart = nullptr, *du = nullptr;    // 3 x nc each
  double *partial = nullptr;                   // RED_BLOCKS + 1
  unsigned long long *umax = nullptr;          // 2 slots
  double *host = nullptr;                      // pinned, 4 doubles
  int nshell = 0;                              // floor(sqrt(3) kcut) + 1 shells
  double *shellbuf = nullptr;                  // [E | factors | eref] x nshell
  double *shellpart = nullptr;                 // RED_BLOCKS x SP_SHELLS partial sums
  std::vector<double> eref_host;
  std::vector<void *> allocs;
  std::string err;
};

namespace {

int spfail(dnsb_spectral *p, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (p) p->err = buf;
  else snprintf(g_create_err, sizeof g_create_err, "%s", buf);
  return code;
}

#define SPK(p, call)                                                                         \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) return spfail(p, DNSB_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)
#define SPKL(p) SPK(p, cudaGetLastError())
#define SPRC(p, expr)                                                     \
  do {                                                                    \
    int rc_ = (expr);                                                     \
    if (rc_) return spfail(p, rc_, "%s", dnsb_last_error((p)->c));        \
  } while (0)

template <class T>
int spalloc(dnsb_spectral *p, T **out, size_t n) {
  void *v = nullptr;
  if (cudaMalloc(&v, n * sizeof(T)) != cudaSuccess)
    return spfail(p, DNSB_ENOMEM, "cudaMalloc(%zu bytes) failed", n * sizeof(T));
  p->allocs.push_back(v);
  *out = (T *)v;
  return 0;
}

long long sp_n3(const dnsb_spectral *p) { return (long long)p->s.n * p->s.n * p->s.n; }

// spec_to_phys! of one component: v = sum over retained modes of u_hat e^{ikx}
int sp_to_phys(dnsb_spectral *p, const double2 *uhc, double *v) {
  dnsb_ctx *c = p->c;
  const Geo &g = c->g;
  const double n3 = (double)sp_n3(p);
  SPK(p, cudaMemsetAsync(c->S, 0, sizeof(double2) * (size_t)g.nkx * g.ny * g.nz, c->stream));
  k_sp_scatter<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, uhc, c->S, n3);
  SPKL(p);
  dim3 grid(c->nkx_active * ((g.nz + c->Ly - 1) / c->Ly));
  k_yfourier<YF_INVERSE><<<grid, SPEC_THREADS, c->smem_y, c->stream>>>(g, c->S, c->py, c->Ly, c->twy,
                                                                       c->lam1, c->lam2, c->lam3);
  SPKL(p);
  SPRC(p, launch_fftz(c, true));
  SPRC(p, launch_irfftx(c, ROUT_REAL, v));
  return 0;
}

// the full forward transform of a real n^3 array into S (unnormalised)
int sp_from_phys(dnsb_spectral *p, const double *r) {
  dnsb_ctx *c = p->c;
  const Geo &g = c->g;
  SPRC(p, launch_rfftx(c, RIN_REAL, r, nullptr, nullptr));
  SPRC(p, launch_fftz(c, false));
  dim3 grid(c->nkx_active * ((g.nz + c->Ly - 1) / c->Ly));
  k_yfourier<YF_FORWARD><<<grid, SPEC_THREADS, c->smem_y, c->stream>>>(g, c->S, c->py, c->Ly, c->twy,
                                                                       c->lam1, c->lam2, c->lam3);
  SPKL(p);
  return 0;
}

// the full forward transform of the product va * vb into S: fused into the
// x-transform's loads where the four-step kernel applies
int sp_from_product(dnsb_spectral *p, const double *va, const double *vb) {
  dnsb_ctx *c = p->c;
  const Geo &g = c->g;
  if (!c->x1) {
    k_sp_product<<<RED_BLOCKS, 256, 0, c->stream>>>(sp_n3(p), va, vb, p->r);
    SPKL(p);
    return sp_from_phys(p, p->r);
  }
  SPRC(p, launch_rfftx(c, RIN_PRODUCT, va, vb, nullptr));
  SPRC(p, launch_fftz(c, false));
  dim3 grid(c->nkx_active * ((g.nz + c->Ly - 1) / c->Ly));
  k_yfourier<YF_FORWARD><<<grid, SPEC_THREADS, c->smem_y, c->stream>>>(g, c->S, c->py, c->Ly, c->twy,
                                                                       c->lam1, c->lam2, c->lam3);
  SPKL(p);
  return 0;
}

// spectral_rhs!: du = -i k_j F[v_i v_j] / n^3; leaves v = the physical velocity
int sp_rhs(dnsb_spectral *p, const double2 *uh, double2 *du) {
  dnsb_ctx *c = p->c;
  const long long n3 = sp_n3(p);
  int rc;
  for (int comp = 0; comp < 3; comp++)
    if ((rc = sp_to_phys(p, uh + comp * p->s.nc, p->v[comp]))) return rc;
  static const int pa[6] = {0, 1, 2, 0, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 0};
  for (int f = 0; f < 6; f++) {
    if ((rc = sp_from_product(p, p->v[pa[f]], p->v[pb[f]]))) return rc;
    k_sp_div<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, c->S, du, pa[f], pb[f], 1.0 / (double)n3);
    SPKL(p);
  }
  return 0;
}

// E[0..nb) (device) = shell energies in a fixed summation order
int sp_shell_energies_dev(dnsb_spectral *p, const double2 *uh, double *E, int nb) {
  cudaStream_t st = p->c->stream;
  if (nb <= SP_SHELLS) {
    k_sp_shells_det<<<RED_BLOCKS, 256, 0, st>>>(p->s, uh, p->shellpart);
    SPKL(p);
    k_sp_shells_fold<<<1, 32, 0, st>>>(p->shellpart, RED_BLOCKS, nb, E);
  } else {
    k_sp_shells_byshell<<<nb, 256, 0, st>>>(p->s, uh, E);
  }
  SPKL(p);
  return 0;
}

int sp_upload_eref(dnsb_spectral *p, const double *eref, int nb) {
  if (p->eref_host.size() == (size_t)nb && std::equal(eref, eref + nb, p->eref_host.begin())) return 0;
  SPK(p, cudaMemcpyAsync(p->shellbuf + 2 * p->nshell, eref, nb * sizeof(double),
                         cudaMemcpyHostToDevice, p->c->stream));
  SPK(p, cudaStreamSynchronize(p->c->stream));
  p->eref_host.assign(eref, eref + nb);
  return 0;
}

int sp_check(dnsb_spectral *p, const void *a) {
  if (!p) return DNSB_EINVAL;
  if (!a) return spfail(p, DNSB_EINVAL, "null array");
  if (cudaSetDevice(p->c->device) != cudaSuccess) return spfail(p, DNSB_ECUDA, "cudaSetDevice failed");
  return 0;
}

}  // namespace

extern "C" {

int dnsb_spectral_create(int n, int kcut, double l, double visc, int device, void *stream,
                         dnsb_spectral **out) {
  if (!out) return spfail(nullptr, DNSB_EINVAL, "null output");
  *out = nullptr;
  if (n < 4 || n % 2) return spfail(nullptr, DNSB_EINVAL, "n must be even");
  if (kcut <= 0) kcut = n / 3;
  if (3 * kcut > n) return spfail(nullptr, DNSB_EINVAL, "aliasing: 3kcut <= n is required (2/3 rule)");
  if (!(l > 0) || !(visc >= 0)) return spfail(nullptr, DNSB_EINVAL, "bad l or visc");
  std::vector<double> dy(n + 2, l / n);
  dnsb_grid gr{};
  gr.nx = gr.ny = gr.nz = n;
  gr.bc_y = DNSB_BC_PERIODIC;
  gr.ydiffusion = DNSB_YDIFF_EXPLICIT;
  gr.dx = gr.dz = l / n;
  gr.dy = dy.data();
  gr.dyu = dy.data();
  gr.visc = visc;
  dnsb_ctx *c = nullptr;
  int rc = dnsb_create(&gr, device, stream, &c);
  if (rc) return rc;  // message in dnsb_last_error(NULL)
  dnsb_spectral *p = new dnsb_spectral();
  p->c = c;
  // only the planes kx <= kcut carry retained modes: the z- and y-transforms
  // between the x-transform and the state skip the others (zero after the
  // scatter, never gathered)
  c->nkx_active = kcut + 1;
  p->visc = visc;
  p->l = l;
  p->s.n = n;
  p->s.kcut = kcut;
  p->s.m = 2 * kcut + 1;
  p->s.nc = (long long)(kcut + 1) * p->s.m * p->s.m;
  p->s.kfac = 2 * M_PI / l;
  const size_t n3 = (size_t)n * n * n;
  if ((rc = spalloc(p, &p->v[0], n3)) || (rc = spalloc(p, &p->v[1], n3)) ||
      (rc = spalloc(p, &p->v[2], n3)) || (rc = spalloc(p, &p->r, n3)) ||
      (rc = spalloc(p, &p->ustart, 3 * (size_t)p->s.nc)) ||
      (rc = spalloc(p, &p->du, 3 * (size_t)p->s.nc)) ||
      (rc = spalloc(p, &p->partial, (size_t)RED_BLOCKS + 1)) || (rc = spalloc(p, &p->umax, 2)) ||
      (rc = spalloc(p, &p->shellbuf, 3 * (size_t)(p->nshell = (int)std::floor(std::sqrt(3.0) * kcut) + 1))) ||
      (rc = spalloc(p, &p->shellpart, (size_t)RED_BLOCKS * SP_SHELLS))) {
    snprintf(g_create_err, sizeof g_create_err, "%s", p->err.c_str());
    dnsb_spectral_destroy(p);
    return rc;
  }
  if (cudaMallocHost(&p->host, 4 * sizeof(double)) != cudaSuccess) {
    snprintf(g_create_err, sizeof g_create_err, "cudaMallocHost failed");
    dnsb_spectral_destroy(p);
    return DNSB_ENOMEM;
  }
  *out = p;
  return 0;
}

void dnsb_spectral_destroy(dnsb_spectral *p) {
  if (!p) return;
  if (p->c) cudaSetDevice(p->c->device);
  for (void *a : p->allocs) cudaFree(a);
  if (p->host) cudaFreeHost(p->host);
  dnsb_destroy(p->c);
  delete p;
}

const char *dnsb_spectral_last_error(const dnsb_spectral *p) { return p ? p->err.c_str() : g_create_err; }

long dnsb_spectral_size(const dnsb_spectral *p) { return p ? (long)p->s.nc : -1; }

int dnsb_spectral_to_phys(dnsb_spectral *p, const double *uh, double *v) {
  int rc = sp_check(p, uh);
  if (rc || (rc = sp_check(p, v))) return rc;
  const long long n3 = sp_n3(p);
  for (int comp = 0; comp < 3; comp++)
    if ((rc = sp_to_phys(p, reinterpret_cast<const double2 *>(uh) + comp * p->s.nc, v + comp * n3)))
      return rc;
  return 0;
}

int dnsb_spectral_from_phys(dnsb_spectral *p, const double *v, double *uh) {
  int rc = sp_check(p, uh);
  if (rc || (rc = sp_check(p, v))) return rc;
  const long long n3 = sp_n3(p);
  dnsb_ctx *c = p->c;
  double2 *u2 = reinterpret_cast<double2 *>(uh);
  for (int comp = 0; comp < 3; comp++) {
    if ((rc = sp_from_phys(p, v + comp * n3))) return rc;
    k_sp_gather<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, c->S, u2 + comp * p->s.nc, 1.0 / (double)n3);
    SPKL(p);
  }
  return 0;
}

int dnsb_spectral_rhs(dnsb_spectral *p, const double *uh, double *du) {
  int rc = sp_check(p, uh);
  if (rc || (rc = sp_check(p, du))) return rc;
  return sp_rhs(p, reinterpret_cast<const double2 *>(uh), reinterpret_cast<double2 *>(du));
}

int dnsb_spectral_project(dnsb_spectral *p, double *uh) {
  int rc = sp_check(p, uh);
  if (rc) return rc;
  k_sp_project<<<RED_BLOCKS, 256, 0, p->c->stream>>>(p->s, reinterpret_cast<double2 *>(uh));
  SPKL(p);
  return 0;
}

int dnsb_spectral_step(dnsb_spectral *p, double *uh, double dt, double *vmax_out) {
  int rc = sp_check(p, uh);
  if (rc) return rc;
  if (!(dt > 0)) return spfail(p, DNSB_EINVAL, "dt must be positive");
  dnsb_ctx *c = p->c;
  double2 *u2 = reinterpret_cast<double2 *>(uh);
  static const double A[3] = {8.0 / 15, 5.0 / 12, 3.0 / 4}, B[3] = {1.0 / 4, 0.0, 0.0},
                      DC[3] = {8.0 / 15, 2.0 / 15, 1.0 / 3};
  SPK(p, cudaMemcpyAsync(p->ustart, u2, sizeof(double2) * 3 * (size_t)p->s.nc,
                         cudaMemcpyDeviceToDevice, c->stream));
  SPK(p, cudaMemsetAsync(p->umax, 0, sizeof(unsigned long long), c->stream));
  for (int i = 0; i < 3; i++) {
    if ((rc = sp_rhs(p, u2, p->du))) return rc;
    if (i == 0) {
      k_sp_vsummax<<<RED_BLOCKS, 256, 0, c->stream>>>(sp_n3(p), p->v[0], p->v[1], p->v[2], p->umax);
      SPKL(p);
    }
    k_sp_ifstage<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, u2, p->ustart, p->du, A[i], B[i],
                                                     p->visc * DC[i] * dt, dt);
    SPKL(p);
    k_sp_project<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, u2);
    SPKL(p);
  }
  if (vmax_out) {
    SPK(p, cudaMemcpyAsync(p->host, p->umax, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    SPK(p, cudaStreamSynchronize(c->stream));
    *vmax_out = p->host[0];
  }
  return 0;
}

int dnsb_spectral_vsummax(dnsb_spectral *p, const double *uh, double *out) {
  int rc = sp_check(p, uh);
  if (rc || (rc = sp_check(p, out))) return rc;
  dnsb_ctx *c = p->c;
  for (int comp = 0; comp < 3; comp++)
    if ((rc = sp_to_phys(p, reinterpret_cast<const double2 *>(uh) + comp * p->s.nc, p->v[comp])))
      return rc;
  SPK(p, cudaMemsetAsync(p->umax, 0, sizeof(unsigned long long), c->stream));
  k_sp_vsummax<<<RED_BLOCKS, 256, 0, c->stream>>>(sp_n3(p), p->v[0], p->v[1], p->v[2], p->umax);
  SPKL(p);
  SPK(p, cudaMemcpyAsync(p->host, p->umax, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SPK(p, cudaStreamSynchronize(c->stream));
  *out = p->host[0];
  return 0;
}

// which: 0 = spectral_energy, 1 = spectral_dissipation, 2 = spectral_maxdiv
int dnsb_spectral_diagnostic(dnsb_spectral *p, const double *uh, int which, double *out) {
  int rc = sp_check(p, uh);
  if (rc || (rc = sp_check(p, out))) return rc;
  if (which < 0 || which > 2) return spfail(p, DNSB_EINVAL, "bad diagnostic");
  dnsb_ctx *c = p->c;
  const double2 *u2 = reinterpret_cast<const double2 *>(uh);
  if (which == 2) {
    SPK(p, cudaMemsetAsync(p->umax + 1, 0, sizeof(unsigned long long), c->stream));
    k_sp_maxdiv<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, u2, p->umax + 1);
    SPKL(p);
    SPK(p, cudaMemcpyAsync(p->host, p->umax + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  } else {
    k_sp_sum<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, u2, which, p->partial);
    SPKL(p);
    k_sum_final<<<1, 1024, 0, c->stream>>>(p->partial, RED_BLOCKS, p->partial + RED_BLOCKS);
    SPKL(p);
    SPK(p, cudaMemcpyAsync(p->host, p->partial + RED_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
  }
  SPK(p, cudaStreamSynchronize(c->stream));
  *out = which == 1 ? p->visc * p->host[0] : p->host[0];
  return 0;
}

int dnsb_spectral_shell_count(const dnsb_spectral *p) { return p ? p->nshell : -1; }

int dnsb_spectral_shell_energies(dnsb_spectral *p, const double *uh, double *E, int nshells) {
  int rc = sp_check(p, uh);
  if (rc || (rc = sp_check(p, E))) return rc;
  if (nshells < 1) return spfail(p, DNSB_EINVAL, "bad shell count");
  const int nb = std::min(nshells, p->nshell);
  if ((rc = sp_shell_energies_dev(p, reinterpret_cast<const double2 *>(uh), p->shellbuf, nb))) return rc;
  SPK(p, cudaMemcpyAsync(E, p->shellbuf, nb * sizeof(double), cudaMemcpyDeviceToHost, p->c->stream));
  SPK(p, cudaStreamSynchronize(p->c->stream));
  for (int i = nb; i < nshells; i++) E[i] = 0;
  return 0;
}

int dnsb_spectral_shell_rescale(dnsb_spectral *p, double *uh, const double *factors, int nshells) {
  int rc = sp_check(p, uh);
  if (rc || (rc = sp_check(p, factors))) return rc;
  if (nshells < 1) return spfail(p, DNSB_EINVAL, "bad shell count");
  const int nb = std::min(nshells, p->nshell);
  double *f = p->shellbuf + p->nshell;
  SPK(p, cudaMemcpyAsync(f, factors, nb * sizeof(double), cudaMemcpyHostToDevice, p->c->stream));
  k_sp_scale_shells<<<RED_BLOCKS, 256, 0, p->c->stream>>>(p->s, reinterpret_cast<double2 *>(uh), f, nb);
  SPKL(p);
  SPK(p, cudaStreamSynchronize(p->c->stream));
  return 0;
}

int dnsb_spectral_random_field(dnsb_spectral *p, double *uh, double totalenergy, double kpeak,
                               unsigned long long seed, const double *profile, int nprofile) {
  int rc = sp_check(p, uh);
  if (rc) return rc;
  if (profile ? nprofile < 1 : !(kpeak > 0)) return spfail(p, DNSB_EINVAL, "bad spectrum profile");
  dnsb_ctx *c = p->c;
  double2 *u2 = reinterpret_cast<double2 *>(uh);
  const double n3 = (double)sp_n3(p);
  for (int comp = 0; comp < 3; comp++) {
    k_sp_noise<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s.n, p->v[comp], comp, seed);
    SPKL(p);
    if ((rc = sp_from_phys(p, p->v[comp]))) return rc;
    k_sp_gather<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, c->S, u2 + comp * p->s.nc, 1.0 / n3);
    SPKL(p);
  }
  k_sp_project<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, u2);
  SPKL(p);
  const int nb = p->nshell;
  std::vector<double> E(nb), f(nb), prof(nb);
  if ((rc = dnsb_spectral_shell_energies(p, uh, E.data(), nb))) return rc;
  double tot = 0;
  for (int i = 0; i < nb; i++) {
    const double k = i;
    prof[i] = profile ? (i < nprofile ? profile[i] : 0.0) : k * k * k * k * exp(-2 * (k / kpeak) * (k / kpeak));
    tot += prof[i];
  }
  if (!(tot > 0)) return spfail(p, DNSB_EINVAL, "spectrum profile sums to zero");
  for (int i = 0; i < nb; i++) {
    const double e0 = totalenergy * prof[i] / tot;
    f[i] = E[i] > 0 ? sqrt(e0 / E[i]) : 0.0;
  }
  return dnsb_spectral_shell_rescale(p, uh, f.data(), nb);
}

int dnsb_spectral_shell_clamp(dnsb_spectral *p, double *uh, const double *eref, int nshells) {
  int rc = sp_check(p, uh);
  if (rc || (rc = sp_check(p, eref))) return rc;
  if (nshells < 1) return spfail(p, DNSB_EINVAL, "bad shell count");
  const int nb = std::min(nshells, p->nshell);
  if ((rc = sp_upload_eref(p, eref, nb))) return rc;
  double *E = p->shellbuf, *f = E + p->nshell, *er = f + p->nshell;
  double2 *u2 = reinterpret_cast<double2 *>(uh);
  if ((rc = sp_shell_energies_dev(p, u2, E, nb))) return rc;
  k_sp_clamp_factors<<<1, 256, 0, p->c->stream>>>(E, er, f, nb);
  SPKL(p);
  k_sp_scale_shells<<<RED_BLOCKS, 256, 0, p->c->stream>>>(p->s, u2, f, nb);
  SPKL(p);
  return 0;
}

int dnsb_spectral_les_cube(dnsb_spectral *p, const double *uh, int M, double *out) {
  int rc = sp_check(p, uh);
  if (rc || (rc = sp_check(p, out))) return rc;
  if (M < 2 || M % 2 || M / 2 > p->s.kcut)
    return spfail(p, DNSB_EINVAL, "LES cube needs an even M with M/2 <= kcut");
  dnsb_ctx *c = p->c;
  const size_t per = (size_t)(M / 2 + 1) * M * M;
  if (c->cube_cap < 9 * per) {
    double2 *nb = nullptr;
    if ((rc = dalloc(c, &nb, 9 * per))) return spfail(p, rc, "%s", dnsb_last_error(c));
    c->cube = nb;
    c->cube_cap = 9 * per;
  }
  const double2 *u2 = reinterpret_cast<const double2 *>(uh);
  const long long n3 = sp_n3(p);
  for (int comp = 0; comp < 3; comp++) {
    k_sp_cube<<<RED_BLOCKS, 256, 0, c->stream>>>(p->s, u2 + comp * p->s.nc, M, c->cube + comp * per);
    SPKL(p);
    if ((rc = sp_to_phys(p, u2 + comp * p->s.nc, p->v[comp]))) return rc;
  }
  static const int pa[6] = {0, 1, 2, 0, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 0};
  for (int f = 0; f < 6; f++) {
    if ((rc = sp_from_product(p, p->v[pa[f]], p->v[pb[f]]))) return rc;
    k_lescube<<<RED_BLOCKS, 256, 0, c->stream>>>(c->g, c->S, M, 1.0 / (double)n3, c->cube + (3 + f) * per);
    SPKL(p);
  }
  SPK(p, cudaMemcpyAsync(out, c->cube, 9 * per * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  SPK(p, cudaStreamSynchronize(c->stream));
  return 0;
}

int dnsb_spectral_phaserandomize(dnsb_spectral *p, double *uh, unsigned long long seed) {
  int rc = sp_check(p, uh);
  if (rc) return rc;
  k_sp_phaserand<<<RED_BLOCKS, 256, 0, p->c->stream>>>(p->s, reinterpret_cast<double2 *>(uh), seed);
  SPKL(p);
  return 0;
}

int dnsb_spectral_set_stream(dnsb_spectral *p, void *stream) {
  if (!p) return DNSB_EINVAL;
  return dnsb_set_stream(p->c, stream);
}

}  // extern "C"

// ====================================================== allocation-free ==
//
// dnsb_poisson_noalloc: the Poisson solve of dnsb_poisson for callers that
// cannot allocate device memory.  Typical such callers hand all device
// memory to a pooling allocator with a hard cap (CUDA.jl's memory pool, a
// framework caching allocator), so a foreign cudaMalloc can fail or force a
// pool flush, or run timed loops in which the implicit device-wide
// synchronisation of cudaMalloc/cudaFree is not acceptable.  They cannot
// create a dnsb_ctx either (dnsb_create allocates), so this entry point
// needs none: the spectrum, the y-solve work array and every coefficient
// and twiddle table live in one file-scope device array of fixed size
// (kNoAllocBytes, held by every GPU that loads the library until exit).
// Inputs and outputs are still the caller's device arrays.
namespace {

constexpr long long kNoAllocMaxSpec = 1LL << 20;  // (nx/2+1)*ny*nz complex values
constexpr int kNoAllocMaxN = 4096;                // nx, ny, nz
// layout in doubles: S (2*spec) | work (spec) | dy dyu rdy rdyu (4*(N+2)) |
// lam1 lam2 lam3 ay by cy (6*N) | twM twN twz twy (2*(N/2 + N/2+1 + N + N))
constexpr long long kNoAllocDoubles = 3 * kNoAllocMaxSpec + 4LL * (kNoAllocMaxN + 2) +
                                      6LL * kNoAllocMaxN + 2LL * (3 * kNoAllocMaxN + 1);
constexpr long long kNoAllocBytes = kNoAllocDoubles * (long long)sizeof(double);
static_assert(kNoAllocBytes < (28LL << 20), "the fixed scratch stays modest (about 26 MB)");

__device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Host staging for the tables and, per device, the grid whose tables the
// device copy holds (static: the entry point allocates nothing, host or
// device).  g_noalloc_mu serialises the set-up and the table uploads of
// all host threads; the kernels are enqueued outside it.
double h_tab[4 * (kNoAllocMaxN + 2) + 6 * kNoAllocMaxN];
double2 h_tw[3 * kNoAllocMaxN + 1];

constexpr int kMaxDevices = 64;
struct NoAllocDev {
  void *ptr;        // device address of g_noalloc_scratch (attributes set for it)
  bool have_grid;   // the device tables hold the grid below
  int nx, ny, nz, bc;
  double dx, dz;
  double dy[kNoAllocMaxN + 2], dyu[kNoAllocMaxN + 2];
};
NoAllocDev g_noalloc_dev[kMaxDevices];
std::mutex g_noalloc_mu;

// With g_noalloc_mu held and device dev current: the device address of the
// scratch array (in host code the symbol is only a stand-in), resolved on
// every call so that a reset device gets its new address, and the
// shared-memory limits of the kernels used, set again when it changes.
int noalloc_setup(int dev, double **out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(nullptr, DNSB_EUNSUP, "device index %d out of range", dev);
  void *ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !ptr)
    return fail(nullptr, DNSB_ECUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
  NoAllocDev &d = g_noalloc_dev[dev];
  if (d.ptr != ptr) {
    const int big = 200 * 1024;
    cudaError_t a = cudaSuccess;
    a = a != cudaSuccess ? a : raise_smem(dev, k_rfftx<RIN_REAL>, big);
    a = a != cudaSuccess ? a : raise_smem(dev, k_fftz<false>, big);
    a = a != cudaSuccess ? a : raise_smem(dev, k_fftz<true>, big);
    a = a != cudaSuccess ? a : raise_smem(dev, k_yfourier<YF_SOLVE>, big);
    a = a != cudaSuccess ? a : raise_smem(dev, k_irfftx<ROUT_INTERIOR>, big);
    if (a != cudaSuccess)
      return fail(nullptr, DNSB_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(a));
    d.ptr = ptr;
    d.have_grid = false;  // a new address: the tables must be uploaded again
  }
  *out = (double *)ptr;
  return 0;
}

// Does the device copy of the tables already describe this grid?
bool noalloc_same_grid(const NoAllocDev &d, const dnsb_grid *gr) {
  if (!d.have_grid || d.nx != gr->nx || d.ny != gr->ny || d.nz != gr->nz || d.bc != gr->bc_y ||
      d.dx != gr->dx || d.dz != gr->dz)
    return false;
  return std::memcmp(d.dy, gr->dy, sizeof(double) * (gr->ny + 2)) == 0 &&
         std::memcmp(d.dyu, gr->dyu, sizeof(double) * (gr->ny + 2)) == 0;
}

}  // namespace

extern "C" int dnsb_poisson_noalloc(const dnsb_grid *gr, const double *r, double *p, void *stream) {
  if (!gr || !r || !p) return fail(nullptr, DNSB_EINVAL, "null argument");
  const int nx = gr->nx, ny = gr->ny, nz = gr->nz;
  if (nx < 2 || ny < 2 || nz < 1 || nx % 2)
    return fail(nullptr, DNSB_EINVAL, "need nx >= 2 even, ny >= 2, nz >= 1 (got %d %d %d)", nx, ny, nz);
  if (gr->bc_y != DNSB_BC_PERIODIC && gr->bc_y != DNSB_BC_WALL)
    return fail(nullptr, DNSB_EINVAL, "bc[2] must be :periodic or :wall");
  if (!gr->dy || !gr->dyu) return fail(nullptr, DNSB_EINVAL, "dy/dyu missing");
  const int M = nx / 2;
  const long long spec = (long long)(M + 1) * ny * nz;
  if (nx > kNoAllocMaxN || ny > kNoAllocMaxN || nz > kNoAllocMaxN || spec > kNoAllocMaxSpec)
    return fail(nullptr, DNSB_EUNSUP,
                "dnsb_poisson_noalloc: grid %dx%dx%d exceeds its fixed scratch "
                "((nx/2+1)*ny*nz <= %lld, nx, ny, nz <= %d)", nx, ny, nz, kNoAllocMaxSpec, kNoAllocMaxN);
  FFTPlan pM{}, pz{}, py{};
  const bool wall = gr->bc_y == DNSB_BC_WALL;
  if (!make_fft_plan(M, pM) || !make_fft_plan(nz, pz) || (!wall && !make_fft_plan(ny, py)))
    return fail(nullptr, DNSB_EUNSUP, "FFT lengths nx/2=%d, nz=%d%s must factor into 2, 3, 5", M, nz,
                wall ? "" : ", ny");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(nullptr, DNSB_ECUDA, "cudaGetDevice failed");
  double *base = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  double *tabs = nullptr;
  double2 *tws = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    int rc = noalloc_setup(dev, &base);
    if (rc) return rc;
    tabs = base + 3 * kNoAllocMaxSpec;  // after S (2*spec) and work (spec): 4*(N+2) + 6*N doubles
    tws = reinterpret_cast<double2 *>(tabs + 4 * (kNoAllocMaxN + 2) + 6 * kNoAllocMaxN);
    NoAllocDev &d = g_noalloc_dev[dev];
    if (!noalloc_same_grid(d, gr)) {
      // tables, computed exactly as in dnsb_create (plan_poisson, griddata)
      double *dy = h_tab, *dyu = dy + (ny + 2), *rdy = dyu + (ny + 2), *rdyu = rdy + (ny + 2);
      double *lam1 = rdyu + (ny + 2), *lam2 = lam1 + (M + 1), *lam3 = lam2 + ny;
      double *ay = lam3 + nz, *by = ay + ny, *cy = by + ny;
      const long long ntab = (cy + ny) - h_tab;
      for (int J = 0; J < ny + 2; J++) {
        dy[J] = gr->dy[J];
        dyu[J] = gr->dyu[J];
        rdy[J] = 1.0 / dy[J];
        rdyu[J] = 1.0 / dyu[J];
      }
      for (int k = 1; k <= M + 1; k++) lam1[k - 1] = modlam(k, nx, gr->dx);
      for (int k = 1; k <= nz; k++) lam3[k - 1] = modlam(k, nz, gr->dz);
      for (int k = 1; k <= ny; k++) lam2[k - 1] = modlam(k, ny, dy[1]);
      for (int j = 1; j <= ny; j++) {
        double a = 0.0, cc = 0.0;
        if (wall) {
          a = j == 1 ? 0.0 : 1 / (dy[j] * dyu[j - 1]);
          cc = j == ny ? 0.0 : 1 / (dy[j] * dyu[j]);
        }
        ay[j - 1] = a;
        cy[j - 1] = cc;
        by[j - 1] = -(a + cc);
      }
      double2 *twM = h_tw, *twN = twM + M, *twz = twN + (M + 1), *twy = twz + nz;
      const long long ntw = (twy + ny) - h_tw;
      for (int t = 0; t < M; t++) twM[t] = unit_root(t, M);
      for (int t = 0; t <= M; t++) twN[t] = unit_root(t, nx);
      for (int t = 0; t < nz; t++) twz[t] = unit_root(t, nz);
      for (int t = 0; t < ny; t++) twy[t] = unit_root(t, ny);
      d.have_grid = false;
      cudaError_t e = cudaMemcpyAsync(tabs, h_tab, ntab * sizeof(double), cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(tws, h_tw, ntw * sizeof(double2), cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return fail(nullptr, DNSB_ECUDA, "table upload: %s", cudaGetErrorString(e));
      // the static host staging is reused by the next upload: wait for the copies
      if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
        return fail(nullptr, DNSB_ECUDA, "%s", cudaGetErrorString(e));
      d.nx = nx; d.ny = ny; d.nz = nz; d.bc = gr->bc_y;
      d.dx = gr->dx; d.dz = gr->dz;
      std::memcpy(d.dy, gr->dy, sizeof(double) * (ny + 2));
      std::memcpy(d.dyu, gr->dyu, sizeof(double) * (ny + 2));
      d.have_grid = true;
    }
  }
  // carve the scratch array
  double2 *S = reinterpret_cast<double2 *>(base);
  double *work = base + 2 * kNoAllocMaxSpec;
  cudaError_t e = cudaSuccess;

  Geo g{};
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.NX = nx + 2; g.NY = ny + 2; g.NZ = nz + 2;
  g.wall = wall;
  g.jymax = wall ? ny - 1 : ny;
  g.nkx = M + 1;
  g.dx = gr->dx; g.dz = gr->dz;
  g.rdx = 1.0 / g.dx; g.rdz = 1.0 / g.dz;
  g.rdx2 = 1.0 / (g.dx * g.dx); g.rdz2 = 1.0 / (g.dz * g.dz);
  g.visc = gr->visc;
  g.dy = tabs;
  g.dyu = tabs + (ny + 2);
  g.rdy = tabs + 2 * (ny + 2);
  g.rdyu = tabs + 3 * (ny + 2);
  const double *d_lam1 = tabs + 4 * (ny + 2), *d_lam2 = d_lam1 + (M + 1), *d_lam3 = d_lam2 + ny;
  const double *d_ay = d_lam3 + nz, *d_by = d_ay + ny, *d_cy = d_by + ny;
  const double2 *d_twM = tws, *d_twN = d_twM + M, *d_twz = d_twN + (M + 1), *d_twy = d_twz + nz;

  // launch shapes as chosen by dnsb_create
  auto pow2floor = [](int v) { int q = 1; while (2 * q <= v) q *= 2; return q; };
  const int budget = 100 * 1024 / (2 * (int)sizeof(double2));
  const int Lx = pow2floor(std::max(1, std::min({8, nz, budget / (M + 2)})));
  const int Lz = std::max(1, std::min(4, budget / (nz + 1)));
  const int Ly = pow2floor(std::max(1, std::min({8, nz, budget / ny})));
  const size_t smem_rx = sizeof(double2) * (2 * (size_t)Lx * (M + 1) + M + (M + 1));
  const size_t smem_ix = sizeof(double2) * (2 * (size_t)Lx * (M + 2) + M + (M + 1));
  const size_t smem_z = sizeof(double2) * (2 * (size_t)Lz * (nz + 1) + nz);
  const size_t smem_y = sizeof(double2) * (2 * (size_t)Ly * ny + ny);
  const long long nlines = (long long)ny * g.nkx;
  const dim3 gx(ny * ((nz + Lx - 1) / Lx)), gz((unsigned)((nlines + Lz - 1) / Lz));
  k_rfftx<RIN_REAL><<<gx, SPEC_THREADS, smem_rx, st>>>(g, S, r, nullptr, nullptr, pM, Lx, d_twM, d_twN);
  k_fftz<false><<<gz, SPEC_THREADS, smem_z, st>>>(g, S, pz, Lz, d_twz);
  if (wall) {
    const long long nl = (long long)g.nkx * nz;
    k_thomas<<<(unsigned)((nl + 127) / 128), 128, 0, st>>>(g, S, work, d_ay, d_by, d_cy, d_lam1, d_lam3);
  } else {
    k_yfourier<YF_SOLVE><<<dim3(g.nkx * ((nz + Ly - 1) / Ly)), SPEC_THREADS, smem_y, st>>>(
        g, S, py, Ly, d_twy, d_lam1, d_lam2, d_lam3);
  }
  k_fftz<true><<<gz, SPEC_THREADS, smem_z, st>>>(g, S, pz, Lz, d_twz);
  k_irfftx<ROUT_INTERIOR><<<gx, SPEC_THREADS, smem_ix, st>>>(g, S, p, pM, Lx, d_twM, d_twN);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return fail(nullptr, DNSB_ECUDA, "launch: %s", cudaGetErrorString(e));
  return 0;
}
