// cnn.cu -- the sub-filter-stress CNN closure: context, TMA tensor maps,
// the small kernels around the tensor-core convolutions (crops, packing,
// Adam, split-K reduction, loss) and the C ABI of include/dnsb_cnn.h.
//
// No counterpart in the reference (DistributedNavierStokes has no learned
// closure); its training pairs follow the reference's SFS sampler
// (src/spectral/les.jl:302-370).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dnsb.h"
#include "../../include/dnsb_cnn.h"
#include "cnn.cuh"
#include "cnn_host.h"

using namespace dnsb::cnn;

namespace {

constexpr int NL = 4;
constexpr int CIN[NL] = {3, 32, 32, 32};
constexpr int COUT[NL] = {32, 32, 32, 6};
constexpr int CICH[NL] = {2, 4, 4, 4};  // input chunks of 8 channels (3 -> 16 padded)
constexpr int COCH[NL] = {4, 4, 4, 2};  // output chunks (6 -> 16 padded)
constexpr int HALO = 4;
constexpr long LOSS_CAP = 1L << 18;     // loss history ring
constexpr unsigned WAIT_LIMIT = 1u << 21;   // polls of up to 1 us each
constexpr int MAX_SMEM = 227 * 1024;

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  });
  return fn;
}

// parameter offsets: per layer W[27][cout][cin] then b[cout]
struct Layout {
  long w[NL], b[NL], total;
  Layout() {
    long o = 0;
    for (int L = 0; L < NL; L++) {
      w[L] = o;
      o += 27L * COUT[L] * CIN[L];
      b[L] = o;
      o += COUT[L];
    }
    total = o;
  }
};
const Layout LAYOUT;

// element offsets (BF16) of the packed B operands of layer L: per (dz, dy)
// pair g and K chunk, the N = 3 x 8 NCH rows (dx, output channel) of 8 K
// values each, in the K-major core-matrix order of the convolution kernel
// (tap t = 3 g + dx; the transposed convolution reads tap 26 - t).
__host__ __device__ inline long pack_fwd(int L, int t, int co, int ci) {
  const int cich = L == 0 ? 2 : 4, coch = L == 3 ? 2 : 4;
  const int g = t / 3, dx = t % 3;
  return (((long)g * cich + ci / 8) * (3 * coch) + dx * coch + co / 8) * 64 + (co % 8) * 8 + ci % 8;
}
__host__ __device__ inline long pack_bwd(int L, int t, int co, int ci) {
  const int cich = L == 0 ? 2 : 4, coch = L == 3 ? 2 : 4;
  const int g = (26 - t) / 3, dx = (26 - t) % 3;
  return (((long)g * coch + co / 8) * (3 * cich) + dx * cich + ci / 8) * 64 + (ci % 8) * 8 + co % 8;
}

struct KernelLayout {  // passed by value to the element-wise kernels
  long w[NL], b[NL], total;
  int cin[NL], cout[NL];
};

KernelLayout kernel_layout() {
  KernelLayout k;
  for (int L = 0; L < NL; L++) {
    k.w[L] = LAYOUT.w[L];
    k.b[L] = LAYOUT.b[L];
    k.cin[L] = CIN[L];
    k.cout[L] = COUT[L];
  }
  k.total = LAYOUT.total;
  return k;
}

struct Packs {
  __nv_bfloat16 *f[NL];  // forward B operands
  __nv_bfloat16 *d[NL];  // transposed (backward-data) B operands, L >= 1
};

// which parameter index p is: layer, and (t, co, ci) or bias co
__device__ inline void locate(const KernelLayout &k, long p, int &L, int &t, int &co, int &ci,
                              bool &bias) {
  L = 0;
  while (L < NL - 1 && p >= k.w[L + 1]) L++;
  if (p >= k.b[L]) {
    bias = true;
    co = (int)(p - k.b[L]);
    t = ci = 0;
  } else {
    bias = false;
    long r = p - k.w[L];
    ci = (int)(r % k.cin[L]);
    r /= k.cin[L];
    co = (int)(r % k.cout[L]);
    t = (int)(r / k.cout[L]);
  }
}

// Adam update (when lr > 0 or adam != 0) and BF16 packing of every weight.
__global__ void k_adam_pack(KernelLayout k, float *params, const float *grads, float *m, float *v,
                            int adam, float lr, const long long *step, Packs packs) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= k.total) return;
  float w = params[p];
  if (adam) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const double tt = (double)(*step + 1);
    const float c1 = (float)(1.0 - pow((double)b1, tt));
    const float c2 = (float)(1.0 - pow((double)b2, tt));
    const float g = grads[p];
    const float mm = b1 * m[p] + (1.f - b1) * g;
    const float vv = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    w = w - lr * ((mm / c1) / (sqrtf(vv / c2) + eps));
    params[p] = w;
  }
  int L, t, co, ci;
  bool bias;
  locate(k, p, L, t, co, ci, bias);
  if (bias) return;
  const __nv_bfloat16 wb = __float2bfloat16_rn(w);
  packs.f[L][pack_fwd(L, t, co, ci)] = wb;
  if (L > 0) packs.d[L][pack_bwd(L, t, co, ci)] = wb;
}

// split-K partials of one layer's weight gradient -> grads (fixed order)
__global__ void k_wgrad_reduce(const float *partial, int ngroups, int nsplit, int N, int G,
                               int cipad, int cin, int cout, int ones_slot, float *gw, float *gb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nw = 27 * cout * cin;
  if (i >= nw + cout) return;
  int gi, m, n;
  if (i < nw) {
    const int ci = i % cin, co = (i / cin) % cout, t = i / (cin * cout);
    gi = t / G;
    m = (t % G) * cipad + ci;
    n = co;
  } else {
    gi = ngroups - 1;
    m = ones_slot * cipad;
    n = i - nw;
  }
  float s = 0.f;
  for (int sp = 0; sp < nsplit; sp++) s += partial[(((long)sp * ngroups + gi) * 128 + m) * N + n];
  if (i < nw) gw[i] = s;
  else gb[n] = s;
}

__device__ inline unsigned long long splitmix(unsigned long long x) {
  unsigned long long z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ inline uint4 chunk3(float a, float b, float c) {
  const float v[8] = {a, b, c, 0.f, 0.f, 0.f, 0.f, 0.f};
  return pack8(v);
}

// random crops of the dataset: input with its halo (chunk 0 of x0) and the
// normalised targets of the crop
__global__ void k_crops(const float *data, int nsnap, int n, int B, int crop, int P,
                        unsigned long long seed, const long long *step, uint4 *x0, float4 *tgt) {
  const long P3 = (long)P * P * P, c3 = (long)crop * crop * crop;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)B * (P3 + c3)) return;
  const bool tpart = i >= (long)B * P3;
  const long r = tpart ? i - (long)B * P3 : i;
  const int b = (int)(tpart ? r / c3 : r / P3);
  long v = tpart ? r % c3 : r % P3;
  const int side = tpart ? crop : P;
  const int x = (int)(v % side), y = (int)((v / side) % side), z = (int)(v / ((long)side * side));
  const unsigned long long key = (unsigned long long)(*step) * 64ull + (unsigned long long)b;
  const unsigned long long h0 = splitmix(seed ^ splitmix(4 * key));
  const int snap = (int)(h0 % (unsigned long long)nsnap);
  const int ox = (int)(splitmix(h0 + 1) % (unsigned long long)n);
  const int oy = (int)(splitmix(h0 + 2) % (unsigned long long)n);
  const int oz = (int)(splitmix(h0 + 3) % (unsigned long long)n);
  const long n3 = (long)n * n * n;
  const float *s = data + (long)snap * 9 * n3;
  const int h = tpart ? 0 : HALO;
  const int gx = ((ox + x - h) % n + n) % n, gy = ((oy + y - h) % n + n) % n, gz = ((oz + z - h) % n + n) % n;
  const long gi = ((long)gz * n + gy) * n + gx;
  if (!tpart) {
    x0[(long)b * 2 * P3 + v] = chunk3(s[gi], s[n3 + gi], s[2 * n3 + gi]);
  } else {
    const long o = (((long)b * P + z) * P + y) * P + x;
    tgt[2 * o] = make_float4(s[3 * n3 + gi], s[4 * n3 + gi], s[5 * n3 + gi], s[6 * n3 + gi]);
    tgt[2 * o + 1] = make_float4(s[7 * n3 + gi], s[8 * n3 + gi], 0.f, 0.f);
  }
}

// a caller batch: x [B][3][P^3], t [B][6][crop^3]
__global__ void k_batch_in(const float *x, const float *t, int B, int crop, int P, uint4 *x0,
                           float4 *tgt) {
  const long P3 = (long)P * P * P, c3 = (long)crop * crop * crop;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)B * (P3 + c3)) return;
  if (i < (long)B * P3) {
    const int b = (int)(i / P3);
    const long v = i % P3;
    const float *xb = x + (long)b * 3 * P3;
    x0[(long)b * 2 * P3 + v] = chunk3(xb[v], xb[P3 + v], xb[2 * P3 + v]);
  } else {
    const long r = i - (long)B * P3;
    const int b = (int)(r / c3);
    const long v = r % c3;
    const int x = (int)(v % crop), y = (int)((v / crop) % crop), z = (int)(v / ((long)crop * crop));
    const float *tb = t + (long)b * 6 * c3;
    const long o = (((long)b * P + z) * P + y) * P + x;
    tgt[2 * o] = make_float4(tb[v], tb[c3 + v], tb[2 * c3 + v], tb[3 * c3 + v]);
    tgt[2 * o + 1] = make_float4(tb[4 * c3 + v], tb[5 * c3 + v], 0.f, 0.f);
  }
}

// the periodic field with a halo of 4: from cell-centred values v[3][n^3]
// or from the staggered ghosted FV fields (the cell average of the two
// faces, operators.jl:71-72); scaled by in_scale
// grid (ceil(P / blockDim.x), P, P): x along the threads, y and z from the
// block (no division per voxel); the halo (HALO < n) wraps by one correction
__global__ void k_infer_in(const double *v, const double *ux, const double *uy, const double *uz,
                           int n, int P, const float *in_scale, uint4 *x0) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
  if (x >= P) return;
  const long i = ((long)z * P + y) * P + x;
  auto wrap = [n](int a) { return a < 0 ? a + n : (a >= n ? a - n : a); };
  const int cx = wrap(x - HALO), cy = wrap(y - HALO), cz = wrap(z - HALO);
  double a, b, c;
  if (v) {
    const long n3 = (long)n * n * n, gi = ((long)cz * n + cy) * n + cx;
    a = v[gi];
    b = v[n3 + gi];
    c = v[2 * n3 + gi];
  } else {
    const long NX = n + 2, NY = n + 2;
    auto G = [&](int I, int J, int K) { return ((long)K * NY + J) * NX + I; };
    const int I = cx + 1, J = cy + 1, K = cz + 1;
    a = 0.5 * (ux[G(I - 1, J, K)] + ux[G(I, J, K)]);
    b = 0.5 * (uy[G(I, J - 1, K)] + uy[G(I, J, K)]);
    c = 0.5 * (uz[G(I, J, K - 1)] + uz[G(I, J, K)]);
  }
  x0[i] = chunk3((float)a * in_scale[0], (float)b * in_scale[1], (float)c * in_scale[2]);
}

// loss of the step (partials in a fixed order) into the history ring; the
// step counter advances when `advance`
__global__ void k_tail(const float *part, int nparts, float inv_count, float *hist, long long *step,
                       int advance) {
  __shared__ float sh[256];
  float s = 0.f;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    hist[*step % LOSS_CAP] = sh[0] * inv_count;
    if (advance) *step += 1;
  }
}

// ---------------------------------------------------------------- host --

struct Volume {
  int P = 0, B = 0, side = 0;  // side: crop (training) or field (inference)
  uint4 *in[NL] = {};          // input of layer L: x0 (2 chunks), h1..h3 (4)
  uint4 *z[3] = {};            // pre-activations of layers 1..3
  uint4 *gz[NL] = {};          // gradients of the layer outputs (training)
  float4 *tgt = nullptr;       // targets (training)
  CUtensorMap fwd[NL], bwd[NL], flatA[NL], flatB[NL];
  int Rf = 0, Rb = 0;          // patch rows of forward / transposed reads
  int subf = 1, subb = 1;      // 126-output sub-tiles per plane load (1-4), forward / transposed
  int Rw = 0, wstages = 0;     // weight gradient: rows per K-block, K-blocks in flight
};

struct Prof {
  cudaEvent_t a, b;
  int kind;
  double flops;
};

}  // namespace

struct dnsb_cnn {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nsm = 148;
  std::string err;
  std::vector<void *> allocs;
  long launches = 0;
  Volume tr, inf;
  bool have_tr = false, have_inf = false;
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
  Packs packs{};
  float *scales = nullptr;     // in[3] (pad 4), out[6]
  float *partial[NL] = {};
  long partial_n[NL] = {};
  float *loss_part = nullptr;
  int loss_nparts = 0, loss_nparts_used = 0;
  float *hist = nullptr;
  long long *step = nullptr;
  long h_steps = 0;
  int *deverr = nullptr;
  const float *data = nullptr;
  int nsnap = 0, ndata = 0;
  bool prof_on = false;
  std::vector<Prof> prof_pending;
  std::vector<cudaEvent_t> evpool;
  double prof_ms[4] = {}, prof_flops[4] = {};
  long prof_n[4] = {};
  unsigned long long serial = 0;  // creation number, unique in the process
  bool pdl = true;  // convolutions launched as programmatic dependents (DNSB_CNN_PDL=0: ordinary)
};

namespace dnsb_internal {

unsigned long long cnn_serial(const dnsb_cnn *c) { return c->serial; }
bool cnn_profiling(const dnsb_cnn *c) { return c->prof_on; }

}  // namespace dnsb_internal

namespace {

std::mutex g_err_mu;
std::string g_create_err;

int cfail(dnsb_cnn *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  else {
    std::lock_guard<std::mutex> l(g_err_mu);
    g_create_err = buf;
  }
  return code;
}

#define CC(c, call)                                                                             \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return cfail(c, DNSB_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,   \
                   __LINE__);                                                                   \
  } while (0)

template <typename T>
int dal(dnsb_cnn *c, T **p, size_t count) {
  void *q = nullptr;
  const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
  if (cudaMalloc(&q, bytes) != cudaSuccess) {
    cudaGetLastError();
    return cfail(c, DNSB_ENOMEM, "cudaMalloc of %zu bytes failed", bytes);
  }
  c->allocs.push_back(q);
  CC(c, cudaMemset(q, 0, bytes));
  *p = (T *)q;
  return 0;
}

int ensure_dev(dnsb_cnn *c) {
  int d = -1;
  if (cudaGetDevice(&d) != cudaSuccess) return cfail(c, DNSB_ECUDA, "cudaGetDevice failed");
  if (d != c->device) CC(c, cudaSetDevice(c->device));
  return 0;
}

int deverr_check(dnsb_cnn *c) {
  int e = 0;
  CC(c, cudaMemcpy(&e, c->deverr, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    cudaMemset(c->deverr, 0, sizeof(int));
    return cfail(c, DNSB_ECUDA, "a tensor-core kernel's device-side wait ran out of its limit (code %d)", e);
  }
  return 0;
}

// patch rows of a tile of `sub` sub-tiles: offsets x0 + s + (dy + e) P + 126 sb
// + m, x0 < P, sb < sub, m < 128
int patch_rows(int P, int s, int e, int sub) {
  const long M = (long)(P - 1) + (long)(sub - 1) * TILE_OUT + (TILE_M - 1) + s + (long)(2 + e) * P;
  return (int)(M / P) + 1;
}

// The chunked-voxel tensors are described with 8-byte elements so that the
// innermost box dimension is a whole x-row (16 P bytes) or a whole run of
// positions (1 KB): TMA moves long rows instead of 16-byte pieces.  The
// copy is byte-exact (no conversion; out-of-bounds elements read as zero).
// Conv plane: dims {2P (x and 8 channels), P (y), P (z), chunks * B}, box
// {2P, R, 1, chunks} -> shared memory [chunk][row][x][16 B] (one ring slot).
int make_map_patch(dnsb_cnn *c, CUtensorMap *m, void *base, int P, int chunks, int B, int R) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return cfail(c, DNSB_ECUDA, "cuTensorMapEncodeTiled is not available");
  if (2 * P > 256 || R > 256 || chunks > 256) return cfail(c, DNSB_EUNSUP, "TMA box beyond 256 (P %d, R %d)", P, R);
  const cuuint64_t dims[4] = {2ull * P, (cuuint64_t)P, (cuuint64_t)P, (cuuint64_t)chunks * B};
  const cuuint64_t strides[3] = {16ull * P, 16ull * P * P, 16ull * P * P * P};
  const cuuint32_t box[4] = {(cuuint32_t)(2 * P), (cuuint32_t)R, 1, (cuuint32_t)chunks};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, base, dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cfail(c, DNSB_ECUDA, "cuTensorMapEncodeTiled (patch) failed: %d", (int)r);
  return 0;
}

constexpr int RING_MAX = 12, RING_MIN = 4;
constexpr size_t CONV_EXTRA = CONV_BARS + CONV_XBUF + 1024;  // barriers, exchange, alignment slack

// shared memory of a convolution with the largest plane ring that fits
// (at most RING_MAX slots); 0 when not even RING_MIN slots fit
size_t conv_smem(int ci, int co, int P, int R, int *nslot, uint32_t *slot, uint32_t *stride,
                 uint32_t *wbytes) {
  *slot = (uint32_t)ci * R * P * 16;
  *stride = (*slot + 1023) & ~1023u;
  *wbytes = 27u * ci * co * 128;
  const long room = (long)MAX_SMEM - (long)*wbytes - (long)CONV_EXTRA;
  const int n = (int)std::min<long>(RING_MAX, room / (long)*stride);
  *nslot = n;
  if (n < RING_MIN) return 0;
  return (size_t)*wbytes + (size_t)n * *stride + CONV_EXTRA;
}

template <int CI, int CO, int MODE>
int setup_conv_attr(dnsb_cnn *c, size_t smem) {
  if (smem > (size_t)MAX_SMEM) return cfail(c, DNSB_EUNSUP, "convolution needs %zu bytes of shared memory", smem);
  CC(c, cudaFuncSetAttribute(k_conv<CI, CO, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return 0;
}

int alloc_volume(dnsb_cnn *c, Volume &V, int side, int B, bool training) {
  V.side = side;
  V.B = B;
  V.P = side + 2 * HALO;
  const int P = V.P;
  const size_t P3 = (size_t)P * P * P;
  int rc;
  if ((rc = dal(c, &V.in[0], (size_t)B * 2 * P3))) return rc;
  for (int L = 1; L < NL; L++)
    if ((rc = dal(c, &V.in[L], (size_t)B * 4 * P3))) return rc;
  if (training) {
    for (int L = 0; L < 3; L++)
      if ((rc = dal(c, &V.z[L], (size_t)B * 4 * P3))) return rc;
    for (int L = 0; L < NL; L++)
      if ((rc = dal(c, &V.gz[L], (size_t)B * COCH[L] * P3))) return rc;
    if ((rc = dal(c, &V.tgt, (size_t)B * P3 * 2))) return rc;
  }
  // up to four 126-output sub-tiles per plane load (fewer copies per
  // output): the most whose wider patch fits the plane and a ring of at
  // least RING_MIN planes
  {
    auto most = [&](int s, int e) {
      for (int sub = 4; sub > 1; sub--) {
        int ns;
        uint32_t sl, st, wb;
        const int r = patch_rows(P, s, e, sub);
        if (r <= P && conv_smem(4, 4, P, r, &ns, &sl, &st, &wb)) return sub;
      }
      return 1;
    };
    V.subf = most(0, 0);
    V.subb = most(-2, 1);
  }
  V.Rf = patch_rows(P, 0, 0, V.subf);
  V.Rb = patch_rows(P, -2, 1, V.subb);
  if (V.Rf > P || V.Rb > P)
    return cfail(c, DNSB_EUNSUP, "side %d too small: the 128-position tiles need %d patch rows", side,
                 std::max(V.Rf, V.Rb));
  {
    int ns;
    uint32_t sl, st, wb;
    if (!conv_smem(4, 4, P, V.Rf, &ns, &sl, &st, &wb) ||
        (training && !conv_smem(4, 4, P, V.Rb, &ns, &sl, &st, &wb)))
      return cfail(c, DNSB_EUNSUP, "side %d too large: a convolution's plane ring (%d slots of %u bytes) "
                   "does not fit in shared memory", side, RING_MIN, sl);
  }
  if (training) {
    // weight-gradient K-blocks of R whole rows (R P positions, a multiple of
    // 16): the most rows with at least two blocks in flight (up to four when
    // they fit), at most 16 rows and P -- fewer, larger copies win (crop 32:
    // 8 rows x 2 blocks 0.289 ms, 6 x 3 0.305, 4 x 4 0.358 per training
    // step); DNSB_WGROWS / DNSB_WGSTAGES override
    int best = 0, bstages = 0;
    for (int r = 1; r <= std::min(16, P); r++) {
      if ((r * P) % 16) continue;
      // 16 chunks of taps + 4 of g, 16 bytes each, per position
      const size_t stage = ((size_t)320 * r * P + 1023) & ~(size_t)1023;
      const int ns = (int)std::min<size_t>(WG_STAGES, ((size_t)MAX_SMEM - 1280) / stage);
      if (ns >= 2) {
        best = r;
        bstages = ns;
      }
    }
    const char *er = getenv("DNSB_WGROWS"), *es = getenv("DNSB_WGSTAGES");
    if (er) {
      const int r = atoi(er);
      const size_t stage = (((size_t)320 * r * P) + 1023) & ~(size_t)1023;
      if (r >= 1 && r <= std::min(16, P) && (r * P) % 16 == 0 && 2 * stage + 1280 <= (size_t)MAX_SMEM) {
        best = r;
        bstages = (int)std::min<size_t>(WG_STAGES, ((size_t)MAX_SMEM - 1280) / stage);
      }
    }
    if (es && best) {
      const size_t stage = (((size_t)320 * best * P) + 1023) & ~(size_t)1023;
      const int ns = atoi(es);
      if (ns >= 2 && ns <= WG_STAGES && ns * stage + 1280 <= (size_t)MAX_SMEM) bstages = ns;
    }
    if (!best)
      return cfail(c, DNSB_EUNSUP, "crop side %d: no weight-gradient block of whole rows fits (side + 8 must "
                   "allow r (side + 8) to be a multiple of 16 with r <= 16)", side);
    V.Rw = best;
    V.wstages = bstages;
  }
  for (int L = 0; L < NL; L++) {
    if ((rc = make_map_patch(c, &V.fwd[L], V.in[L], P, CICH[L], B, V.Rf))) return rc;
    if (training) {
      if ((rc = make_map_patch(c, &V.flatA[L], V.in[L], P, CICH[L], B, V.Rw))) return rc;
      if ((rc = make_map_patch(c, &V.flatB[L], V.gz[L], P, COCH[L], B, V.Rw))) return rc;
      if (L > 0 && (rc = make_map_patch(c, &V.bwd[L], V.gz[L], P, COCH[L], B, V.Rb))) return rc;
    }
  }
  return 0;
}

cudaEvent_t ev_get(dnsb_cnn *c) {
  if (!c->evpool.empty()) {
    cudaEvent_t e = c->evpool.back();
    c->evpool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void prof_begin(dnsb_cnn *c, Prof &p, int kind, double flops) {
  p.kind = kind;
  p.flops = flops;
  if (!c->prof_on) return;
  p.a = ev_get(c);
  p.b = ev_get(c);
  cudaEventRecord(p.a, c->stream);
}
void prof_end(dnsb_cnn *c, Prof &p) {
  c->launches++;
  if (!c->prof_on) return;
  cudaEventRecord(p.b, c->stream);
  c->prof_pending.push_back(p);
}

int grid_for(dnsb_cnn *c, const void *kernel, size_t smem, long work, int threads) {
  int per = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess || per < 1) {
    cudaGetLastError();
    per = 1;
  }
  return (int)std::max<long>(1, std::min<long>(work, (long)c->nsm * per));
}

// one forward / transposed convolution of layer L on volume V
template <int CI, int CO, int MODE>
int run_conv(dnsb_cnn *c, Volume &V, int L, const CUtensorMap &map, bool transposed, uint4 *out,
             uint4 *zout, const uint4 *zin, double *infer_out, int kind) {
  ConvArgs a{};
  a.P = V.P;
  a.Pz = V.P;
  a.B = V.B;
  a.s = transposed ? -2 : 0;
  a.e = transposed ? 1 : 0;
  a.R = transposed ? V.Rb : V.Rf;
  a.sub = transposed ? V.subb : V.subf;
  // output box of a forward layer L: P - 2 (L+1); of the transposed one: the
  // box of layer L's input (layer L-1's output)
  a.Do = transposed ? V.P - 2 * L : V.P - 2 * (L + 1);
  a.tpp = (a.Do * a.P + a.sub * TILE_OUT - 1) / (a.sub * TILE_OUT);
  a.ntiles = V.B * a.Do * a.tpp;
  const size_t smem = conv_smem(CI, CO, a.P, a.R, &a.nslot, &a.slot_bytes, &a.slot_stride, &a.w_bytes);
  if (!smem) return cfail(c, DNSB_EUNSUP, "convolution plane ring does not fit in shared memory");
  a.wait_limit = WAIT_LIMIT;
  a.wpack = reinterpret_cast<const uint4 *>(transposed ? c->packs.d[L] : c->packs.f[L]);
  a.bias = c->params + LAYOUT.b[L];
  a.out = out;
  a.zout = zout;
  a.zin = zin;
  a.target = V.tgt;
  a.loss_scale = 2.0f / (float)((double)V.B * V.side * V.side * V.side * 6);
  a.loss_part = c->loss_part;
  a.infer_out = infer_out;
  a.oscale = c->scales + 4;
  a.err = c->deverr;
  int rc = setup_conv_attr<CI, CO, MODE>(c, smem);
  if (rc) return rc;
  const int grid = grid_for(c, (const void *)k_conv<CI, CO, MODE>, smem, a.ntiles, CONV_THREADS);
  if (MODE == FWD_LOSS) {
    if (grid > c->loss_nparts) return cfail(c, DNSB_EUNSUP, "loss partials: grid %d > %d", grid, c->loss_nparts);
    c->loss_nparts_used = grid;
  }
  const double flops = 2.0 * 27 * CIN[L] * COUT[L] * V.B * pow((double)(V.P - 2 * (L + 1)), 3);
  Prof p;
  prof_begin(c, p, kind, flops);
  {
    // programmatic dependent launch (the kernel waits before any memory access)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(CONV_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = c->pdl ? 1 : 0;
    CC(c, cudaLaunchKernelEx(&cfg, k_conv<CI, CO, MODE>, map, a));
  }
  prof_end(c, p);
  CC(c, cudaGetLastError());
  return 0;
}

template <int CI, int CO>
int run_wgrad(dnsb_cnn *c, Volume &V, int L) {
  WgradArgs a{};
  a.P = V.P;
  a.Pz = V.P;
  a.B = V.B;
  a.Do = V.P - 2 * (L + 1);
  a.R = V.Rw;
  a.KB = V.Rw * V.P;
  a.stages = V.wstages;
  a.kpp = (a.Do + a.R - 1) / a.R;
  a.nk = V.B * a.Do * a.kpp;
  constexpr int G = 16 / CI;
  a.ngroups = (NTAPS + G - 1) / G;
  a.ones_slot = NTAPS - (a.ngroups - 1) * G;
  a.a_bytes = (uint32_t)G * CI * a.KB * 16;
  a.stage_bytes = ((a.a_bytes + (uint32_t)CO * a.KB * 16) + 1023) & ~1023u;
  a.wait_limit = WAIT_LIMIT;
  a.err = c->deverr;
  const size_t smem = (size_t)a.stages * a.stage_bytes + 256 + 1024;
  if (smem > (size_t)MAX_SMEM) return cfail(c, DNSB_EUNSUP, "weight gradient needs %zu bytes", smem);
  CC(c, cudaFuncSetAttribute(k_wgrad<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_wgrad<CI, CO>, NTHREADS, smem) != cudaSuccess || per < 1) {
    cudaGetLastError();
    per = 1;
  }
  a.nsplit = std::max(1, std::min(a.nk, (c->nsm * per) / a.ngroups));
  const long need = (long)a.nsplit * a.ngroups * 128 * (8 * CO);
  if (need > c->partial_n[L]) return cfail(c, DNSB_EUNSUP, "weight-gradient partials: %ld > %ld", need, c->partial_n[L]);
  a.partial = c->partial[L];
  const double flops = 2.0 * 27 * CIN[L] * COUT[L] * V.B * pow((double)a.Do, 3);
  Prof p;
  prof_begin(c, p, 2, flops);
  {
    // programmatic dependent launch (the kernel waits before any memory access)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(a.ngroups * a.nsplit));
    cfg.blockDim = dim3(NTHREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = c->pdl ? 1 : 0;
    CC(c, cudaLaunchKernelEx(&cfg, k_wgrad<CI, CO>, V.flatA[L], V.flatB[L], a));
  }
  prof_end(c, p);
  CC(c, cudaGetLastError());
  const int N = 8 * CO;
  const int nout = 27 * COUT[L] * CIN[L] + COUT[L];
  Prof p2;
  prof_begin(c, p2, 3, 0);
  k_wgrad_reduce<<<(nout + 255) / 256, 256, 0, c->stream>>>(
      c->partial[L], a.ngroups, a.nsplit, N, G, 8 * CI, CIN[L], COUT[L], a.ones_slot,
      c->grads + LAYOUT.w[L], c->grads + LAYOUT.b[L]);
  prof_end(c, p2);
  CC(c, cudaGetLastError());
  return 0;
}

// forward with the loss, backward, gradients reduced (training volume)
int fwd_bwd(dnsb_cnn *c) {
  Volume &V = c->tr;
  int rc;
  if ((rc = run_conv<2, 4, FWD_GELU>(c, V, 0, V.fwd[0], false, V.in[1], V.z[0], nullptr, nullptr, 0)) ||
      (rc = run_conv<4, 4, FWD_GELU>(c, V, 1, V.fwd[1], false, V.in[2], V.z[1], nullptr, nullptr, 0)) ||
      (rc = run_conv<4, 4, FWD_GELU>(c, V, 2, V.fwd[2], false, V.in[3], V.z[2], nullptr, nullptr, 0)) ||
      (rc = run_conv<4, 2, FWD_LOSS>(c, V, 3, V.fwd[3], false, V.gz[3], nullptr, nullptr, nullptr, 0)))
    return rc;
  if ((rc = run_wgrad<4, 2>(c, V, 3)) ||
      (rc = run_conv<2, 4, DGRAD>(c, V, 3, V.bwd[3], true, V.gz[2], nullptr, V.z[2], nullptr, 1)) ||
      (rc = run_wgrad<4, 4>(c, V, 2)) ||
      (rc = run_conv<4, 4, DGRAD>(c, V, 2, V.bwd[2], true, V.gz[1], nullptr, V.z[1], nullptr, 1)) ||
      (rc = run_wgrad<4, 4>(c, V, 1)) ||
      (rc = run_conv<4, 4, DGRAD>(c, V, 1, V.bwd[1], true, V.gz[0], nullptr, V.z[0], nullptr, 1)) ||
      (rc = run_wgrad<2, 4>(c, V, 0)))
    return rc;
  return 0;
}

int adam_pack(dnsb_cnn *c, bool adam, float lr) {
  const KernelLayout kl = kernel_layout();
  Prof p;
  prof_begin(c, p, 3, 0);
  k_adam_pack<<<(unsigned)((kl.total + 255) / 256), 256, 0, c->stream>>>(
      kl, c->params, c->grads, c->m, c->v, adam ? 1 : 0, lr, c->step, c->packs);
  prof_end(c, p);
  CC(c, cudaGetLastError());
  return 0;
}

int tail(dnsb_cnn *c, bool advance) {
  Volume &V = c->tr;
  const double count = (double)V.B * V.side * V.side * V.side * 6;
  Prof p;
  prof_begin(c, p, 3, 0);
  k_tail<<<1, 256, 0, c->stream>>>(c->loss_part, c->loss_nparts_used, (float)(1.0 / count), c->hist,
                                   c->step, advance ? 1 : 0);
  prof_end(c, p);
  CC(c, cudaGetLastError());
  return 0;
}

int prof_harvest(dnsb_cnn *c) {
  if (c->prof_pending.empty()) return 0;
  CC(c, cudaStreamSynchronize(c->stream));
  for (auto &p : c->prof_pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    c->prof_ms[p.kind] += ms;
    c->prof_n[p.kind] += 1;
    c->prof_flops[p.kind] += p.flops;
    c->evpool.push_back(p.a);
    c->evpool.push_back(p.b);
  }
  c->prof_pending.clear();
  return 0;
}

}  // namespace

extern "C" {

int dnsb_cnn_create(int device, void *stream, int batch, int crop, int nfield, dnsb_cnn **out) {
  if (!out) return cfail(nullptr, DNSB_EINVAL, "null output");
  *out = nullptr;
  if (batch < 0 || crop < 0 || nfield < 0 || (batch > 0) != (crop > 0) || (batch == 0 && nfield == 0))
    return cfail(nullptr, DNSB_EINVAL, "need batch > 0 with crop > 0, or nfield > 0");
  if (crop + 2 * HALO > 256 || nfield + 2 * HALO > 256 || batch > 64)
    return cfail(nullptr, DNSB_EUNSUP, "crop + 8 and nfield + 8 must be <= 256, batch <= 64");
  if (!encode_fn()) return cfail(nullptr, DNSB_ECUDA, "cuTensorMapEncodeTiled is not available");
  dnsb_cnn *c = new dnsb_cnn();
  static std::atomic<unsigned long long> created{0};
  c->serial = ++created;
  c->device = device;
  c->stream = (cudaStream_t)stream;
  {
    const char *e = getenv("DNSB_CNN_PDL");
    if (e && atoi(e) == 0) c->pdl = false;
  }
  auto bail = [&](int rc) {
    if (!c->err.empty()) cfail(nullptr, rc, "%s", c->err.c_str());
    dnsb_cnn_destroy(c);
    return rc;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bail(cfail(c, DNSB_ECUDA, "cudaSetDevice(%d) failed", device));
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
  if (major < 10) return bail(cfail(c, DNSB_EUNSUP, "the tensor-core kernels need sm_100 (compute capability %d)", major));
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
  int rc;
  if ((rc = dal(c, &c->params, LAYOUT.total)) || (rc = dal(c, &c->grads, LAYOUT.total)) ||
      (rc = dal(c, &c->m, LAYOUT.total)) || (rc = dal(c, &c->v, LAYOUT.total)) ||
      (rc = dal(c, &c->scales, 16)) || (rc = dal(c, &c->hist, LOSS_CAP)) ||
      (rc = dal(c, &c->step, 1)) || (rc = dal(c, &c->deverr, 4)))
    return bail(rc);
  for (int L = 0; L < NL; L++) {
    if ((rc = dal(c, &c->packs.f[L], 27L * CICH[L] * COCH[L] * 64))) return bail(rc);
    if (L > 0 && (rc = dal(c, &c->packs.d[L], 27L * CICH[L] * COCH[L] * 64))) return bail(rc);
  }
  const float ones[16] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
  if (cudaMemcpy(c->scales, ones, sizeof ones, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(cfail(c, DNSB_ECUDA, "scale upload failed"));
  if (batch > 0) {
    if ((rc = alloc_volume(c, c->tr, crop, batch, true))) return bail(rc);
    c->have_tr = true;
    for (int L = 0; L < NL; L++) {
      const int G = 16 / CICH[L];
      const int ngroups = (NTAPS + G - 1) / G;
      c->partial_n[L] = (long)c->nsm * 2 * 128 * 8 * COCH[L] + (long)ngroups * 128 * 32;
      if ((rc = dal(c, &c->partial[L], c->partial_n[L]))) return bail(rc);
    }
  }
  c->loss_nparts = 2 * c->nsm + 8;
  if ((rc = dal(c, &c->loss_part, c->loss_nparts))) return bail(rc);
  if (nfield > 0) {
    if ((rc = alloc_volume(c, c->inf, nfield, 1, false))) return bail(rc);
    c->have_inf = true;
  }
  *out = c;
  return 0;
}

void dnsb_cnn_destroy(dnsb_cnn *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  else cudaDeviceSynchronize();
  for (auto &p : c->prof_pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (auto e : c->evpool) cudaEventDestroy(e);
  for (void *p : c->allocs) cudaFree(p);
  delete c;
}

const char *dnsb_cnn_last_error(const dnsb_cnn *c) {
  if (c) return c->err.c_str();
  std::lock_guard<std::mutex> l(g_err_mu);
  return g_create_err.c_str();
}

int dnsb_cnn_set_stream(dnsb_cnn *c, void *stream) {
  if (!c) return DNSB_EINVAL;
  c->stream = (cudaStream_t)stream;
  return 0;
}

int dnsb_cnn_sync(dnsb_cnn *c) {
  if (!c) return DNSB_EINVAL;
  int rc;
  if ((rc = ensure_dev(c))) return rc;
  CC(c, cudaStreamSynchronize(c->stream));
  return deverr_check(c);
}

long dnsb_cnn_launch_count(const dnsb_cnn *c) { return c ? c->launches : 0; }

int dnsb_cnn_param_count(const dnsb_cnn *) { return (int)LAYOUT.total; }

int dnsb_cnn_set_params(dnsb_cnn *c, const float *params) {
  if (!c || !params) return c ? cfail(c, DNSB_EINVAL, "null params") : DNSB_EINVAL;
  int rc;
  if ((rc = ensure_dev(c))) return rc;
  CC(c, cudaMemcpyAsync(c->params, params, LAYOUT.total * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CC(c, cudaMemsetAsync(c->m, 0, LAYOUT.total * sizeof(float), c->stream));
  CC(c, cudaMemsetAsync(c->v, 0, LAYOUT.total * sizeof(float), c->stream));
  CC(c, cudaMemsetAsync(c->step, 0, sizeof(long long), c->stream));
  c->h_steps = 0;
  if ((rc = adam_pack(c, false, 0.f))) return rc;
  CC(c, cudaStreamSynchronize(c->stream));
  return 0;
}

int dnsb_cnn_init(dnsb_cnn *c, unsigned long long seed) {
  if (!c) return DNSB_EINVAL;
  std::vector<float> h(LAYOUT.total);
  for (int L = 0; L < NL; L++) {
    const double bound = 1.0 / std::sqrt(27.0 * CIN[L]);
    for (long i = LAYOUT.w[L]; i < LAYOUT.w[L] + 27L * COUT[L] * CIN[L] + COUT[L]; i++) {
      unsigned long long z = seed + (unsigned long long)i + 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z ^= z >> 31;
      const double u = ((double)(z >> 11) + 0.5) * 0x1.0p-53;
      h[i] = (float)((2 * u - 1) * bound);
    }
  }
  return dnsb_cnn_set_params(c, h.data());
}

int dnsb_cnn_get_params(dnsb_cnn *c, float *params) {
  if (!c || !params) return c ? cfail(c, DNSB_EINVAL, "null params") : DNSB_EINVAL;
  int rc;
  if ((rc = ensure_dev(c))) return rc;
  CC(c, cudaMemcpyAsync(params, c->params, LAYOUT.total * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CC(c, cudaStreamSynchronize(c->stream));
  return deverr_check(c);
}

int dnsb_cnn_set_scales(dnsb_cnn *c, const float *in3, const float *out6) {
  if (!c || !in3 || !out6) return c ? cfail(c, DNSB_EINVAL, "null scales") : DNSB_EINVAL;
  int rc;
  if ((rc = ensure_dev(c))) return rc;
  float h[16] = {in3[0], in3[1], in3[2], 1.f, out6[0], out6[1], out6[2], out6[3], out6[4], out6[5]};
  CC(c, cudaMemcpyAsync(c->scales, h, sizeof h, cudaMemcpyHostToDevice, c->stream));
  CC(c, cudaStreamSynchronize(c->stream));
  return 0;
}

int dnsb_cnn_set_dataset(dnsb_cnn *c, const float *data, int nsnap, int n) {
  if (!c || !data || nsnap < 1 || n < 1) return c ? cfail(c, DNSB_EINVAL, "bad dataset") : DNSB_EINVAL;
  c->data = data;
  c->nsnap = nsnap;
  c->ndata = n;
  return 0;
}

int dnsb_cnn_train(dnsb_cnn *c, int nsteps, float lr, unsigned long long seed) {
  if (!c) return DNSB_EINVAL;
  if (!c->have_tr) return cfail(c, DNSB_EINVAL, "no training geometry (batch = 0)");
  if (!c->data) return cfail(c, DNSB_EINVAL, "no dataset");
  if (nsteps < 0 || !(lr > 0)) return cfail(c, DNSB_EINVAL, "need nsteps >= 0, lr > 0");
  int rc;
  if ((rc = ensure_dev(c))) return rc;
  Volume &V = c->tr;
  const long P3 = (long)V.P * V.P * V.P, c3 = (long)V.side * V.side * V.side;
  const long work = (long)V.B * (P3 + c3);
  for (int s = 0; s < nsteps; s++) {
    Prof p;
    prof_begin(c, p, 3, 0);
    k_crops<<<(unsigned)((work + 255) / 256), 256, 0, c->stream>>>(
        c->data, c->nsnap, c->ndata, V.B, V.side, V.P, seed, c->step, V.in[0], V.tgt);
    prof_end(c, p);
    CC(c, cudaGetLastError());
    if ((rc = fwd_bwd(c)) || (rc = adam_pack(c, true, lr)) || (rc = tail(c, true))) return rc;
    c->h_steps++;
  }
  return 0;
}

int dnsb_cnn_steps(dnsb_cnn *c, long *steps) {
  if (!c || !steps) return DNSB_EINVAL;
  int rc;
  if ((rc = ensure_dev(c))) return rc;
  long long s = 0;
  CC(c, cudaMemcpyAsync(&s, c->step, sizeof s, cudaMemcpyDeviceToHost, c->stream));
  CC(c, cudaStreamSynchronize(c->stream));
  *steps = (long)s;
  return deverr_check(c);
}

int dnsb_cnn_losses(dnsb_cnn *c, float *out, long first, long count) {
  if (!c || !out || first < 0 || count < 0) return c ? cfail(c, DNSB_EINVAL, "bad range") : DNSB_EINVAL;
  long steps = 0;
  int rc;
  if ((rc = dnsb_cnn_steps(c, &steps))) return rc;
  if (first + count > steps || first < steps - LOSS_CAP)
    return cfail(c, DNSB_EINVAL, "losses %ld..%ld not held (steps %ld, history %ld)", first,
                 first + count, steps, LOSS_CAP);
  for (long i = 0; i < count;) {
    const long s = (first + i) % LOSS_CAP;
    const long n = std::min(count - i, LOSS_CAP - s);
    CC(c, cudaMemcpy(out + i, c->hist + s, n * sizeof(float), cudaMemcpyDeviceToHost));
    i += n;
  }
  return 0;
}

int dnsb_cnn_batch(dnsb_cnn *c, const float *x, const float *t, int nadam, float lr, float *loss_out,
                   float *grads_out) {
  if (!c || !x || !t || nadam < 0) return c ? cfail(c, DNSB_EINVAL, "bad argument") : DNSB_EINVAL;
  if (!c->have_tr) return cfail(c, DNSB_EINVAL, "no training geometry (batch = 0)");
  if (nadam > 0 && !(lr > 0)) return cfail(c, DNSB_EINVAL, "need lr > 0");
  int rc;
  if ((rc = ensure_dev(c))) return rc;
  Volume &V = c->tr;
  const long P3 = (long)V.P * V.P * V.P, c3 = (long)V.side * V.side * V.side;
  const long work = (long)V.B * (P3 + c3);
  Prof p;
  prof_begin(c, p, 3, 0);
  k_batch_in<<<(unsigned)((work + 255) / 256), 256, 0, c->stream>>>(x, t, V.B, V.side, V.P, V.in[0], V.tgt);
  prof_end(c, p);
  CC(c, cudaGetLastError());
  for (int i = 0; i < std::max(1, nadam); i++) {
    if ((rc = fwd_bwd(c))) return rc;
    if (i == 0) {
      if ((rc = tail(c, false))) return rc;
      if (grads_out)
        CC(c, cudaMemcpyAsync(grads_out, c->grads, LAYOUT.total * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
      if (loss_out) {
        CC(c, cudaStreamSynchronize(c->stream));
        long long s = 0;
        CC(c, cudaMemcpy(&s, c->step, sizeof s, cudaMemcpyDeviceToHost));
        CC(c, cudaMemcpy(loss_out, c->hist + s % LOSS_CAP, sizeof(float), cudaMemcpyDeviceToHost));
      }
    }
    if (nadam > 0) {
      if ((rc = adam_pack(c, true, lr)) || (rc = tail(c, true))) return rc;
      c->h_steps++;
    }
  }
  CC(c, cudaStreamSynchronize(c->stream));
  return deverr_check(c);
}

static int infer_common(dnsb_cnn *c, const double *v, const double *ux, const double *uy,
                        const double *uz, double *tau) {
  if (!c || !tau) return c ? cfail(c, DNSB_EINVAL, "null argument") : DNSB_EINVAL;
  if (!c->have_inf) return cfail(c, DNSB_EINVAL, "no inference geometry (nfield = 0)");
  int rc;
  if ((rc = ensure_dev(c))) return rc;
  Volume &V = c->inf;
  if (V.side <= HALO) return cfail(c, DNSB_EUNSUP, "inference side %d <= halo %d", V.side, HALO);
  Prof p;
  prof_begin(c, p, 3, 0);
  {
    const unsigned bx = std::min(256u, (unsigned)(V.P + 31) / 32 * 32);
    k_infer_in<<<dim3((V.P + bx - 1) / bx, V.P, V.P), bx, 0, c->stream>>>(v, ux, uy, uz, V.side, V.P, c->scales,
                                                                         V.in[0]);
  }
  prof_end(c, p);
  CC(c, cudaGetLastError());
  // inference keeps no pre-activations (zout = nullptr)
  if ((rc = run_conv<2, 4, FWD_GELU>(c, V, 0, V.fwd[0], false, V.in[1], nullptr, nullptr, nullptr, 0)) ||
      (rc = run_conv<4, 4, FWD_GELU>(c, V, 1, V.fwd[1], false, V.in[2], nullptr, nullptr, nullptr, 0)) ||
      (rc = run_conv<4, 4, FWD_GELU>(c, V, 2, V.fwd[2], false, V.in[3], nullptr, nullptr, nullptr, 0)) ||
      (rc = run_conv<4, 2, FWD_INFER>(c, V, 3, V.fwd[3], false, nullptr, nullptr, nullptr, tau, 0)))
    return rc;
  return 0;
}

int dnsb_cnn_infer_cells(dnsb_cnn *c, const double *v, double *tau) {
  if (!v) return c ? cfail(c, DNSB_EINVAL, "null v") : DNSB_EINVAL;
  return infer_common(c, v, nullptr, nullptr, nullptr, tau);
}

int dnsb_cnn_infer(dnsb_cnn *c, const double *ux, const double *uy, const double *uz, double *tau) {
  if (!ux || !uy || !uz) return c ? cfail(c, DNSB_EINVAL, "null field") : DNSB_EINVAL;
  return infer_common(c, nullptr, ux, uy, uz, tau);
}

int dnsb_cnn_profile(dnsb_cnn *c, int enable) {
  if (!c) return DNSB_EINVAL;
  int rc;
  if ((rc = prof_harvest(c))) return rc;
  c->prof_on = enable != 0;
  for (int k = 0; k < 4; k++) c->prof_ms[k] = c->prof_flops[k] = 0, c->prof_n[k] = 0;
  return 0;
}

int dnsb_cnn_profile_read(dnsb_cnn *c, int kind, double *ms, long *launches, double *flops) {
  if (!c || kind < 0 || kind > 3) return DNSB_EINVAL;
  int rc;
  if ((rc = prof_harvest(c))) return rc;
  if (ms) *ms = c->prof_ms[kind];
  if (launches) *launches = c->prof_n[kind];
  if (flops) *flops = c->prof_flops[kind];
  return 0;
}

}  // extern "C"
