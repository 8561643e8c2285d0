// cnn.cuh -- tensor-core kernels of the sub-filter-stress CNN closure.
//
// The network (no counterpart in the reference, which has no learned
// closure): 4 layers of 3x3x3 convolutions, channels 3 -> 32 -> 32 -> 32 ->
// 6, bias, GELU (tanh form) after the first three, periodic padding on the full
// field.  Every convolution is an implicit GEMM on the 5th-generation tensor
// cores: BF16 operands staged in shared memory by TMA, FP32 accumulators in
// tensor memory (tcgen05.mma, cta_group::1, M = 128), read back with
// tcgen05.ld for a fused epilogue.
//
// Activation layout ("chunked voxels"): a volume of P x P x Pz voxels per
// sample; channels in chunks of 8 BF16 values (16 bytes); element
// [b][chunk][z][y][x][8].  Every layer of a network lives in the same
// geometry (same P, Pz): layer L's output occupies the box [0, Do)^3, Do =
// P - 2L, and the input voxel of output (x, y, z) for tap (dx, dy, dz) is
// (x + s + dx, y + s + dy, z + s + dz) with s = 0 (forward, "valid"
// convolution) or s = -2 (the transposed convolution of the backward pass;
// the box of the input is surrounded by zeros).  Voxels outside an output's
// box hold zeros: the buffers are cleared once and every kernel writes zeros
// at the positions of its tiles that are outside the box.
//
// Forward / transposed convolution (k_conv): one tile = 128 consecutive
// positions f = y*P + x of one plane of one sample (rows of the GEMM).  With
// the input patch of that tile staged as whole rows [chunk][dz][row][x][16 B]
// (one 4-D TMA box: x-rows of 16 P bytes x R rows x 3 planes x CI chunks), the 128
// GEMM rows of every (dy, dz) tap pair are 128 consecutive 16-byte rows of
// the patch starting at offset x0 + s + (dy + e) P, e = 1 for s < 0 (one
// extra row below the tile so that offsets stay >= 0).  So the A operand is a
// K-major canonical layout without swizzle (8-row core matrices of 128
// contiguous bytes, SBO = 128 B, LBO = the chunk stride), addressed by its
// start alone: no im2col copy.  The three x-taps are columns of the GEMM
// (N = 3 x output channels), and the epilogue adds row m + dx of column
// block dx into output m, so a tile yields 126 outputs.  Positions with
// x >= Do inside a row compute garbage that the epilogue replaces by zeros.
// B (the weights) is resident in shared memory for the whole persistent
// CTA, packed in the K-major core-matrix order.
//
// Weight gradient (k_wgrad): D[(tap slot j, ci)][co] = sum_o h[o + t_j][ci]
// g[o][co] over the output positions o (the GEMM's K).  Both operands are
// MN-major canonical layouts without swizzle, straight from the chunked
// activations: a K-block of R whole rows of one plane (R P positions) is one
// TMA box [chunk][R rows][x] per tap, the tap's x shift running past the row
// end into zeros where g is zero anyway; 128 / (8 CI) taps fill the 128 rows (the slot
// after the last real tap holds ones, which makes that row the bias
// gradient).  Split-K partials are reduced in a fixed order.
//
// Warp roles: warp 0 issues the TMA copies, warp 1 owns the tensor memory
// and issues the MMAs (one thread), the other warps run the epilogue (warp
// w reads TMEM lanes 32 (w % 4) .. + 31): warps 2-5 of the weight gradient
// (192 threads), two groups of four (warps 2-5, 6-9) taking alternate tiles
// of the convolution (320 threads).  Every
// mbarrier wait is bounded; a wait that runs out raises the CTA's abort flag
// and the global error word, every role leaves its loop, the copies and MMAs
// in flight are waited for (bounded), the tensor memory is freed and the CTA
// returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace dnsb {
namespace cnn {

constexpr int NTHREADS = 192;       // weight gradient: TMA, MMA, 4 epilogue warps
constexpr int CONV_GROUPS = 4;      // convolution epilogue: groups of 4 warps taking tiles in turn
constexpr int CONV_THREADS = 96 + 128 * CONV_GROUPS;  // TMA, two MMA, epilogue warps
constexpr int NTAPS = 27;
constexpr int TILE_M = 128;      // GEMM rows (positions) of a convolution tile
constexpr int TILE_OUT = 126;    // outputs of a convolution tile (rows m, m + 1, m + 2 feed output m)
constexpr int CONV_BARS = 512;   // bytes of barriers and flags after the plane ring
constexpr int CONV_XBUF = CONV_GROUPS * 2 * 3 * 2 * 32 * 4;  // lane-quarter boundary exchange, bytes
constexpr int WG_STAGES = 4;
constexpr int CV_STAGES = 2;
enum { DEVERR_CNN_TIMEOUT = 2 };

enum Mode { FWD_GELU = 0, FWD_LOSS = 1, FWD_INFER = 2, DGRAD = 3 };

// ----------------------------------------------------------- PTX helpers --

__device__ __forceinline__ uint32_t saddr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mb_init(uint64_t *b, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void mb_expect(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mb_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
}
__device__ __forceinline__ bool mb_try(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// try_wait that may suspend the thread for up to `ns` nanoseconds while the
// phase is incomplete (returns as soon as it completes)
__device__ __forceinline__ bool mb_try_sleep(uint64_t *b, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}
// non-blocking test of the phase (no suspension)
__device__ __forceinline__ bool mb_test(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: a test first (a phase already complete costs no
// suspending try, measured at ~300 cycles on a completed phase), then at
// most `limit` polls, each suspending up to 1 us (so a waiting role takes
// no issue slots from the working warps); gives up early once the CTA's
// abort flag is raised.
__device__ __forceinline__ bool mb_wait(uint64_t *b, uint32_t parity, unsigned limit,
                                        volatile int *abort_flag) {
  if (mb_test(b, parity)) return true;
  for (unsigned it = 0; it < limit; it++) {
    if (mb_try_sleep(b, parity, 1000)) return true;
    if ((it & 15) == 15 && *abort_flag) return false;
  }
  return false;
}
// named barrier over `n` threads that also ORs a predicate across them
__device__ __forceinline__ bool bar_or(int id, int n, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n barrier.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void tma3(void *dst, const CUtensorMap *m, int c0, int c1, int c2,
                                     uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          saddr(dst)),
      "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(saddr(bar))
      : "memory");
}
__device__ __forceinline__ void tma4(void *dst, const CUtensorMap *m, int c0, int c1, int c2, int c3,
                                     uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
          saddr(dst)),
      "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(saddr(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          saddr(dst)),
      "l"(src), "r"(bytes), "r"(saddr(bar))
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// shared-memory matrix descriptor, no swizzle (layout type 0), version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: BF16 x BF16 -> FP32, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int n, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   saddr(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
// 32 lanes x N columns of FP32 (this warp's lane quarter), into v[0..N)
template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float *v);
template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// three 32-lane x 8-column loads (columns c0, c1, c2) and one wait, into v[0..24)
__device__ __forceinline__ void tmem_ld3x8(uint32_t c0, uint32_t c1, uint32_t c2, float *v) {
  uint32_t r[24];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%24];\n"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8,%9,%10,%11,%12,%13,%14,%15}, [%25];\n"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16,%17,%18,%19,%20,%21,%22,%23}, [%26];\n"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23])
      : "r"(c0), "r"(c1), "r"(c2)
      : "memory");
#pragma unroll
  for (int i = 0; i < 24; i++) v[i] = __uint_as_float(r[i]);
}

// GELU in its tanh form, 0.5 z (1 + tanh(u)) with u = sqrt(2/pi) (z +
// 0.044715 z^3), on the hardware tanh (tanh.approx.f32: about 2^-11
// relative, below the BF16 rounding that follows): six instructions, one
// of them on the special-function unit.
constexpr float GELU_C = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float GELU_A = 0.044715f;
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_f(float z) {
  const float u = z * fmaf(GELU_C * GELU_A, z * z, GELU_C);
  const float h = 0.5f * z;
  return fmaf(h, tanh_hw(u), h);
}
// d/dz [0.5 z (1 + t)] = 0.5 (1 + t) + 0.5 z (1 - t^2) u'(z)
__device__ __forceinline__ float gelu_grad_f(float z) {
  const float z2 = z * z;
  const float t = tanh_hw(z * fmaf(GELU_C * GELU_A, z2, GELU_C));
  const float du = fmaf(3.f * GELU_C * GELU_A, z2, GELU_C);
  return fmaf(0.5f * z * fmaf(-t, t, 1.f), du, fmaf(0.5f, t, 0.5f));
}

__device__ __forceinline__ uint4 pack8(const float *v) {
  uint4 o;
  __nv_bfloat162 t;
  t = __floats2bfloat162_rn(v[0], v[1]);
  o.x = *reinterpret_cast<uint32_t *>(&t);
  t = __floats2bfloat162_rn(v[2], v[3]);
  o.y = *reinterpret_cast<uint32_t *>(&t);
  t = __floats2bfloat162_rn(v[4], v[5]);
  o.z = *reinterpret_cast<uint32_t *>(&t);
  t = __floats2bfloat162_rn(v[6], v[7]);
  o.w = *reinterpret_cast<uint32_t *>(&t);
  return o;
}
__device__ __forceinline__ void unpack8(uint4 q, float *v) {
  const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    v[2 * i] = __uint_as_float(w[i] << 16);
    v[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
  }
}

// ------------------------------------------------------------ geometry --

struct ConvArgs {
  int P, Pz, B;        // volume pitch (x, y), planes, samples
  int Do;              // output box side
  int s, e, R;         // input offset (0 / -2), extra patch row, patch rows
  int sub;             // 126-output sub-tiles per tile (1 to 4), one plane load each tile
  int tpp;             // tiles per plane: ceil(Do * P / (126 sub))
  int ntiles;          // B * tpp * Do output tiles, z fastest
  int nslot;           // input planes held in the shared-memory ring
  uint32_t slot_bytes;   // one input plane: CI * R * P * 16 (one TMA box)
  uint32_t slot_stride;  // slot_bytes rounded up to 1 KB
  uint32_t w_bytes;      // 27 * CI * CO * 128
  unsigned wait_limit;
  const uint4 *wpack;    // packed weights (B operand), w_bytes
  const float *bias;     // Cout values (forward modes)
  uint4 *out;            // [b][CO][Pz][P^2] x 16 B (FWD_GELU, FWD_LOSS, DGRAD)
  uint4 *zout;           // FWD_GELU: the pre-activation, same layout
  const uint4 *zin;      // DGRAD: the pre-activation of the output's layer
  const float4 *target;  // FWD_LOSS: [b][Pz][P^2][8] floats
  float loss_scale;      // FWD_LOSS: 2 / count
  float *loss_part;      // FWD_LOSS: one partial sum per CTA
  double *infer_out;     // FWD_INFER: 6 arrays of Do^3 values ([z][y][x])
  const float *oscale;   // FWD_INFER: per-component output scale
  int *err;
};

// Forward / transposed convolution, CI input chunks (the GEMM's K, 16
// channels per MMA), CO output chunks.  One MMA covers the three x-taps of
// a (dz, dy) pair: its N = 3 * 8 CO columns are (dx, output channel), so
// D[m][(dx, c)] = sum over (dz, dy, ci) of in[m + x0 + s + (dy + e) P, plane
// z + s + dz][ci] W[dz, dy, dx][c][ci], and the convolution at position m
// is D[m][(0, c)] + D[m + 1][(1, c)] + D[m + 2][(2, c)].  The epilogue forms
// that sum with warp shuffles (rows of a TMEM lane quarter are the lanes
// of one warp) and, for the two rows that cross into the next quarter,
// through shared memory; a tile of 128 rows thus yields TILE_OUT = 126
// outputs and costs 9 CI / 2 MMAs of N = 24 CO instead of 27 CI / 2 of N =
// 8 CO (the tensor core takes about as long for N = 96 as for N = 32).
// Tiles are numbered z fastest (tile = ((b tpp) + j) Do + z) and every CTA
// takes one contiguous range of them, marching up z: the input planes
// z+s .. z+s+2 of a tile sit in a ring of nslot shared-memory slots, so a
// tile loads one new plane (three at the start of a column) and the planes
// are released to the producer after their last use.
template <int CI, int CO, int MODE>
__global__ void __launch_bounds__(CONV_THREADS, 1)
    k_conv(const __grid_constant__ CUtensorMap tin, const ConvArgs a) {
  constexpr int NW = 8 * CO;                            // outputs per position
  constexpr int N = 3 * NW;                             // MMA columns: 96 or 48
  constexpr int NACC = 4;                               // accumulators in flight
  // one epilogue group per accumulator: a group then waits for its
  // accumulator's phases in order, so a parity wait never meets a barrier
  // two phases behind (with fewer groups than accumulators it can)
  static_assert(CONV_GROUPS == NACC, "one epilogue group per accumulator");
  constexpr uint32_t ACC_STRIDE = N <= 64 ? 64 : 128;   // TMEM columns per accumulator
  constexpr uint32_t NCOLS = NACC * ACC_STRIDE;         // 256 or 512 columns
  constexpr int MAXSLOT = 12;
  constexpr int XB = 3 * 2 * NW;                        // exchange floats per group and buffer
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1 KB-aligned base (TMA destinations; the host adds 1 KB of slack)
  unsigned char *smem = smem_raw + ((1024u - (saddr(smem_raw) & 1023u)) & 1023u);
  unsigned char *wsm = smem;
  unsigned char *ring = smem + a.w_bytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(ring + a.nslot * a.slot_stride);
  uint64_t *full = bars, *empty = bars + MAXSLOT, *tfull = bars + 2 * MAXSLOT,
           *tempty = bars + 2 * MAXSLOT + NACC, *wbar = bars + 2 * MAXSLOT + 2 * NACC;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2 * MAXSLOT + 2 * NACC + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 2 * MAXSLOT + 2 * NACC + 2);
  float *lsum = reinterpret_cast<float *>(bars + 2 * MAXSLOT + 2 * NACC + 3);  // 16 floats
  float *bsm = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(bars) + 352);  // 32 biases
  // boundary rows handed between TMEM lane quarters: [group][buffer][quarter
  // 1..3][2][NW] (row 32q's x-shift 2 for lane 30 of the quarter below; row
  // 32q's x-shift 1 + row 32q + 1's x-shift 2 for its lane 31)
  float *xbuf = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(bars) + CONV_BARS);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this CTA's tiles
  const int t0 = (int)((long long)a.ntiles * blockIdx.x / gridDim.x);
  const int t1 = (int)((long long)a.ntiles * (blockIdx.x + 1) / gridDim.x);
  // the next convolution may launch now: its blocks start once this grid's
  // blocks have all started (this grid is one wave: grid_for) and wait for
  // its completion before touching memory
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  if (threadIdx.x == 0) {
    for (int i = 0; i < a.nslot; i++) {
      mb_init(&full[i], 1);
      mb_init(&empty[i], 2);  // released by both issuing lanes
    }
    for (int i = 0; i < NACC; i++) {
      mb_init(&tfull[i], 1);
      mb_init(&tempty[i], 4);
    }
    mb_init(wbar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(tslot, NCOLS);
  // programmatic dependent launch: the barrier set-up and the tensor-memory
  // allocation above overlap the tail of the previous convolution; every
  // read of global memory (biases, weights, input planes, zin, targets) and
  // every write follows the wait (a no-op for an ordinary launch)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (warp == 2) bsm[lane] = MODE != DGRAD && lane < (CO == 4 ? 32 : 6) ? __ldg(a.bias + lane) : 0.f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  const int P2 = a.P * a.P;

  if (warp == 0) {
    if (lane == 0) {
      // weights once, then the input planes of the tiles in order
      mb_expect(wbar, a.w_bytes);
      bulk_load(wsm, a.wpack, a.w_bytes, wbar);
      // one lane runs this loop serially: the tile coordinates and the
      // ring slot advance by increments (no division per plane)
      int g = 0, sl = 0, ph = 0;  // planes issued; slot and phase of the next
      int z = t0 % a.Do, j = (t0 / a.Do) % a.tpp, b = t0 / (a.Do * a.tpp);
      int y0 = (j * a.sub * TILE_OUT) / a.P;
      bool ok = true;
      for (int t = t0; ok && t < t1; t++) {
        const bool fresh = t == t0 || z == 0;
        for (int zp = fresh ? 0 : 2; zp < 3; zp++, g++) {
          if (*abort_flag || !mb_wait(&empty[sl], ph ^ 1, a.wait_limit, abort_flag)) {
            ok = false;
            break;
          }
          mb_expect(&full[sl], a.slot_bytes);
          tma4(ring + sl * a.slot_stride, &tin, 0, y0 + a.s - a.e, z + a.s + zp, b * CI, &full[sl]);
          if (++sl == a.nslot) sl = 0, ph ^= 1;
        }
        if (++z == a.Do) {  // next column of tiles
          z = 0;
          if (++j == a.tpp) j = 0, b++;
          y0 = (j * a.sub * TILE_OUT) / a.P;
        }
      }
      if (!ok) {
        *abort_flag = 1;
        atomicExch(a.err, DEVERR_CNN_TIMEOUT);
      }
      // the copies issued last land before the CTA may leave
      for (int g2 = g - a.nslot < 0 ? 0 : g - a.nslot; g2 < g; g2++)
        mb_wait(&full[g2 % a.nslot], (g2 / a.nslot) & 1, a.wait_limit, abort_flag);
      mb_wait(wbar, 0, a.wait_limit, abort_flag);
    }
  } else if (warp == 1 || warp == 2) {
    if (lane == 0) {
      // Two issuing lanes (warps 1 and 2) take the sub-tiles in turn (sub-tile
      // i on lane i % 2): while one does its waits and bookkeeping, the
      // other's MMAs keep the tensor pipe fed.  Both wait for every plane and
      // both release it (the empty barriers count two arrivals: a commit
      // arrives once that lane's earlier MMAs are done).
      const int r = warp - 1;
      constexpr uint32_t idesc = idesc_bf16(N, false, false);
      // Descriptors are built once; per MMA only the start-address field
      // (bits 0-13, 16-byte units) moves, by an offset added to the whole
      // 64-bit word (starts stay below 256 KB, so the field never carries).
      const uint32_t cstride_u = (uint32_t)a.R * a.P;  // chunk stride in a slot, 16-byte units
      const uint64_t bdesc0 = sdesc(saddr(wsm), 3 * CO * 128u, 128);
      const uint64_t adesc_st = sdesc(0, cstride_u * 16u, 128);  // start 0
      const uint32_t ring_u = saddr(ring) >> 4, stride_u = a.slot_stride >> 4;
      uint32_t yrow[3];  // (dy + e) P, 16-byte units
#pragma unroll
      for (int q = 0; q < 3; q++) yrow[q] = (uint32_t)((q + a.e) * a.P);
      // each lane runs this loop serially: plane slots, tile coordinates and
      // accumulators advance by increments (no division per tile)
      int i = 0, last_a = -1, last_aph = 0;
      int gs = 0, gph = 0;  // slot and phase of the next plane to arrive
      int ac = r, aph = 0;  // accumulator (i % NACC) of this lane's next sub-tile and its phase
      int z = t0 % a.Do, j = (t0 / a.Do) % a.tpp;
      int x0 = (j * a.sub * TILE_OUT) % a.P;  // the tile's first position in patch row y0
      // phases seen complete ahead of their wait, by tests placed among the
      // MMAs (the issue is throttled by the tensor pipe, so the tests cost
      // nothing there): the next accumulator's release, the next plane
      bool acc_ready = false, plane_ready = false;
      bool ok = mb_wait(wbar, 0, a.wait_limit, abort_flag);
      for (int t = t0; ok && t < t1; t++) {
        const bool fresh = t == t0 || z == 0;
        const bool last = t == t1 - 1 || z == a.Do - 1;
        const bool more = t + 1 < t1;
        for (int q = fresh ? 0 : 2; q < 3 && ok; q++) {
          if (!plane_ready) ok = !*abort_flag && mb_wait(&full[gs], gph, a.wait_limit, abort_flag);
          plane_ready = false;
          if (++gs == a.nslot) gs = 0, gph ^= 1;
        }
        if (!ok) break;
        // slots of the last three planes loaded: planes z+s, z+s+1, z+s+2
        int sz[3];
        sz[2] = gs == 0 ? a.nslot - 1 : gs - 1;
        sz[1] = sz[2] == 0 ? a.nslot - 1 : sz[2] - 1;
        sz[0] = sz[1] == 0 ? a.nslot - 1 : sz[1] - 1;
        uint64_t ab[3];
#pragma unroll
        for (int dz = 0; dz < 3; dz++)
          ab[dz] = adesc_st + (uint64_t)(ring_u + (uint32_t)sz[dz] * stride_u + (uint32_t)(x0 + a.s));
        for (int sb = 0; sb < a.sub; sb++, i++) {
          if ((i & 1) != r) continue;
          if (!acc_ready && (*abort_flag || !mb_wait(&tempty[ac], aph ^ 1, a.wait_limit, abort_flag))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t dacc = tbase + (uint32_t)ac * ACC_STRIDE;
          const uint64_t so = (uint64_t)(sb * TILE_OUT);  // the sub-tile's rows, 16-byte units
          const int nac = ac + 2 >= NACC ? ac + 2 - NACC : ac + 2, naph = ac + 2 >= NACC ? aph ^ 1 : aph;
#pragma unroll
          for (int zy = 0; zy < 9; zy++) {
            if (zy == 5) {
              acc_ready = mb_test(&tempty[nac], naph ^ 1);
              if (sb + 2 >= a.sub && more) plane_ready = mb_test(&full[gs], gph);
            }
            const uint64_t at = ab[zy / 3] + so + (uint64_t)yrow[zy % 3];
#pragma unroll
            for (int k = 0; k < CI / 2; k++)
              mma_bf16(dacc, at + (uint64_t)(2 * k) * cstride_u,
                       bdesc0 + (uint64_t)((zy * CI + 2 * k) * 3 * CO * 8), idesc, (zy | k) != 0 ? 1u : 0u);
          }
          mma_commit(&tfull[ac]);
          last_a = ac;
          last_aph = aph;
          ac = nac;
          aph = naph;
        }
        if (!ok) break;
        // release the planes this tile used for the last time
        mma_commit(&empty[sz[0]]);
        if (last) {
          mma_commit(&empty[sz[1]]);
          mma_commit(&empty[sz[2]]);
        }
        if (++z == a.Do) {  // next column of tiles
          z = 0;
          if (++j == a.tpp) j = 0;
          x0 = (j * a.sub * TILE_OUT) % a.P;
        }
      }
      if (!ok) {
        *abort_flag = 1;
        atomicExch(a.err, DEVERR_CNN_TIMEOUT);
      }
      // the MMAs issued last complete before the tensor memory is freed
      if (last_a >= 0) mb_wait(&tfull[last_a], last_aph, a.wait_limit, abort_flag);
    }
  } else {
    // epilogue: CONV_GROUPS groups of 4 warps take the tiles in turn (group
    // e / 4 the tiles with local index i % CONV_GROUPS == e / 4); warp w
    // reads TMEM lanes 32 (w % 4) .. + 31 (rows m = 32 (w % 4) + lane of its
    // tile), 8 columns of each x-shift at a time
    const int e = warp - 3, q = warp & 3, grp = e >> 2;
    const int m = q * 32 + lane;
    const float keep1 = lane < 31 ? 1.f : 0.f, keep2 = lane < 30 ? 1.f : 0.f;
    float osc[6];
#pragma unroll
    for (int k = 0; k < 6; k++) osc[k] = MODE == FWD_INFER ? __ldg(a.oscale + k) : 0.f;
    const bool store_z = a.zout != nullptr;
    float *xg = xbuf + grp * 2 * XB;
    float lacc = 0.f;
    // the tile's (b, j, z) and this thread's positions in its sub-tiles,
    // updated as z marches
    int z = t0 % a.Do, j = (t0 / a.Do) % a.tpp, b = t0 / (a.Do * a.tpp);
    int fA = 0, xA = 0, yA = 0;  // this thread's row in sub-tile 0: offset, x, y
    // a sub-tile further: TILE_OUT = q126 rows of P + r126
    const int q126 = TILE_OUT / a.P, r126 = TILE_OUT - q126 * a.P;
    const long long cstr = (long long)a.Pz * P2;  // one chunk of 8 channels further
    const float4 *bias4 = reinterpret_cast<const float4 *>(bsm);
    bool fresh = true, stop = false;
    int i = 0, own = 0;
    for (int t = t0; t < t1 && !stop; t++) {
      if (fresh) {
        fA = j * a.sub * TILE_OUT + m;
        yA = fA / a.P;
        xA = fA - yA * a.P;
        fresh = false;
      }
      const int zc = z, bc = b;
      if (++z == a.Do) {  // next column
        z = 0;
        fresh = true;
        if (++j == a.tpp) {
          j = 0;
          b++;
        }
      }
      int x = xA, y = yA;
      for (int sb = 0; sb < a.sub; sb++, i++, x += r126, y += q126) {
        if (x >= a.P) x -= a.P, y++;
        const bool mine = (i % CONV_GROUPS) == grp;
        const int ac = i % NACC, aph = (i / NACC) & 1;
        float v[NW];
        if (mine) {
          float *xw = xg + (own & 1) * XB;
          bool ok = !*abort_flag && mb_wait(&tfull[ac], aph, a.wait_limit, abort_flag);
          ok = __all_sync(0xffffffffu, ok);
          if (ok) {
            tc_fence_after();
            const uint32_t ta = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)ac * ACC_STRIDE;
#pragma unroll
            for (int c = 0; c < CO; c++) {
              float d[24];  // columns 8c.. of x-shift 0, 1, 2
              tmem_ld3x8(ta + 8 * c, ta + NW + 8 * c, ta + 2 * NW + 8 * c, d);
              // lane 0: its x-shift 2; lane 1: lane 0's x-shift 1 + its x-shift 2
              float hx[8];
#pragma unroll
              for (int k = 0; k < 8; k++) {
                const float up = __shfl_up_sync(0xffffffffu, d[8 + k], 1);
                hx[k] = lane == 0 ? d[16 + k] : up + d[16 + k];
              }
              if (q > 0 && lane < 2) {
                float4 *xs = reinterpret_cast<float4 *>(xw + 2 * (q - 1) * NW + lane * NW + 8 * c);
                xs[0] = make_float4(hx[0], hx[1], hx[2], hx[3]);
                xs[1] = make_float4(hx[4], hx[5], hx[6], hx[7]);
              }
#pragma unroll
              for (int k = 0; k < 8; k++) {
                const float s1 = __shfl_down_sync(0xffffffffu, d[8 + k], 1);
                const float s2 = __shfl_down_sync(0xffffffffu, d[16 + k], 2);
                v[8 * c + k] = fmaf(s2, keep2, fmaf(s1, keep1, d[k]));
              }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mb_arrive(&tempty[ac]);
          }
          // the group's four warps agree on going on, and the boundary rows
          // written above are visible after this barrier
          if (bar_or(1 + grp, 128, !ok)) {
            *abort_flag = 1;
            atomicExch(a.err, DEVERR_CNN_TIMEOUT);
            stop = true;
            break;
          }
          if (q < 3 && lane >= 30) {
            const float4 *xr = reinterpret_cast<const float4 *>(xw + 2 * q * NW + (lane - 30) * NW);
#pragma unroll
            for (int c = 0; c < NW / 4; c++) {  // quarter q + 1's rows
              const float4 h = xr[c];
              v[4 * c] += h.x;
              v[4 * c + 1] += h.y;
              v[4 * c + 2] += h.z;
              v[4 * c + 3] += h.w;
            }
          }
          own++;
        }
        if (!mine || m >= TILE_OUT) continue;
        const int f = fA + sb * TILE_OUT;
        if (f >= P2) continue;
        const bool valid = x < a.Do && y < a.Do;
        const long long vox = (long long)zc * P2 + f;
        if (MODE == FWD_GELU) {
          const long long o0 = (long long)bc * CO * cstr + vox;
#pragma unroll
          for (int c = 0; c < CO; c++) {
            const float4 b0 = bias4[2 * c], b1 = bias4[2 * c + 1];
            const float bb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
            float zv[8], hv[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
              const float zz = valid ? v[8 * c + k] + bb[k] : 0.f;
              zv[k] = zz;
              hv[k] = gelu_f(zz);
            }
            const long long o = o0 + c * cstr;
            if (store_z) a.zout[o] = pack8(zv);
            a.out[o] = pack8(hv);
          }
        } else if (MODE == FWD_LOSS) {
          // 6 output components in chunk 0 (N = 16: chunk 1 stays zero)
          float tv[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
          if (valid) {
            const float4 *tp = a.target + ((long long)bc * a.Pz * P2 + vox) * 2;
            const float4 t0v = tp[0], t1v = tp[1];
            tv[0] = t0v.x; tv[1] = t0v.y; tv[2] = t0v.z; tv[3] = t0v.w;
            tv[4] = t1v.x; tv[5] = t1v.y;
          }
          float gv[8];
#pragma unroll
          for (int k = 0; k < 8; k++) {
            float g = 0.f;
            if (valid && k < 6) {
              const float d = v[k] + bsm[k] - tv[k];
              lacc += d * d;
              g = a.loss_scale * d;
            }
            gv[k] = g;
          }
          const long long o = ((long long)(bc * CO) * a.Pz) * P2 + vox;
          a.out[o] = pack8(gv);
        } else if (MODE == FWD_INFER) {
          if (valid) {
            const long long n3 = (long long)a.Do * a.Do * a.Do;
            const long long o = ((long long)zc * a.Do + y) * a.Do + x;
#pragma unroll
            for (int k = 0; k < 6; k++) a.infer_out[k * n3 + o] = (double)((v[k] + bsm[k]) * osc[k]);
          }
        } else {  // DGRAD: g = dL/dh * gelu'(z) of the output's layer
#pragma unroll
          for (int c = 0; c < CO; c++) {
            const long long o = ((long long)(bc * CO + c) * a.Pz) * P2 + vox;
            float gv[8];
            if (valid) {
              float zv[8];
              unpack8(a.zin[o], zv);
#pragma unroll
              for (int k = 0; k < 8; k++) gv[k] = v[8 * c + k] * gelu_grad_f(zv[k]);
            } else {
#pragma unroll
              for (int k = 0; k < 8; k++) gv[k] = 0.f;
            }
            a.out[o] = pack8(gv);
          }
        }
      }
    }
    if (MODE == FWD_LOSS) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) lacc += __shfl_xor_sync(0xffffffffu, lacc, o);
      if (lane == 0) lsum[e] = lacc;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (MODE == FWD_LOSS && threadIdx.x == 0) {
    float l = 0.f;
    for (int k = 0; k < 4 * CONV_GROUPS; k++) l += lsum[k];
    a.loss_part[blockIdx.x] = l;
  }
  if (warp == 1) {
    tc_fence_after();
    tmem_free(tbase, NCOLS);
  }
}

// ------------------------------------------------------ weight gradient --

struct WgradArgs {
  int P, Pz, B;     // volume geometry
  int Do;           // output box side (of g)
  int R, KB;        // rows per K-block and its positions R * P (a multiple of 16)
  int stages;       // K-blocks in flight (<= WG_STAGES)
  int kpp;          // K-blocks per plane: ceil(Do / R)
  int nk;           // B * Do * kpp
  int ngroups;      // ceil(27 / G) tap groups
  int nsplit;       // K splits (grid = ngroups * nsplit)
  int ones_slot;    // slot of the last group holding ones (bias row)
  uint32_t a_bytes, stage_bytes;
  unsigned wait_limit;
  float *partial;   // [split][group][128][N]
  int *err;
};

// h: CI chunks (A operand, tap-shifted), g: CO chunks (B operand).
template <int CI, int CO>
__global__ void __launch_bounds__(NTHREADS, 1)
    k_wgrad(const __grid_constant__ CUtensorMap th, const __grid_constant__ CUtensorMap tg,
            const WgradArgs a) {
  constexpr int N = 8 * CO;
  constexpr int G = 16 / CI;             // tap slots per group (M = 128 rows)
  constexpr uint32_t NCOLS = N < 32 ? 32 : N;
  const uint32_t SLOT = (uint32_t)CI * a.KB * 16;  // bytes of one tap slot
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((1024u - (saddr(smem_raw) & 1023u)) & 1023u);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + a.stages * a.stage_bytes);
  uint64_t *full = bars, *empty = bars + WG_STAGES, *done = bars + 2 * WG_STAGES;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2 * WG_STAGES + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 2 * WG_STAGES + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x % a.ngroups, split = blockIdx.x / a.ngroups;
  const int tap0 = grp * G;
  const int ntap = min(G, NTAPS - tap0);
  const bool ones = grp == a.ngroups - 1 && a.ones_slot < G;
  const int k0 = (int)((long long)a.nk * split / a.nsplit);
  const int k1 = (int)((long long)a.nk * (split + 1) / a.nsplit);
  // programmatic dependent launch: dependents may launch once every block
  // of this grid has started; they wait for its completion before memory
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  if (threadIdx.x == 0) {
    for (int i = 0; i < a.stages; i++) {
      mb_init(&full[i], 1);
      mb_init(&empty[i], 1);
    }
    mb_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (ones) {
    // the slot after the last tap: BF16 ones, in every stage, never copied over
    const uint32_t one2 = 0x3F803F80u;
    for (int st = 0; st < a.stages; st++) {
      uint32_t *p = reinterpret_cast<uint32_t *>(smem + st * a.stage_bytes + a.ones_slot * SLOT);
      for (int i = threadIdx.x; i < (int)(SLOT / 4); i += NTHREADS) p[i] = one2;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(tslot, NCOLS);
  // the previous kernel's outputs (activations, gradients) complete and
  // visible past this (a no-op for an ordinary launch)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;

  if (warp == 0) {
    if (lane == 0) {
      const uint32_t bytes = (uint32_t)ntap * SLOT + (uint32_t)CO * a.KB * 16;
      int i = 0, issued = 0;
      for (int k = k0; k < k1; k++, i++) {
        const int s = i % a.stages, ph = (i / a.stages) & 1;
        if (*abort_flag || !mb_wait(&empty[s], ph ^ 1, a.wait_limit, abort_flag)) {
          *abort_flag = 1;
          atomicExch(a.err, DEVERR_CNN_TIMEOUT);
          break;
        }
        const int jb = k % a.kpp, rest = k / a.kpp;
        const int z = rest % a.Do, b = rest / a.Do;
        const int y0 = jb * a.R;
        unsigned char *st = smem + s * a.stage_bytes;
        mb_expect(&full[s], bytes);
        // R whole rows per box; a tap's x shift runs past the row end into
        // zeros, where g (zero outside its output box) takes nothing
        for (int j = 0; j < ntap; j++) {
          const int tap = tap0 + j;
          const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
          tma4(st + j * SLOT, &th, 2 * dx, y0 + dy, z + dz, b * CI, &full[s]);
        }
        tma4(st + a.a_bytes, &tg, 0, y0, z, b * CO, &full[s]);
        issued = i + 1;
      }
      // let the last copies of every stage land before leaving
      for (int i2 = issued - a.stages < 0 ? 0 : issued - a.stages; i2 < issued; i2++)
        mb_wait(&full[i2 % a.stages], (i2 / a.stages) & 1, a.wait_limit, abort_flag);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16(N, true, true);
      int i = 0;
      bool ok = true, any = false;
      for (int k = k0; k < k1; k++, i++) {
        const int s = i % a.stages, ph = (i / a.stages) & 1;
        if (*abort_flag || !mb_wait(&full[s], ph, a.wait_limit, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = saddr(smem + s * a.stage_bytes);
        const uint32_t sb = sa + a.a_bytes;
        const int nkk = a.KB / 16;
        for (int kk = 0; kk < nkk; kk++) {
          // MN-major, no swizzle: SBO = stride of 8-element MN groups (one
          // chunk's K-block, 16 KB bytes), LBO = stride of 8-row K groups (128 B)
          const uint64_t ad = sdesc(sa + kk * 256, 128, (uint32_t)a.KB * 16);
          const uint64_t bd = sdesc(sb + kk * 256, 128, (uint32_t)a.KB * 16);
          mma_bf16(tbase, ad, bd, idesc, (i | kk) != 0);
        }
        mma_commit(&empty[s]);
        any = true;
      }
      if (!ok) {
        *abort_flag = 1;
        atomicExch(a.err, DEVERR_CNN_TIMEOUT);
      }
      if (any) mma_commit(done);
      else mb_arrive(done);
    }
  } else {
    const int q = warp & 3;
    const int m = q * 32 + lane;
    const bool ok = mb_wait(done, 0, a.wait_limit, abort_flag) && !*abort_flag;
    if (!ok) {
      *abort_flag = 1;
      atomicExch(a.err, DEVERR_CNN_TIMEOUT);
    }
    tc_fence_after();
    float v[N];
    tmem_ld<N>(tbase + ((uint32_t)(q * 32) << 16), v);
    float *dst = a.partial + (((long long)split * a.ngroups + grp) * 128 + m) * N;
    const bool empty_range = k1 <= k0;
#pragma unroll
    for (int c = 0; c < N; c += 4)
      *reinterpret_cast<float4 *>(dst + c) =
          empty_range || !ok ? make_float4(0.f, 0.f, 0.f, 0.f)
                             : make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_free(tbase, NCOLS);
  }
}

}  // namespace cnn
}  // namespace dnsb
