// common.cuh -- geometry descriptor, ghosted indexing and ghost images.
//
// Field layout (the reference's `scalarfield`, src/fields.jl:4-5): ghosted
// (nx+2) x (ny+2) x (nz+2) doubles, column-major (x fastest), ghost width 1.
// C index I equals the reference's cell index i: interior I = 1..nx, ghosts
// I = 0 and nx+1 (likewise J, K).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dnsb {

enum Stag { STAG_X = 0, STAG_Y = 1, STAG_Z = 2, STAG_P = 3 };

struct Fields3 {
  double *x, *y, *z;
};
struct CFields3 {
  const double *x, *y, *z;
};

struct Geo {
  int nx, ny, nz;       // interior cells
  int NX, NY, NZ;       // ghosted extents
  int wall;             // bc[2] == :wall
  int jymax;            // last active u.y row (ny-1 walls, ny periodic)
  int nkx;              // nx/2 + 1
  double dx, dz, rdx, rdz, rdx2, rdz2;
  double visc, fx, fy, fz, epsy;
  const double *dy, *dyu, *rdy, *rdyu;  // device, ny+2 entries (ghosted J)
};

// Linear index of ghosted cell (I, J, K).  32-bit: a context refuses grids
// whose ghosted field reaches 2^31 values, so offsets stay in one IMAD.
__host__ __device__ __forceinline__ int gidx(const Geo &g, int I, int J, int K) {
  return I + g.NX * (J + g.NY * K);
}

// Spectrum layout: S[kz + nz*(j + ny*kx)] (kz fastest, then y, kx slowest),
// so z-lines are contiguous, y-lines are kz-coalesced and one kx-plane is a
// contiguous block.
__host__ __device__ __forceinline__ long long sidx(const Geo &g, int kx, int j, int kz) {
  return (long long)kz + (long long)g.nz * ((long long)j + (long long)g.ny * (long long)kx);
}

// Ghost images of an interior value, i.e. the ghost cells that the
// reference's single-rank exchange_halo! (src/halo.jl:81-126, fill_wall!
// :26-45) fills from interior cell (I, J, K): periodic wraps in x and z
// (and y when periodic); at walls a mirror with sign -1 (tangential),
// +1 (pressure), and for the wall-normal component zero wall faces
// (J = 0, J = ny) plus the antisymmetric ghost J = ny+1 <- -(J = ny-1).
// Writing v to every image after writing the interior keeps the halo of a
// field valid without a separate exchange pass; the x, y and z fills of the
// reference compose into exactly this product of per-axis images.
// Interior threads only test the edge predicate; edge threads run
// straight-line predicated stores (no local memory).
// The images alone (no interior store), from the grid extents passed by
// value so that no caller has to spill its Geo to local memory.
__device__ __forceinline__ void store_images_core(double *__restrict__ f, int nx, int ny, int nz,
                                                  int NX, int NY, int wall, int I, int J, int K,
                                                  double v, int stag) {
  const int Ia = (I == 1) ? nx + 1 : (I == nx) ? 0 : -1;  // nx >= 2: at most one
  const int Ka = (K == 1) ? nz + 1 : (K == nz) ? 0 : -1;
  const int Kb = (K == 1 && K == nz) ? 0 : -1;             // nz == 1
  int Ja = -1, Jb = -1, Jc = -1;
  double fa = 0.0, fb = 0.0, fc = 0.0;
  if (!wall) {
    Ja = (J == 1) ? ny + 1 : (J == ny) ? 0 : -1;
    fa = 1.0;
  } else if (stag == STAG_Y) {
    if (J == 1) { Ja = 0; fa = 0.0; }
    if (J == ny - 1) { Jb = ny; fb = 0.0; Jc = ny + 1; fc = -1.0; }
  } else {
    const double s = stag == STAG_P ? 1.0 : -1.0;
    if (J == 1) { Ja = 0; fa = s; }
    if (J == ny) { Jb = ny + 1; fb = s; }
  }
#pragma unroll
  for (int zc = 0; zc < 3; zc++) {
    const int Kz = zc == 0 ? K : zc == 1 ? Ka : Kb;
    if (Kz < 0) continue;
#pragma unroll
    for (int yc = 0; yc < 4; yc++) {
      const int Jy = yc == 0 ? J : yc == 1 ? Ja : yc == 2 ? Jb : Jc;
      if (Jy < 0) continue;
      const double fy = yc == 0 ? 1.0 : yc == 1 ? fa : yc == 2 ? fb : fc;
      const double vv = fy == 0.0 ? 0.0 : fy * v;
#pragma unroll
      for (int xc = 0; xc < 2; xc++) {
        const int Ix = xc == 0 ? I : Ia;
        if (Ix < 0 || (xc == 0 && yc == 0 && zc == 0)) continue;
        f[Ix + NX * (Jy + NY * Kz)] = vv;
      }
    }
  }
}

__device__ __forceinline__ bool img_edge(const Geo &g, int I, int J, int K) {
  return (I == 1) | (I == g.nx) | (K == 1) | (K == g.nz) | (J == 1) | (J >= g.ny - 1);
}

__device__ __forceinline__ void store_img(double *__restrict__ f, const Geo &g, int I, int J,
                                          int K, double v, int stag) {
  f[gidx(g, I, J, K)] = v;
  if (!img_edge(g, I, J, K)) return;
  store_images_core(f, g.nx, g.ny, g.nz, g.NX, g.NY, g.wall, I, J, K, v, stag);
}

// Out-of-line images for callers that write the interior value themselves
// and only need the ghost images of edge cells (keeps unrolled loops small).
__device__ __noinline__ void store_images_of(double *__restrict__ f, int nx, int ny, int nz,
                                             int NX, int NY, int wall, int I, int J, int K,
                                             double v, int stag) {
  store_images_core(f, nx, ny, nz, NX, NY, wall, I, J, K, v, stag);
}

// Cooperative copy loop with B loads in flight per thread: element t of
// [0, total) is read with ld(t) and written with st(t, value).  All B loads
// of a batch are issued before the first store, so a thread keeps B
// requests outstanding instead of one.
template <int B, class Ld, class St>
__device__ __forceinline__ void batched_copy(int total, Ld ld, St st) {
  const int nth = blockDim.x * blockDim.y;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  for (int base = tid; base < total; base += B * nth) {
    decltype(ld(0)) r[B];
#pragma unroll
    for (int u = 0; u < B; u++) {
      const int t = base + u * nth;
      if (t < total) r[u] = ld(t);
    }
#pragma unroll
    for (int u = 0; u < B; u++) {
      const int t = base + u * nth;
      if (t < total) st(t, r[u]);
    }
  }
}

// Interior source of a ghost cell (inverse of the image map); returns false
// when the cell holds an exact zero (wall face of the normal component).
__device__ __forceinline__ bool ghost_src(const Geo &g, int stag, int &I, int &J, int &K,
                                          double &s) {
  s = 1.0;
  if (I == 0) I = g.nx; else if (I == g.nx + 1) I = 1;
  if (K == 0) K = g.nz; else if (K == g.nz + 1) K = 1;
  if (!g.wall) {
    if (J == 0) J = g.ny; else if (J == g.ny + 1) J = 1;
    return true;
  }
  if (stag == STAG_Y) {
    if (J == 0 || J == g.ny) return false;
    if (J == g.ny + 1) { J = g.ny - 1; s = -1.0; }
    return true;
  }
  double sg = stag == STAG_P ? 1.0 : -1.0;
  if (J == 0) { J = 1; s = sg; }
  else if (J == g.ny + 1) { J = g.ny; s = sg; }
  return true;
}

}  // namespace dnsb
