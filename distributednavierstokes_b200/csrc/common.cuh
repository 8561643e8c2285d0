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

__host__ __device__ __forceinline__ long long gidx(const Geo &g, int I, int J, int K) {
  return (long long)I + (long long)g.NX * ((long long)J + (long long)g.NY * (long long)K);
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
struct Img {
  int n;
  int pos[3];
  double sgn[3];
};

__device__ __forceinline__ void img_periodic(Img &m, int I, int n) {
  m.n = 1;
  m.pos[0] = I;
  m.sgn[0] = 1.0;
  if (I == 1) { m.pos[m.n] = n + 1; m.sgn[m.n++] = 1.0; }
  if (I == n) { m.pos[m.n] = 0; m.sgn[m.n++] = 1.0; }
}

// y images; a sign of 0 marks a wall face that receives an exact zero
__device__ __forceinline__ void img_y(Img &m, const Geo &g, int J, int stag) {
  if (!g.wall) { img_periodic(m, J, g.ny); return; }
  m.n = 1;
  m.pos[0] = J;
  m.sgn[0] = 1.0;
  if (stag == STAG_Y) {
    if (J == 1) { m.pos[m.n] = 0; m.sgn[m.n++] = 0.0; }
    if (J == g.ny - 1) {
      m.pos[m.n] = g.ny; m.sgn[m.n++] = 0.0;
      m.pos[m.n] = g.ny + 1; m.sgn[m.n++] = -1.0;
    }
  } else {
    double s = stag == STAG_P ? 1.0 : -1.0;
    if (J == 1) { m.pos[m.n] = 0; m.sgn[m.n++] = s; }
    if (J == g.ny) { m.pos[m.n] = g.ny + 1; m.sgn[m.n++] = s; }
  }
}

// Ghost images only (not the interior cell itself); the slow path of
// store_img, kept out of line so that interior threads carry no image
// bookkeeping.
__device__ __noinline__ void store_images_only(double *__restrict__ f, const Geo &g, int I, int J,
                                               int K, double v, int stag) {
  Img mx, my, mz;
  img_periodic(mx, I, g.nx);
  img_y(my, g, J, stag);
  img_periodic(mz, K, g.nz);
  for (int c = 0; c < mz.n; c++)
    for (int b = 0; b < my.n; b++) {
      double vv = my.sgn[b] == 0.0 ? 0.0 : my.sgn[b] * v;
      for (int a = 0; a < mx.n; a++)
        if (a | b | c) f[gidx(g, mx.pos[a], my.pos[b], mz.pos[c])] = vv;
    }
}

// Store v at interior (I, J, K) and at all its ghost images.
__device__ __forceinline__ void store_img(double *__restrict__ f, const Geo &g, int I, int J,
                                          int K, double v, int stag) {
  f[gidx(g, I, J, K)] = v;
  const bool edge = (I == 1) | (I == g.nx) | (K == 1) | (K == g.nz) | (J == 1) | (J >= g.ny - 1);
  if (edge) store_images_only(f, g, I, J, K, v, stag);
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
