// gradmom.cuh -- the projection of one semi-implicit RK3 stage fused with
// the momentum of the next.
//
// Between stages s and s+1 of step! (src/timestep.jl:41-63) with implicit
// y-diffusion, the reference runs
//   pressuregrad!/project: u = u* - grad delta, p += delta / (alpha_s dt)
//                          (timestep.jl:49-52, operators.jl:180-220)
//   momentum! + imex_update! of stage s+1 (operators.jl:44-145,
//                          ydiffusion.jl:71-154)
// and u after the projection is read by nothing but that momentum (the
// Crank-Nicolson solve of stage s+1 overwrites it).  k_gradmom_march
// therefore never stores it: it stages u*, delta and p in shared memory
// plane by plane (the z-marching scheme of k_momentum_march), rebuilds
// u = u* - grad delta on the CTA's tile and its one-cell halo, and feeds the
// momentum arithmetic from there; p + delta / (alpha_s dt) is formed where
// it is read.  Halo cells outside the interior are the ghost images of
// exchange_halo! (halo.jl:26-45,81-126): periodic images follow from the
// images already held by u* and delta (one more period is read for the
// gradient at the last ghost layer), wall images mirror interior rows.
#pragma once
#include <cuda.h>
#include "common.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace dnsb {

// Raw planes are staged as GP_X x GP_Y boxes starting at (I0-1, J0-1): one
// halo cell on the low sides, two on the high sides (the gradient of the
// last halo cell reads one further cell); rows of 18 aligned 16-byte chunks.
constexpr int GP_X = MC_X + 4, GP_Y = MC_Y + 3, GP_N = GP_X * GP_Y;

// Projection fused with the next stage's momentum (implicit y-diffusion).
// Reads u* (ux, uy, uz after the Crank-Nicolson solve of stage s), delta,
// p_in (lagged pressure before stage s's update), q; writes p_out =
// p_in + delta * radt on the interior with ghost images, q, and V (the
// Crank-Nicolson right-hand side of stage s+1, as k_momentum<IMPLICIT>);
// each CTA walks `planes` z-planes (grid z = ceil(nz / planes)).
// p_out must not alias p_in (other CTAs stage p_in while this one writes).
// 3 CTAs of 256 per SM (80 registers, no spills; faster than 2)
__global__ void __launch_bounds__(MC_X *MC_Y, 3)
    k_gradmom_march(Geo g, int planes, CFields3 us, const double *__restrict__ delta,
                    const double *__restrict__ p_in, double *__restrict__ p_out, double radt,
                    Fields3 q, Fields3 out, double A, double dt, double B, double adt,
                    const double2 *__restrict__ ymet, double theta) {
  extern __shared__ __align__(16) double gsm[];
  double *ustar = gsm;                    // [2 slots][3][GP_N]   u* (one plane ahead)
  double *pold = ustar + 2 * 3 * GP_N;    // [3 slots][GP_N]      p_in
  double *dl = pold + 3 * GP_N;           // [4 slots][GP_N]      delta
  double *unew = dl + 4 * GP_N;           // [3 slots][3][GP_N]   projected u
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + MC_X * ty;
  constexpr int NT = MC_X * MC_Y;
  const int I0 = blockIdx.x * MC_X + 1, J0 = blockIdx.y * MC_Y + 1;
  const int K0 = blockIdx.z * planes + 1, K1 = min(g.nz, K0 + planes - 1);
  const bool wall = g.wall;
  constexpr int CH = GP_X / 2;
  static_assert(GP_Y * CH <= NT, "one staging chunk per thread and field plane");
  // This thread's 16-byte chunk of every staged GP_X x GP_Y box: the same
  // in-plane offsets for every plane and field.  x and y beyond the ghosted
  // array wrap by one period (periodic directions; wall rows there are never
  // read).
  const long long plane = (long long)g.NX * g.NY;
  bool stage = tid < GP_Y * CH;
  int goff = 0, soff = 0;
  if (stage) {
    const int ch = tid % CH, hy = tid / CH;
    int x = I0 - 1 + 2 * ch, y = J0 - 1 + hy;
    if (x >= g.NX) x -= g.nx;
    if (y >= g.NY) {
      if (wall) stage = false;
      y -= g.ny;
    }
    // on grids narrower than the box, columns/rows still beyond the array
    // after one wrap are never read by an interior cell: not copied
    if (x + 1 >= g.NX || y >= g.NY) stage = false;
    goff = x + g.NX * y;
    soff = 2 * ch + GP_X * hy;
  }
  // the box of field f at plane z (z beyond the array wraps, z is periodic)
  auto box = [&](const double *f, int z, double *dst) {
    if (z >= g.NZ) z -= g.nz;
    if (stage) cp_async16(dst + soff, f + (plane * z + goff));
  };
  auto us_slot = [&](int z) { return ustar + (z & 1) * 3 * GP_N; };
  auto p_slot = [&](int z) { return pold + (z % 3) * GP_N; };
  auto d_slot = [&](int z) { return dl + (z & 3) * GP_N; };
  auto un_slot = [&](int z) { return unew + (z % 3) * 3 * GP_N; };
  auto issue_us = [&](int z) {
    double *s = us_slot(z);
    box(us.x, z, s);
    box(us.y, z, s + GP_N);
    box(us.z, z, s + 2 * GP_N);
  };
  // Per-CTA row map of the projected tile (the same for every plane): row hy
  // of component c holds sgn * (value of staged row src); sgn = 0 for the
  // zero wall faces and for rows beyond the ghosted array; rg = the
  // y-metric of the gradient of the y component at that row.
  constexpr int HX = MC_X + 2, HY = MC_Y + 2;
  __shared__ int rsrc[3][HY];
  __shared__ double rsgn[3][HY], rg[HY];
  if (tid < 3 * HY) {
    const int c = tid / HY, hy = tid - c * HY;
    const int y = J0 - 1 + hy;
    int hs = hy;
    double sgn = y <= g.NY - 1 ? 1.0 : 0.0;
    if (wall && sgn != 0.0) {
      if (c == STAG_Y) {
        if (y == 0 || y == g.ny) sgn = 0.0;                   // wall faces
        else if (y == g.ny + 1) { hs = hy - 2; sgn = -1.0; }  // -(ny-1)
      } else {
        if (y == 0) { hs = 1; sgn = -1.0; }                   // -(1)
        else if (y == g.ny + 1) { hs = hy - 1; sgn = -1.0; }  // -(ny)
      }
    }
    rsrc[c][hy] = hs;
    rsgn[c][hy] = sgn;
    if (c == STAG_Y) rg[hy] = sgn != 0.0 ? __ldg(g.rdyu + (J0 - 1 + hs)) : 0.0;
  }
  // projected u of plane z on the HX x HY tile + halo, from u* of plane z
  // and delta of planes z, z+1 (all staged); thread (tx, ty) covers columns
  // tx, tx + MC_X and rows ty, ty + MC_Y of each component
  // CTAs away from the walls take every row as it is (no row map)
  const bool plain = wall ? (J0 >= 2 && J0 + MC_Y <= g.ny - 1) : (J0 + MC_Y <= g.ny + 1);
  auto project_plane = [&](int z, double *dst) {
    const double *su = us_slot(z), *d0 = d_slot(z), *d1 = d_slot(z + 1);
#pragma unroll
    for (int c = 0; c < 3; c++) {
#pragma unroll
      for (int ry = 0; ry < 2; ry++) {
        const int hy = ty + ry * MC_Y;
        if (hy >= HY) continue;
        const int srow = GP_X * (plain ? hy : rsrc[c][hy]);
        const double sgn = plain ? 1.0 : rsgn[c][hy];
        const double gy = c == STAG_Y ? rg[hy] : 0.0;
#pragma unroll
        for (int rx = 0; rx < 2; rx++) {
          const int hx = tx + rx * MC_X;
          if (hx >= HX) continue;
          const int a = hx + srow;
          double v;
          if (c == STAG_X) v = su[a] - (d0[a + 1] - d0[a]) * g.rdx;
          else if (c == STAG_Y) v = su[GP_N + a] - (d0[a + GP_X] - d0[a]) * gy;
          else v = su[2 * GP_N + a] - (d1[a] - d0[a]) * g.rdz;
          dst[c * GP_N + hx + GP_X * hy] = plain ? v : sgn * v;
        }
      }
    }
  };
  // prologue: u* of K0-1, K0; p of K0; delta of K0-1, K0, K0+1
  issue_us(K0 - 1);
  box(delta, K0 - 1, d_slot(K0 - 1));
  box(delta, K0, d_slot(K0));
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  // ring slots, rotated once per plane
  double *un_prev = un_slot(K0 - 1), *un_cur = un_slot(K0), *un_next = un_slot(K0 + 1);
  double *p_cur = p_slot(K0), *p_next = p_slot(K0 + 1), *p_nn = p_slot(K0 + 2);
  project_plane(K0 - 1, un_prev);
  __syncthreads();  // u* slot of K0-1 is reused by K0+1 below
  issue_us(K0);
  box(delta, K0 + 1, d_slot(K0 + 1));
  box(p_in, K0, p_cur);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  project_plane(K0, un_cur);
  // plane K+1's raw data for the first iteration
  issue_us(K0 + 1);
  box(p_in, K0 + 1, p_next);
  box(delta, K0 + 2, d_slot(K0 + 2));
  cp_async_commit();
  const int I = I0 + tx, J = J0 + ty;
  const bool inside = I <= g.nx && J <= g.ny;
  constexpr int SY = GP_X;
  const int h = (tx + 1) + SY * (ty + 1);
  for (int K = K0; K <= K1; K++) {
    MomNb nb;
    const int c0 = gidx(g, inside ? I : 1, inside ? J : 1, K);
    nb.qx0 = inside ? q.x[c0] : 0.0;
    nb.qy0 = inside ? q.y[c0] : 0.0;
    nb.qz0 = inside ? q.z[c0] : 0.0;
    cp_async_wait<0>();  // u*, p of K+1 and delta of K+2 have landed
    __syncthreads();     // ... for every thread; plane K-1's raw slots are free
    project_plane(K + 1, un_next);
    if (K + 1 <= K1) {   // raw data of plane K+2 for the next iteration
      issue_us(K + 2);
      box(p_in, K + 2, p_nn);
      box(delta, K + 3, d_slot(K + 3));
    }
    cp_async_commit();
    __syncthreads();     // projected plane K+1 complete
    if (inside) {
      const double *pk = p_cur + h, *pk1 = p_next + h;
      const double *dk = d_slot(K) + h, *dk1 = d_slot(K + 1) + h;
      nb.p0 = pk[0] + dk[0] * radt;
      nb.pE = pk[1] + dk[1] * radt;
      nb.pN = pk[SY] + dk[SY] * radt;
      nb.pT = pk1[0] + dk1[0] * radt;
      const double *ub = un_prev + h, *uc = un_cur + h, *ut = un_next + h;
      const double *bx = ub, *cx = uc, *tx_ = ut;
      const double *by = ub + GP_N, *cy = uc + GP_N, *ty_ = ut + GP_N;
      const double *bz = ub + 2 * GP_N, *cz = uc + 2 * GP_N, *tz_ = ut + 2 * GP_N;
      nb.ux0 = cx[0]; nb.uxE = cx[1]; nb.uxW = cx[-1]; nb.uxN = cx[SY]; nb.uxS = cx[-SY];
      nb.uxT = tx_[0]; nb.uxB = bx[0]; nb.uxWN = cx[SY - 1]; nb.uxWT = tx_[-1];
      nb.uy0 = cy[0]; nb.uyE = cy[1]; nb.uyW = cy[-1]; nb.uyN = cy[SY]; nb.uyS = cy[-SY];
      nb.uyT = ty_[0]; nb.uyB = by[0]; nb.uySE = cy[1 - SY]; nb.uyST = ty_[-SY];
      nb.uz0 = cz[0]; nb.uzE = cz[1]; nb.uzW = cz[-1]; nb.uzN = cz[SY]; nb.uzS = cz[-SY];
      nb.uzT = tz_[0]; nb.uzB = bz[0]; nb.uzEB = bz[1]; nb.uzNB = bz[SY];
      const MomCell m = mom_compute<MOM_IMPLICIT>(g, J, nb, A, dt, B, adt, 1, ymet, theta);
      mom_store<MOM_IMPLICIT>(g, I, J, K, m, q, out);
      store_img(p_out, g, I, J, K, nb.p0, STAG_P);
    }
    double *t = un_prev;
    un_prev = un_cur;
    un_cur = un_next;
    un_next = t;
    t = p_cur;
    p_cur = p_next;
    p_next = p_nn;
    p_nn = t;
  }
  cp_async_wait<0>();
}

// Dynamic shared memory of k_gradmom_march.
constexpr size_t GRADMOM_SMEM = sizeof(double) * (2 * 3 + 3 + 4 + 3 * 3) * GP_N;

// k_gradmom_pipe: k_gradmom_march with the projection one plane further
// ahead, so that one barrier per plane separates the phases instead of two.
// Iteration K projects plane K+2 and computes the momentum of plane K, which
// reads only planes K and K+1 (projected in earlier iterations) from shared
// memory; the five values of plane K-1 it needs (u_x, u_y, u_z at the cell,
// u_z east and north) are the ones this thread read as plane K's centre in
// the previous iteration and stay in registers.  Ring slots: u* 2, p 3,
// delta 5, projected u 3 (x 3 components).
__global__ void __launch_bounds__(MC_X *MC_Y, 3)
    k_gradmom_pipe(Geo g, int planes, CFields3 us, const double *__restrict__ delta,
                   const double *__restrict__ p_in, double *__restrict__ p_out, double radt,
                   Fields3 q, Fields3 out, double A, double dt, double B, double adt,
                   const double2 *__restrict__ ymet, double theta) {
  extern __shared__ __align__(16) double gsm[];
  double *ustar = gsm;                    // [2 slots][3][GP_N]
  double *pold = ustar + 2 * 3 * GP_N;    // [3 slots][GP_N]
  double *dl = pold + 3 * GP_N;           // [5 slots][GP_N]
  double *unew = dl + 5 * GP_N;           // [3 slots][3][GP_N]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + MC_X * ty;
  const int I0 = blockIdx.x * MC_X + 1, J0 = blockIdx.y * MC_Y + 1;
  const int K0 = blockIdx.z * planes + 1, K1 = min(g.nz, K0 + planes - 1);
  const bool wall = g.wall;
  constexpr int CH = GP_X / 2;
  const long long plane = (long long)g.NX * g.NY;
  bool stage = tid < GP_Y * CH;
  int goff = 0, soff = 0;
  if (stage) {
    const int ch = tid % CH, hy = tid / CH;
    int x = I0 - 1 + 2 * ch, y = J0 - 1 + hy;
    if (x >= g.NX) x -= g.nx;
    if (y >= g.NY) {
      if (wall) stage = false;
      y -= g.ny;
    }
    if (x + 1 >= g.NX || y >= g.NY) stage = false;
    goff = x + g.NX * y;
    soff = 2 * ch + GP_X * hy;
  }
  auto box = [&](const double *f, int z, double *dst) {
    if (z >= g.NZ) z -= g.nz;
    if (stage) cp_async16(dst + soff, f + (plane * z + goff));
  };
  auto us_slot = [&](int z) { return ustar + (z & 1) * 3 * GP_N; };
  auto issue_us = [&](int z) {
    double *s = us_slot(z);
    box(us.x, z, s);
    box(us.y, z, s + GP_N);
    box(us.z, z, s + 2 * GP_N);
  };
  constexpr int HX = MC_X + 2, HY = MC_Y + 2;
  __shared__ int rsrc[3][HY];
  __shared__ double rsgn[3][HY], rg[HY];
  if (tid < 3 * HY) {
    const int c = tid / HY, hy = tid - c * HY;
    const int y = J0 - 1 + hy;
    int hs = hy;
    double sgn = y <= g.NY - 1 ? 1.0 : 0.0;
    if (wall && sgn != 0.0) {
      if (c == STAG_Y) {
        if (y == 0 || y == g.ny) sgn = 0.0;
        else if (y == g.ny + 1) { hs = hy - 2; sgn = -1.0; }
      } else {
        if (y == 0) { hs = 1; sgn = -1.0; }
        else if (y == g.ny + 1) { hs = hy - 1; sgn = -1.0; }
      }
    }
    rsrc[c][hy] = hs;
    rsgn[c][hy] = sgn;
    if (c == STAG_Y) rg[hy] = sgn != 0.0 ? __ldg(g.rdyu + (J0 - 1 + hs)) : 0.0;
  }
  const bool plain = wall ? (J0 >= 2 && J0 + MC_Y <= g.ny - 1) : (J0 + MC_Y <= g.ny + 1);
  // projected u of one plane from its u* and delta of it and the plane above
  auto project_plane = [&](const double *su, const double *d0, const double *d1, double *dst) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
#pragma unroll
      for (int ry = 0; ry < 2; ry++) {
        const int hy = ty + ry * MC_Y;
        if (hy >= HY) continue;
        const int srow = GP_X * (plain ? hy : rsrc[c][hy]);
        const double sgn = plain ? 1.0 : rsgn[c][hy];
        const double gy = c == STAG_Y ? rg[hy] : 0.0;
#pragma unroll
        for (int rx = 0; rx < 2; rx++) {
          const int hx = tx + rx * MC_X;
          if (hx >= HX) continue;
          const int a = hx + srow;
          double v;
          if (c == STAG_X) v = su[a] - (d0[a + 1] - d0[a]) * g.rdx;
          else if (c == STAG_Y) v = su[GP_N + a] - (d0[a + GP_X] - d0[a]) * gy;
          else v = su[2 * GP_N + a] - (d1[a] - d0[a]) * g.rdz;
          dst[c * GP_N + hx + GP_X * hy] = plain ? v : sgn * v;
        }
      }
    }
  };
  // rotating slots: d[i] holds delta of plane K+i (i = 0..4), un_* the
  // projected planes K, K+1, K+2, p_* the lagged pressure of K, K+1, K+2
  double *d[5] = {dl, dl + GP_N, dl + 2 * GP_N, dl + 3 * GP_N, dl + 4 * GP_N};
  double *dm1 = d[4];  // delta of K0-1 in the slot that K0+4 takes later
  double *un_cur = unew, *un_next = unew + 3 * GP_N, *un_new = unew + 6 * GP_N;
  double *un_m1 = un_new;  // plane K0-1 in the slot that K0+2 takes later
  double *p_cur = pold, *p_next = pold + GP_N, *p_nn = pold + 2 * GP_N;
  // prologue: project K0-1, K0, K0+1; raw data of K0+2 in flight
  issue_us(K0 - 1);
  box(delta, K0 - 1, dm1);
  box(delta, K0, d[0]);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  project_plane(us_slot(K0 - 1), dm1, d[0], un_m1);
  issue_us(K0);
  box(delta, K0 + 1, d[1]);
  box(p_in, K0, p_cur);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();     // u* of K0 and delta of K0+1 landed; slot of u* K0-1 free after this
  project_plane(us_slot(K0), d[0], d[1], un_cur);
  __syncthreads();     // every thread is done with u* of K0-1
  issue_us(K0 + 1);
  box(delta, K0 + 2, d[2]);
  box(p_in, K0 + 1, p_next);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  project_plane(us_slot(K0 + 1), d[1], d[2], un_next);
  __syncthreads();     // projected K0-1, K0, K0+1 complete; u* of K0 free
  const int I = I0 + tx, J = J0 + ty;
  const bool inside = I <= g.nx && J <= g.ny;
  constexpr int SY = GP_X;
  const int h = (tx + 1) + SY * (ty + 1);
  // plane K0-1 as seen from the first cell: centre values and u_z east/north
  double bx0 = un_m1[h], by0 = un_m1[GP_N + h], bz0 = un_m1[2 * GP_N + h];
  double bzE = un_m1[2 * GP_N + h + 1], bzN = un_m1[2 * GP_N + h + SY];
  if (K0 + 1 <= K1) {
    issue_us(K0 + 2);
    box(delta, K0 + 3, d[3]);
  }
  cp_async_commit();
  for (int K = K0; K <= K1; K++) {
    MomNb nb;
    const int c0 = gidx(g, inside ? I : 1, inside ? J : 1, K);
    nb.qx0 = inside ? q.x[c0] : 0.0;
    nb.qy0 = inside ? q.y[c0] : 0.0;
    nb.qz0 = inside ? q.z[c0] : 0.0;
    cp_async_wait<0>();  // u* of K+2, delta of K+3, p of K+1 have landed
    __syncthreads();     // ... for every thread; projected K+1 complete; slots of K-1 free
    if (K + 1 <= K1) {
      project_plane(us_slot(K + 2), d[2], d[3], un_new);
      if (K + 2 <= K1) {   // raw data of the next iteration's projection
        issue_us(K + 3);
        box(delta, K + 4, d[4]);
      }
      box(p_in, K + 2, p_nn);
    }
    cp_async_commit();
    if (inside) {
      const double *pk = p_cur + h, *pk1 = p_next + h;
      const double *dk = d[0] + h, *dk1 = d[1] + h;
      nb.p0 = pk[0] + dk[0] * radt;
      nb.pE = pk[1] + dk[1] * radt;
      nb.pN = pk[SY] + dk[SY] * radt;
      nb.pT = pk1[0] + dk1[0] * radt;
      const double *cx = un_cur + h, *tx_ = un_next + h;
      const double *cy = cx + GP_N, *ty_ = tx_ + GP_N;
      const double *cz = cx + 2 * GP_N, *tz_ = tx_ + 2 * GP_N;
      nb.ux0 = cx[0]; nb.uxE = cx[1]; nb.uxW = cx[-1]; nb.uxN = cx[SY]; nb.uxS = cx[-SY];
      nb.uxT = tx_[0]; nb.uxB = bx0; nb.uxWN = cx[SY - 1]; nb.uxWT = tx_[-1];
      nb.uy0 = cy[0]; nb.uyE = cy[1]; nb.uyW = cy[-1]; nb.uyN = cy[SY]; nb.uyS = cy[-SY];
      nb.uyT = ty_[0]; nb.uyB = by0; nb.uySE = cy[1 - SY]; nb.uyST = ty_[-SY];
      nb.uz0 = cz[0]; nb.uzE = cz[1]; nb.uzW = cz[-1]; nb.uzN = cz[SY]; nb.uzS = cz[-SY];
      nb.uzT = tz_[0]; nb.uzB = bz0; nb.uzEB = bzE; nb.uzNB = bzN;
      bx0 = nb.ux0; by0 = nb.uy0; bz0 = nb.uz0; bzE = nb.uzE; bzN = nb.uzN;
      const MomCell m = mom_compute<MOM_IMPLICIT>(g, J, nb, A, dt, B, adt, 1, ymet, theta);
      mom_store<MOM_IMPLICIT>(g, I, J, K, m, q, out);
      store_img(p_out, g, I, J, K, nb.p0, STAG_P);
    }
    double *t = un_cur;
    un_cur = un_next;
    un_next = un_new;
    un_new = t;
    t = p_cur;
    p_cur = p_next;
    p_next = p_nn;
    p_nn = t;
    t = d[0];
    d[0] = d[1];
    d[1] = d[2];
    d[2] = d[3];
    d[3] = d[4];
    d[4] = t;
  }
  cp_async_wait<0>();
}

// staged-plane stride of k_gradmom_tma (doubles): GP_N rounded up to 16
constexpr int GS = (GP_N + 15) / 16 * 16;
// Dynamic shared memory of k_gradmom_tma (with 128 bytes of alignment slack).
constexpr size_t GRADMOM_TMA_SMEM = sizeof(double) * ((size_t)(2 * 3 + 3 + 5) * GS + 3 * 3 * GP_N) + 128;
static_assert(GS * sizeof(double) % 128 == 0, "TMA destinations 128-byte aligned");

// k_gradmom_tma: k_gradmom_pipe with the raw planes (u*, delta, p) staged
// by the tensor-memory accelerator instead of per-thread cp.async: per
// plane one thread issues five 2-D boxes (cp.async.bulk.tensor, one
// mbarrier phase per batch), the iteration's copies for the next plane are
// issued before its projection instead of after it, and the wrap columns
// of the last x tile come from registers loaded one iteration ahead.  Same
// arithmetic, same shared-memory ring.  A wait that runs out of wait_limit
// polls records DEVERR_TMA_TIMEOUT in *err and the CTA returns (after
// waiting, bounded, for its last copies).
__global__ void __launch_bounds__(MC_X *MC_Y, 3)
    k_gradmom_tma(const __grid_constant__ CUtensorMap m_usx, const __grid_constant__ CUtensorMap m_usy,
                  const __grid_constant__ CUtensorMap m_usz, const __grid_constant__ CUtensorMap m_d,
                  const __grid_constant__ CUtensorMap m_p, Geo g, int planes, CFields3 us,
                  const double *__restrict__ delta, const double *__restrict__ p_in,
                  double *__restrict__ p_out, double radt, Fields3 q, Fields3 out, double A, double dt,
                  double B, double adt, const double2 *__restrict__ ymet, double theta, int *err,
                  unsigned wait_limit) {
  // TMA destinations start on 128-byte boundaries: the base is aligned at
  // run time (the host adds 128 bytes of slack) and the staged planes are
  // GS >= GP_N doubles apart (GS * 8 a multiple of 128)
  extern __shared__ __align__(128) double gsm_raw[];
  double *gsm = gsm_raw + ((128u - (smem_u32(gsm_raw) & 127u)) & 127u) / 8;
  double *ustar = gsm;                    // [2 slots][3][GS]
  double *pold = ustar + 2 * 3 * GS;      // [3 slots][GS]
  double *dl = pold + 3 * GS;             // [5 slots][GS]
  double *unew = dl + 5 * GS;             // [3 slots][3][GP_N]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + MC_X * ty;
  const int I0 = blockIdx.x * MC_X + 1, J0 = blockIdx.y * MC_Y + 1;
  const int K0 = blockIdx.z * planes + 1, K1 = min(g.nz, K0 + planes - 1);
  const bool wall = g.wall;
  const long long plane = (long long)g.NX * g.NY;
  constexpr int NT = MC_X * MC_Y;
  constexpr uint32_t BOX_BYTES = GP_X * GP_Y * sizeof(double);
  // Staging by TMA: thread 0 issues one GP_X x GP_Y box (rows J0-1.., columns
  // I0-1..) per field plane of a batch, all counted on one mbarrier whose
  // phase n is batch n.  Rows beyond the array read as zeros (y has walls:
  // they are never read).  Columns beyond the array are the periodic images
  // one period on (the last x tile): nwrap columns per row, loaded by
  // threads into registers when the batch is issued and stored after it
  // has landed.
  __shared__ uint64_t gbar;
  const int nwrap = max(0, I0 - 1 + GP_X - g.NX);
  int nbq = 0, nbatch = 0;
  double wv0 = 0.0, wv1 = 0.0;
  double *wd0 = nullptr, *wd1 = nullptr;
  // one box of field f at plane z into dst, part of the current batch
  auto box = [&](const double *f, int z, double *dst) {
    if (z >= g.NZ) z -= g.nz;
    if (tid == 0) {
      const CUtensorMap *m = f == us.x ? &m_usx : f == us.y ? &m_usy : f == us.z ? &m_usz
                             : f == delta ? &m_d : &m_p;
      if (nbq == 0) fence_proxy_async_smem();  // the slots' earlier reads (before the last barrier) come first
      mbar_expect_tx_only(&gbar, BOX_BYTES);
      tma_load3(dst, m, I0 - 1, J0 - 1, z, &gbar);
    }
    // wrap element w = (box, row, column) of this box for w = tid, tid + NT
    const int per = GP_Y * nwrap, lo = nbq * per;
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int w = tid + r * NT - lo;
      if (w >= 0 && w < per) {
        const int hy = w / nwrap, c = GP_X - nwrap + w % nwrap;
        const int x = I0 - 1 + c - g.nx, y = J0 - 1 + hy;
        if (x < g.NX && y < g.NY) {
          const double v = __ldg(f + (plane * z + x + (long long)g.NX * y));
          if (r == 0) {
            wv0 = v;
            wd0 = dst + c + GP_X * hy;
          } else {
            wv1 = v;
            wd1 = dst + c + GP_X * hy;
          }
        }
      }
    }
    nbq++;
  };
  // closes the batch of the boxes queued since the last call (one arrival)
  auto issue_batch = [&]() {
    if (tid == 0) mbar_arrive(&gbar);
    nbq = 0;
    nbatch++;
  };
  // waits for the last batch, stores the wrap columns, then the CTA barrier;
  // false (uniform over the CTA) when a wait ran out: the caller returns
  auto land_batch = [&]() -> bool {
    const bool ok = mbar_wait_n(&gbar, (uint32_t)((nbatch - 1) & 1), wait_limit);
    if (wd0) *wd0 = wv0;
    if (wd1) *wd1 = wv1;
    wd0 = wd1 = nullptr;
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(err, DEVERR_TMA_TIMEOUT);
        mbar_wait_n(&gbar, (uint32_t)((nbatch - 1) & 1), DNSB_WAIT_LIMIT);  // drain
      }
      return false;
    }
    return true;
  };
  auto us_slot = [&](int z) { return ustar + (z & 1) * 3 * GS; };
  auto issue_us = [&](int z) {
    double *s = us_slot(z);
    box(us.x, z, s);
    box(us.y, z, s + GS);
    box(us.z, z, s + 2 * GS);
  };
  constexpr int HX = MC_X + 2, HY = MC_Y + 2;
  __shared__ int rsrc[3][HY];
  __shared__ double rsgn[3][HY], rg[HY];
  if (tid < 3 * HY) {
    const int c = tid / HY, hy = tid - c * HY;
    const int y = J0 - 1 + hy;
    int hs = hy;
    double sgn = y <= g.NY - 1 ? 1.0 : 0.0;
    if (wall && sgn != 0.0) {
      if (c == STAG_Y) {
        if (y == 0 || y == g.ny) sgn = 0.0;
        else if (y == g.ny + 1) { hs = hy - 2; sgn = -1.0; }
      } else {
        if (y == 0) { hs = 1; sgn = -1.0; }
        else if (y == g.ny + 1) { hs = hy - 1; sgn = -1.0; }
      }
    }
    rsrc[c][hy] = hs;
    rsgn[c][hy] = sgn;
    if (c == STAG_Y) rg[hy] = sgn != 0.0 ? __ldg(g.rdyu + (J0 - 1 + hs)) : 0.0;
  }
  const bool plain = wall ? (J0 >= 2 && J0 + MC_Y <= g.ny - 1) : (J0 + MC_Y <= g.ny + 1);
  // projected u of one plane from its u* and delta of it and the plane above
  auto project_plane = [&](const double *su, const double *d0, const double *d1, double *dst) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
#pragma unroll
      for (int ry = 0; ry < 2; ry++) {
        const int hy = ty + ry * MC_Y;
        if (hy >= HY) continue;
        const int srow = GP_X * (plain ? hy : rsrc[c][hy]);
        const double sgn = plain ? 1.0 : rsgn[c][hy];
        const double gy = c == STAG_Y ? rg[hy] : 0.0;
#pragma unroll
        for (int rx = 0; rx < 2; rx++) {
          const int hx = tx + rx * MC_X;
          if (hx >= HX) continue;
          const int a = hx + srow;
          double v;
          if (c == STAG_X) v = su[a] - (d0[a + 1] - d0[a]) * g.rdx;
          else if (c == STAG_Y) v = su[GS + a] - (d0[a + GP_X] - d0[a]) * gy;
          else v = su[2 * GS + a] - (d1[a] - d0[a]) * g.rdz;
          dst[c * GP_N + hx + GP_X * hy] = plain ? v : sgn * v;
        }
      }
    }
  };
  // rotating slots: d[i] holds delta of plane K+i (i = 0..4), un_* the
  // projected planes K, K+1, K+2, p_* the lagged pressure of K, K+1, K+2
  double *d[5] = {dl, dl + GS, dl + 2 * GS, dl + 3 * GS, dl + 4 * GS};
  double *dm1 = d[4];  // delta of K0-1 in the slot that K0+4 takes later
  double *un_cur = unew, *un_next = unew + 3 * GP_N, *un_new = unew + 6 * GP_N;
  double *un_m1 = un_new;  // plane K0-1 in the slot that K0+2 takes later
  double *p_cur = pold, *p_next = pold + GS, *p_nn = pold + 2 * GS;
  // prologue: project K0-1, K0, K0+1; raw data of K0+2 in flight
  if (tid == 0) {
    mbar_init(&gbar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  issue_us(K0 - 1);
  box(delta, K0 - 1, dm1);
  box(delta, K0, d[0]);
  issue_batch();
  if (!land_batch()) return;
  project_plane(us_slot(K0 - 1), dm1, d[0], un_m1);
  issue_us(K0);
  box(delta, K0 + 1, d[1]);
  box(p_in, K0, p_cur);
  issue_batch();
  if (!land_batch()) return;  // u* of K0 and delta of K0+1 landed
  project_plane(us_slot(K0), d[0], d[1], un_cur);
  __syncthreads();     // every thread is done with u* of K0-1
  issue_us(K0 + 1);
  box(delta, K0 + 2, d[2]);
  box(p_in, K0 + 1, p_next);
  issue_batch();
  if (!land_batch()) return;
  project_plane(us_slot(K0 + 1), d[1], d[2], un_next);
  __syncthreads();     // projected K0-1, K0, K0+1 complete; u* of K0 free
  const int I = I0 + tx, J = J0 + ty;
  const bool inside = I <= g.nx && J <= g.ny;
  constexpr int SY = GP_X;
  const int h = (tx + 1) + SY * (ty + 1);
  // plane K0-1 as seen from the first cell: centre values and u_z east/north
  double bx0 = un_m1[h], by0 = un_m1[GP_N + h], bz0 = un_m1[2 * GP_N + h];
  double bzE = un_m1[2 * GP_N + h + 1], bzN = un_m1[2 * GP_N + h + SY];
  if (K0 + 1 <= K1) {
    issue_us(K0 + 2);
    box(delta, K0 + 3, d[3]);
  }
  issue_batch();
  for (int K = K0; K <= K1; K++) {
    MomNb nb;
    const int c0 = gidx(g, inside ? I : 1, inside ? J : 1, K);
    nb.qx0 = inside ? q.x[c0] : 0.0;
    nb.qy0 = inside ? q.y[c0] : 0.0;
    nb.qz0 = inside ? q.z[c0] : 0.0;
    // u* of K+2, delta of K+3, p of K+1 have landed; projected K+1 complete;
    // slots of K-1 free
    if (!land_batch()) return;
    if (K + 1 <= K1) {
      if (K + 2 <= K1) {   // raw data of the next iteration's projection
        issue_us(K + 3);
        box(delta, K + 4, d[4]);
      }
      box(p_in, K + 2, p_nn);
    }
    issue_batch();
    if (K + 1 <= K1) project_plane(us_slot(K + 2), d[2], d[3], un_new);
    if (inside) {
      const double *pk = p_cur + h, *pk1 = p_next + h;
      const double *dk = d[0] + h, *dk1 = d[1] + h;
      nb.p0 = pk[0] + dk[0] * radt;
      nb.pE = pk[1] + dk[1] * radt;
      nb.pN = pk[SY] + dk[SY] * radt;
      nb.pT = pk1[0] + dk1[0] * radt;
      const double *cx = un_cur + h, *tx_ = un_next + h;
      const double *cy = cx + GP_N, *ty_ = tx_ + GP_N;
      const double *cz = cx + 2 * GP_N, *tz_ = tx_ + 2 * GP_N;
      nb.ux0 = cx[0]; nb.uxE = cx[1]; nb.uxW = cx[-1]; nb.uxN = cx[SY]; nb.uxS = cx[-SY];
      nb.uxT = tx_[0]; nb.uxB = bx0; nb.uxWN = cx[SY - 1]; nb.uxWT = tx_[-1];
      nb.uy0 = cy[0]; nb.uyE = cy[1]; nb.uyW = cy[-1]; nb.uyN = cy[SY]; nb.uyS = cy[-SY];
      nb.uyT = ty_[0]; nb.uyB = by0; nb.uySE = cy[1 - SY]; nb.uyST = ty_[-SY];
      nb.uz0 = cz[0]; nb.uzE = cz[1]; nb.uzW = cz[-1]; nb.uzN = cz[SY]; nb.uzS = cz[-SY];
      nb.uzT = tz_[0]; nb.uzB = bz0; nb.uzEB = bzE; nb.uzNB = bzN;
      bx0 = nb.ux0; by0 = nb.uy0; bz0 = nb.uz0; bzE = nb.uzE; bzN = nb.uzN;
      const MomCell m = mom_compute<MOM_IMPLICIT>(g, J, nb, A, dt, B, adt, 1, ymet, theta);
      mom_store<MOM_IMPLICIT>(g, I, J, K, m, q, out);
      store_img(p_out, g, I, J, K, nb.p0, STAG_P);
    }
    double *t = un_cur;
    un_cur = un_next;
    un_next = un_new;
    un_new = t;
    t = p_cur;
    p_cur = p_next;
    p_next = p_nn;
    p_nn = t;
    t = d[0];
    d[0] = d[1];
    d[1] = d[2];
    d[2] = d[3];
    d[3] = d[4];
    d[4] = t;
  }
  // the last batch lands before the CTA leaves
  if (tid == 0) mbar_wait_n(&gbar, (uint32_t)((nbatch - 1) & 1), DNSB_WAIT_LIMIT);
}

// Dynamic shared memory of k_gradmom_pipe.
constexpr size_t GRADMOM_PIPE_SMEM = sizeof(double) * (2 * 3 + 3 + 5 + 3 * 3) * GP_N;

// k_gradmom_deep: k_gradmom_pipe with the raw data staged two planes ahead
// instead of one.  Iteration K waits for the copies issued in iteration K-2
// (cp.async.wait_group 1 leaves the previous iteration's in flight) and
// issues u* of K+4, delta of K+5 and p of K+3, so two planes of loads are
// in flight per CTA; the ring slots are indexed by plane number (u* 3,
// p 4, delta 6, projected u 3 x 3 components: 88.7 KB, 2 CTAs per SM).
constexpr int GD_US = 3, GD_P = 4, GD_D = 6, GD_UN = 3;
__global__ void __launch_bounds__(MC_X *MC_Y, 2)
    k_gradmom_deep(Geo g, int planes, CFields3 us, const double *__restrict__ delta,
                   const double *__restrict__ p_in, double *__restrict__ p_out, double radt,
                   Fields3 q, Fields3 out, double A, double dt, double B, double adt,
                   const double2 *__restrict__ ymet, double theta) {
  extern __shared__ __align__(16) double gsm[];
  double *ustar = gsm;                       // [GD_US][3][GP_N]
  double *pold = ustar + GD_US * 3 * GP_N;   // [GD_P][GP_N]
  double *dl = pold + GD_P * GP_N;           // [GD_D][GP_N]
  double *unew = dl + GD_D * GP_N;           // [GD_UN][3][GP_N]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + MC_X * ty;
  const int I0 = blockIdx.x * MC_X + 1, J0 = blockIdx.y * MC_Y + 1;
  const int K0 = blockIdx.z * planes + 1, K1 = min(g.nz, K0 + planes - 1);
  const bool wall = g.wall;
  constexpr int CH = GP_X / 2;
  const long long plane = (long long)g.NX * g.NY;
  bool stage = tid < GP_Y * CH;
  int goff = 0, soff = 0;
  if (stage) {
    const int ch = tid % CH, hy = tid / CH;
    int x = I0 - 1 + 2 * ch, y = J0 - 1 + hy;
    if (x >= g.NX) x -= g.nx;
    if (y >= g.NY) {
      if (wall) stage = false;
      y -= g.ny;
    }
    if (x + 1 >= g.NX || y >= g.NY) stage = false;
    goff = x + g.NX * y;
    soff = 2 * ch + GP_X * hy;
  }
  auto box = [&](const double *f, int z, double *dst) {
    if (z >= g.NZ) z -= g.nz;
    if (stage) cp_async16(dst + soff, f + (plane * z + goff));
  };
  auto us_slot = [&](int z) { return ustar + (z % GD_US) * 3 * GP_N; };
  auto p_slot = [&](int z) { return pold + (z % GD_P) * GP_N; };
  auto d_slot = [&](int z) { return dl + (z % GD_D) * GP_N; };
  auto un_slot = [&](int z) { return unew + (z % GD_UN) * 3 * GP_N; };
  auto issue_us = [&](int z) {
    double *s = us_slot(z);
    box(us.x, z, s);
    box(us.y, z, s + GP_N);
    box(us.z, z, s + 2 * GP_N);
  };
  constexpr int HX = MC_X + 2, HY = MC_Y + 2;
  __shared__ int rsrc[3][HY];
  __shared__ double rsgn[3][HY], rg[HY];
  if (tid < 3 * HY) {
    const int c = tid / HY, hy = tid - c * HY;
    const int y = J0 - 1 + hy;
    int hs = hy;
    double sgn = y <= g.NY - 1 ? 1.0 : 0.0;
    if (wall && sgn != 0.0) {
      if (c == STAG_Y) {
        if (y == 0 || y == g.ny) sgn = 0.0;
        else if (y == g.ny + 1) { hs = hy - 2; sgn = -1.0; }
      } else {
        if (y == 0) { hs = 1; sgn = -1.0; }
        else if (y == g.ny + 1) { hs = hy - 1; sgn = -1.0; }
      }
    }
    rsrc[c][hy] = hs;
    rsgn[c][hy] = sgn;
    if (c == STAG_Y) rg[hy] = sgn != 0.0 ? __ldg(g.rdyu + (J0 - 1 + hs)) : 0.0;
  }
  const bool plain = wall ? (J0 >= 2 && J0 + MC_Y <= g.ny - 1) : (J0 + MC_Y <= g.ny + 1);
  // projected u of plane z from its u* and delta of z and z+1
  auto project_plane = [&](int z) {
    const double *su = us_slot(z), *d0 = d_slot(z), *d1 = d_slot(z + 1);
    double *dst = un_slot(z);
#pragma unroll
    for (int c = 0; c < 3; c++) {
#pragma unroll
      for (int ry = 0; ry < 2; ry++) {
        const int hy = ty + ry * MC_Y;
        if (hy >= HY) continue;
        const int srow = GP_X * (plain ? hy : rsrc[c][hy]);
        const double sgn = plain ? 1.0 : rsgn[c][hy];
        const double gy = c == STAG_Y ? rg[hy] : 0.0;
#pragma unroll
        for (int rx = 0; rx < 2; rx++) {
          const int hx = tx + rx * MC_X;
          if (hx >= HX) continue;
          const int a = hx + srow;
          double v;
          if (c == STAG_X) v = su[a] - (d0[a + 1] - d0[a]) * g.rdx;
          else if (c == STAG_Y) v = su[GP_N + a] - (d0[a + GP_X] - d0[a]) * gy;
          else v = su[2 * GP_N + a] - (d1[a] - d0[a]) * g.rdz;
          dst[c * GP_N + hx + GP_X * hy] = plain ? v : sgn * v;
        }
      }
    }
  };
  // prologue: project K0-1, K0, K0+1; then two sets of raw data in flight:
  // (u* K0+2, delta K0+3, p K0+1) and (u* K0+3, delta K0+4, p K0+2)
  issue_us(K0 - 1);
  box(delta, K0 - 1, d_slot(K0 - 1));
  box(delta, K0, d_slot(K0));
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  project_plane(K0 - 1);
  issue_us(K0);
  box(delta, K0 + 1, d_slot(K0 + 1));
  box(p_in, K0, p_slot(K0));
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  project_plane(K0);
  __syncthreads();     // every thread is done with u* of K0-1 (slot of K0+2)
  issue_us(K0 + 1);
  box(delta, K0 + 2, d_slot(K0 + 2));
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  project_plane(K0 + 1);
  __syncthreads();     // projected K0-1, K0, K0+1 complete; u* of K0 free
  if (K0 + 1 <= K1) {
    issue_us(K0 + 2);
    box(delta, K0 + 3, d_slot(K0 + 3));
  }
  box(p_in, K0 + 1, p_slot(K0 + 1));
  cp_async_commit();
  if (K0 + 2 <= K1) {
    issue_us(K0 + 3);
    box(delta, K0 + 4, d_slot(K0 + 4));
  }
  if (K0 + 1 <= K1) box(p_in, K0 + 2, p_slot(K0 + 2));
  cp_async_commit();
  const int I = I0 + tx, J = J0 + ty;
  const bool inside = I <= g.nx && J <= g.ny;
  constexpr int SY = GP_X;
  const int h = (tx + 1) + SY * (ty + 1);
  // plane K0-1 as seen from the first cell: centre values and u_z east/north
  const double *um1 = un_slot(K0 - 1);
  double bx0 = um1[h], by0 = um1[GP_N + h], bz0 = um1[2 * GP_N + h];
  double bzE = um1[2 * GP_N + h + 1], bzN = um1[2 * GP_N + h + SY];
  for (int K = K0; K <= K1; K++) {
    MomNb nb;
    const int c0 = gidx(g, inside ? I : 1, inside ? J : 1, K);
    nb.qx0 = inside ? q.x[c0] : 0.0;
    nb.qy0 = inside ? q.y[c0] : 0.0;
    nb.qz0 = inside ? q.z[c0] : 0.0;
    cp_async_wait<1>();  // the set of iteration K-2: u* K+2, delta K+3, p K+1
    __syncthreads();     // ... for every thread; projected K+1 complete; slots of K-1 free
    if (K + 1 <= K1) project_plane(K + 2);
    if (K + 3 <= K1) {   // raw data two iterations ahead
      issue_us(K + 4);
      box(delta, K + 5, d_slot(K + 5));
    }
    if (K + 2 <= K1) box(p_in, K + 3, p_slot(K + 3));
    cp_async_commit();
    if (inside) {
      const double *pk = p_slot(K) + h, *pk1 = p_slot(K + 1) + h;
      const double *dk = d_slot(K) + h, *dk1 = d_slot(K + 1) + h;
      nb.p0 = pk[0] + dk[0] * radt;
      nb.pE = pk[1] + dk[1] * radt;
      nb.pN = pk[SY] + dk[SY] * radt;
      nb.pT = pk1[0] + dk1[0] * radt;
      const double *cx = un_slot(K) + h, *tx_ = un_slot(K + 1) + h;
      const double *cy = cx + GP_N, *ty_ = tx_ + GP_N;
      const double *cz = cx + 2 * GP_N, *tz_ = tx_ + 2 * GP_N;
      nb.ux0 = cx[0]; nb.uxE = cx[1]; nb.uxW = cx[-1]; nb.uxN = cx[SY]; nb.uxS = cx[-SY];
      nb.uxT = tx_[0]; nb.uxB = bx0; nb.uxWN = cx[SY - 1]; nb.uxWT = tx_[-1];
      nb.uy0 = cy[0]; nb.uyE = cy[1]; nb.uyW = cy[-1]; nb.uyN = cy[SY]; nb.uyS = cy[-SY];
      nb.uyT = ty_[0]; nb.uyB = by0; nb.uySE = cy[1 - SY]; nb.uyST = ty_[-SY];
      nb.uz0 = cz[0]; nb.uzE = cz[1]; nb.uzW = cz[-1]; nb.uzN = cz[SY]; nb.uzS = cz[-SY];
      nb.uzT = tz_[0]; nb.uzB = bz0; nb.uzEB = bzE; nb.uzNB = bzN;
      bx0 = nb.ux0; by0 = nb.uy0; bz0 = nb.uz0; bzE = nb.uzE; bzN = nb.uzN;
      const MomCell m = mom_compute<MOM_IMPLICIT>(g, J, nb, A, dt, B, adt, 1, ymet, theta);
      mom_store<MOM_IMPLICIT>(g, I, J, K, m, q, out);
      store_img(p_out, g, I, J, K, nb.p0, STAG_P);
    }
  }
  cp_async_wait<0>();
}

// Dynamic shared memory of k_gradmom_deep.
constexpr size_t GRADMOM_DEEP_SMEM = sizeof(double) * (GD_US * 3 + GD_P + GD_D + GD_UN * 3) * GP_N;

}  // namespace dnsb
