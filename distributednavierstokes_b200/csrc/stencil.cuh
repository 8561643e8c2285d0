// stencil.cuh -- staggered finite-volume stencils on ghosted fields.
//
// Restates src/operators.jl (divergence, momentum, pressure gradient) and
// the pointwise parts of src/timestep.jl / src/ydiffusion.jl, fused per RK
// stage: the momentum kernel also applies the explicit register update
// (timestep.jl:54-58) or forms the semi-implicit explicit increment
// v = u + B q - alpha dt grad p (ydiffusion.jl:133-135); the gradient kernel
// also updates the lagged pressure (timestep.jl:49-51), writes ghost images
// (replacing exchange_halo!) and reduces max|u| for the next CFL step.
// Divisions by grid metrics use precomputed reciprocals (<= 1 ulp apart from
// the reference's divisions); halving uses *0.5 (exact).
#pragma once
#include "common.cuh"
#include "tma.cuh"

namespace dnsb {

enum MomMode { MOM_ONLY = 0, MOM_EXPLICIT = 1, MOM_IMPLICIT = 2 };

// Per-row metrics of the momentum stencil, packed for 16-byte loads:
// ymet[6 J + 0..5] = (dy_J, dy_{J+1}), (1/dy_J, 1/dy_{J+1}),
// (1/dyu_J, 1/dyu_{J-1}), (at, bt), (ct, an), (bn, cn) of row j = J-1 of
// the Crank-Nicolson operator (ydiffusion_coefficients, src/ydiffusion.jl:31-51).
constexpr int YMET = 6;

// Right-hand side of the Crank-Nicolson row j = J-1 of one component
// (imexrhs_kernel!, src/ydiffusion.jl:71-91): v + theta (a u_S + b u_0 +
// c u_N), the wall rows folded into the coefficients (a_0 = 0 and
// c_{ny-1} = 0 multiply finite ghost values).
__device__ __forceinline__ double cn_rhs(double a, double b, double c, double v, double theta,
                                         double uS, double u0, double uN) {
  return v + theta * ((a * uS + b * u0) + c * uN);
}

// momentum_kernel! (src/operators.jl:44-145) at one interior cell: loads
// the 3x3x3 staggered neighbourhood (27 values) plus q and p, returns the
// new RK registers q and the stage increment v (MOM_EXPLICIT: u + B q;
// MOM_IMPLICIT: u + B q - adt grad p on active DOFs, plus theta Dy u^n:
// the Crank-Nicolson right-hand side).  Each component's v is finished
// right after its q so that its wall-normal neighbours die early.
struct MomCell {
  double qx, qy, qz;  // new registers
  double vx, vy, vz;  // stage increments
};

// The staggered neighbourhood of one cell (E/W: I+-1, N/S: J+-1, T/B:
// K+-1) with q and p there: the inputs of momentum_kernel!.
struct MomNb {
  double ux0, uxE, uxW, uxN, uxS, uxT, uxB, uxWN, uxWT;
  double uy0, uyE, uyW, uyN, uyS, uyT, uyB, uySE, uyST;
  double uz0, uzE, uzW, uzN, uzS, uzT, uzB, uzEB, uzNB;
  double qx0, qy0, qz0, p0, pE, pN, pT;
};

template <int MODE>
__device__ __forceinline__ MomCell mom_compute(const Geo &g, int J, const MomNb &nb, double A,
                                               double dt, double B, double adt, int readq,
                                               const double2 *__restrict__ ymet, double theta);

// momentum_cell: the neighbourhood straight from HBM (one load per value).
template <int MODE>
__device__ __forceinline__ MomCell momentum_cell(const Geo &g, int I, int J, int K, const Fields3 &q,
                                                 const CFields3 &u, const double *__restrict__ p,
                                                 double A, double dt, double B, double adt,
                                                 int readq, const double2 *__restrict__ ymet,
                                                 double theta) {
  // 64-bit offsets here: measured faster than 32-bit ones for this kernel
  const long long sy = g.NX, sz = (long long)g.NX * g.NY;
  const long long c0 = (long long)I + g.NX * ((long long)J + (long long)g.NY * K);
  const double *ux = u.x, *uy = u.y, *uz = u.z;
  MomNb nb;
#define LDG(p, o) __ldg((p) + (o))
  nb.ux0 = LDG(ux, c0); nb.uxE = LDG(ux, c0 + 1); nb.uxW = LDG(ux, c0 - 1);
  nb.uxN = LDG(ux, c0 + sy); nb.uxS = LDG(ux, c0 - sy);
  nb.uxT = LDG(ux, c0 + sz); nb.uxB = LDG(ux, c0 - sz);
  nb.uxWN = LDG(ux, c0 - 1 + sy); nb.uxWT = LDG(ux, c0 - 1 + sz);
  nb.uy0 = LDG(uy, c0); nb.uyE = LDG(uy, c0 + 1); nb.uyW = LDG(uy, c0 - 1);
  nb.uyN = LDG(uy, c0 + sy); nb.uyS = LDG(uy, c0 - sy);
  nb.uyT = LDG(uy, c0 + sz); nb.uyB = LDG(uy, c0 - sz);
  nb.uySE = LDG(uy, c0 + 1 - sy); nb.uyST = LDG(uy, c0 - sy + sz);
  nb.uz0 = LDG(uz, c0); nb.uzE = LDG(uz, c0 + 1); nb.uzW = LDG(uz, c0 - 1);
  nb.uzN = LDG(uz, c0 + sy); nb.uzS = LDG(uz, c0 - sy);
  nb.uzT = LDG(uz, c0 + sz); nb.uzB = LDG(uz, c0 - sz);
  nb.uzEB = LDG(uz, c0 + 1 - sz); nb.uzNB = LDG(uz, c0 + sy - sz);
#undef LDG
  nb.qx0 = readq ? q.x[c0] : 0.0;
  nb.qy0 = readq ? q.y[c0] : 0.0;
  nb.qz0 = readq ? q.z[c0] : 0.0;
  nb.p0 = nb.pE = nb.pN = nb.pT = 0.0;
  if (MODE == MOM_IMPLICIT) {
    nb.p0 = __ldg(p + c0);
    nb.pE = __ldg(p + c0 + 1);
    nb.pN = __ldg(p + c0 + sy);
    nb.pT = __ldg(p + c0 + sz);
  }
  return mom_compute<MODE>(g, J, nb, A, dt, B, adt, readq, ymet, theta);
}

// The arithmetic of momentum_kernel! on a loaded neighbourhood.
template <int MODE>
__device__ __forceinline__ MomCell mom_compute(const Geo &g, int J, const MomNb &nb, double A,
                                               double dt, double B, double adt, int readq,
                                               const double2 *__restrict__ ymet, double theta) {
  const double ux0 = nb.ux0, uxE = nb.uxE, uxW = nb.uxW, uxN = nb.uxN, uxS = nb.uxS;
  const double uxT = nb.uxT, uxB = nb.uxB, uxWN = nb.uxWN, uxWT = nb.uxWT;
  const double uy0 = nb.uy0, uyE = nb.uyE, uyW = nb.uyW, uyN = nb.uyN, uyS = nb.uyS;
  const double uyT = nb.uyT, uyB = nb.uyB, uySE = nb.uySE, uyST = nb.uyST;
  const double uz0 = nb.uz0, uzE = nb.uzE, uzW = nb.uzW, uzN = nb.uzN, uzS = nb.uzS;
  const double uzT = nb.uzT, uzB = nb.uzB, uzEB = nb.uzEB, uzNB = nb.uzNB;
  const double qx0 = nb.qx0, qy0 = nb.qy0, qz0 = nb.qz0;
  const double p0 = nb.p0, pE = nb.pE, pN = nb.pN, pT = nb.pT;
  const double2 *ym = ymet + YMET * J;
  const double2 m0 = __ldg(ym), m1 = __ldg(ym + 1), m2 = __ldg(ym + 2);
  const double dyJ = m0.x, dyJ1 = m0.y, rdyJ = m1.x, rdyJ1 = m1.y, rdyuJ = m2.x, rdyuJm = m2.y;
  const double ey = g.epsy, nu = g.visc;
  // The convective products are formed from unhalved midpoint sums and the
  // flux divergence is scaled by 1/4 once: scaling by powers of two is
  // exact, so this equals the reference's halved-midpoint form.
  MomCell m;
  // x momentum, at the right x-face of cell (I, J, K)
  {
    const double uce = ux0 + uxE, ucw = uxW + ux0;
    const double vn = uy0 + uyE, un = ux0 + uxN;
    const double vs = uyS + uySE, us = uxS + ux0;
    const double wt = uz0 + uzE, ut = ux0 + uxT;
    const double wb = uzB + uzEB, ub = uxB + ux0;
    const double conv = 0.25 * ((uce * uce - ucw * ucw) * g.rdx + (vn * un - vs * us) * rdyJ +
                                (wt * ut - wb * ub) * g.rdz);
    const double diff = (uxE - 2 * ux0 + uxW) * g.rdx2 +
                        ey * ((uxN - ux0) * rdyuJ - (ux0 - uxS) * rdyuJm) * rdyJ +
                        (uxT - 2 * ux0 + uxB) * g.rdz2;
    const double f = dt * (-conv + nu * diff + g.fx);
    m.qx = readq ? A * qx0 + f : f;
    if (MODE == MOM_EXPLICIT) {
      m.vx = ux0 + B * m.qx;  // u <- u + B q on ranges[c] (timestep.jl:54-58)
    } else {
      // v = u + B q - alpha dt grad p (ydiffusion.jl:133-135)
      const double2 m3 = __ldg(ym + 3), m4 = __ldg(ym + 4);
      m.vx = cn_rhs(m3.x, m3.y, m4.x, (ux0 + B * m.qx) - adt * (pE - p0) * g.rdx, theta, uxS, ux0,
                    uxN);
    }
  }
  // y momentum, at the top y-face; Delta-y weighted transporters
  {
    const double ue = (ux0 * dyJ + uxN * dyJ1) * rdyuJ, ve = uy0 + uyE;
    const double uw = (uxW * dyJ + uxWN * dyJ1) * rdyuJ, vw = uyW + uy0;
    const double vcn = uy0 + uyN, vcs = uyS + uy0;
    const double wtv = (uz0 * dyJ + uzN * dyJ1) * rdyuJ, vt = uy0 + uyT;
    const double wbv = (uzB * dyJ + uzNB * dyJ1) * rdyuJ, vb = uyB + uy0;
    const double conv = 0.25 * ((ue * ve - uw * vw) * g.rdx + (vcn * vcn - vcs * vcs) * rdyuJ +
                                (wtv * vt - wbv * vb) * g.rdz);
    const double diff = (uyE - 2 * uy0 + uyW) * g.rdx2 +
                        ey * ((uyN - uy0) * rdyJ1 - (uy0 - uyS) * rdyJ) * rdyuJ +
                        (uyT - 2 * uy0 + uyB) * g.rdz2;
    const double f = dt * (-conv + nu * diff + g.fy);
    m.qy = readq ? A * qy0 + f : f;
    const bool yact = J <= g.jymax;
    if (MODE == MOM_EXPLICIT) {
      m.vy = yact ? uy0 + B * m.qy : uy0;
    } else {
      const double v = yact ? (uy0 + B * m.qy) - adt * (pN - p0) * rdyuJ : uy0;
      const double2 m4 = __ldg(ym + 4), m5 = __ldg(ym + 5);
      m.vy = cn_rhs(m4.y, m5.x, m5.y, v, theta, uyS, uy0, uyN);
    }
  }
  // z momentum, at the back z-face
  {
    const double ue = ux0 + uxT, we = uz0 + uzE;
    const double uw = uxW + uxWT, ww = uzW + uz0;
    const double vnw = uy0 + uyT, wn = uz0 + uzN;
    const double vsw = uyS + uyST, ws = uzS + uz0;
    const double wct = uz0 + uzT, wcb = uzB + uz0;
    const double conv = 0.25 * ((ue * we - uw * ww) * g.rdx + (vnw * wn - vsw * ws) * rdyJ +
                                (wct * wct - wcb * wcb) * g.rdz);
    const double diff = (uzE - 2 * uz0 + uzW) * g.rdx2 +
                        ey * ((uzN - uz0) * rdyuJ - (uz0 - uzS) * rdyuJm) * rdyJ +
                        (uzT - 2 * uz0 + uzB) * g.rdz2;
    const double f = dt * (-conv + nu * diff + g.fz);
    m.qz = readq ? A * qz0 + f : f;
    if (MODE == MOM_EXPLICIT) {
      m.vz = uz0 + B * m.qz;
    } else {
      const double2 m3 = __ldg(ym + 3), m4 = __ldg(ym + 4);
      m.vz = cn_rhs(m3.x, m3.y, m4.x, (uz0 + B * m.qz) - adt * (pT - p0) * g.rdz, theta, uzS, uz0,
                    uzN);
    }
  }
  return m;
}

template <int MODE>
__device__ __forceinline__ void mom_store(const Geo &g, int I, int J, int K, const MomCell &m,
                                          const Fields3 &q, const Fields3 &out);

// momentum_kernel! (src/operators.jl:44-145), one thread per interior cell.
// MOM_ONLY: q <- A q + dt F(u).
// MOM_EXPLICIT: also W_c = u_c + B q_c on active DOFs, with ghost images.
// MOM_IMPLICIT: also the Crank-Nicolson right-hand side
//   V_c = (u_c + B q_c - adt d_c p) + theta Dy u_c
// (coef = [at bt ct an bn cn] rows of ny), so the y-solve reads only V.
// All 34 loads are held at once: 2 CTAs of 256 per SM keep the kernel free
// of spills (measured faster than 3-4 CTAs with spills).
template <int MODE>
__global__ void __launch_bounds__(256, 2) k_momentum(Geo g, Fields3 q, CFields3 u, Fields3 out,
                                                  const double *__restrict__ p, double A, double dt,
                                                  double B, double adt, int readq,
                                                  const double2 *__restrict__ ymet, double theta) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  if (I > g.nx || J > g.ny) return;
  const MomCell m = momentum_cell<MODE == MOM_ONLY ? MOM_EXPLICIT : MODE>(
      g, I, J, K, q, u, p, A, dt, B, adt, readq, ymet, theta);
  mom_store<MODE>(g, I, J, K, m, q, out);
}

// Stores of one cell of k_momentum / k_momentum_tile.
template <int MODE>
__device__ __forceinline__ void mom_store(const Geo &g, int I, int J, int K, const MomCell &m,
                                          const Fields3 &q, const Fields3 &out) {
  const int c0 = gidx(g, I, J, K);
  const bool yact = J <= g.jymax;
  q.x[c0] = m.qx;
  if (yact) q.y[c0] = m.qy;
  q.z[c0] = m.qz;
  if (MODE == MOM_EXPLICIT) {
    store_img(out.x, g, I, J, K, m.vx, STAG_X);
    if (yact) store_img(out.y, g, I, J, K, m.vy, STAG_Y);
    store_img(out.z, g, I, J, K, m.vz, STAG_Z);
  } else if (MODE == MOM_IMPLICIT) {
    out.x[c0] = m.vx;
    out.y[c0] = m.vy;
    out.z[c0] = m.vz;
  }
}

// Column of k_momentum_march: MC_X x MC_Y cells per CTA (one thread each)
// walking `planes` planes in z (MC_Z on large grids; fewer where the grid
// would otherwise leave SMs idle).  Planes are staged with a one-cell halo in x
// and y in a ring of four.
constexpr int MC_X = 32, MC_Y = 8, MC_Z = 16;  // measured best of 8-64 planes, 4-8 rows
constexpr int MP_X = MC_X + 2, MP_Y = MC_Y + 2, MP_N = MP_X * MP_Y;

// momentum_kernel! with the velocity planes staged in shared memory: the
// CTA keeps planes K-1, K, K+1 of u.x, u.y, u.z (each MP_X x MP_Y, rows
// starting at I0 - 1, a multiple of 32, so every 16-byte cp.async is
// aligned when the fields are 16-byte aligned and nx is even) and copies
// plane K+2 into the fourth slot while it computes plane K.  Same
// arithmetic and stores as k_momentum.
// 3 CTAs of 256 per SM (80 registers; faster than 2 CTAs without the cap)
template <int MODE>
__global__ void __launch_bounds__(MC_X *MC_Y, 3)
    k_momentum_march(Geo g, Fields3 q, CFields3 u, Fields3 out, const double *__restrict__ p,
                     double A, double dt, double B, double adt, int readq,
                     const double2 *__restrict__ ymet, double theta, int planes,
                     const double *__restrict__ dtp) {
  __shared__ __align__(16) double ring[4][3][MP_N];
  if (dtp) dt = *dtp;  // the step size from device memory (a step inside a CUDA graph)
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + MC_X * ty;
  const int I0 = blockIdx.x * MC_X + 1, J0 = blockIdx.y * MC_Y + 1;
  const int K0 = blockIdx.z * planes + 1, K1 = min(g.nz, K0 + planes - 1);
  constexpr int CH = MP_X / 2;  // 16-byte chunks per halo row
  static_assert(MP_Y * CH <= MC_X * MC_Y, "one staging chunk per thread and field plane");
  // this thread's chunk of every staged plane (the same in-plane offset for
  // all planes and components); chunks outside the ghosted array are never
  // read by an interior cell
  const long long plane = (long long)g.NX * g.NY;
  int goff = 0, soff = 0;
  bool stage = tid < MP_Y * CH;
  if (stage) {
    const int ch = tid % CH, hy = tid / CH;
    const int x = I0 - 1 + 2 * ch, y = J0 - 1 + hy;
    stage = x + 1 < g.NX && y < g.NY;
    goff = x + g.NX * y;
    soff = 2 * ch + MP_X * hy;
  }
  // copies plane z (0..NZ-1) of the three components into its ring slot
  auto issue = [&](int z) {
    double(*slot)[MP_N] = ring[z & 3];
    if (stage) {
      const long long o = plane * z + goff;
      cp_async16(&slot[0][soff], u.x + o);
      cp_async16(&slot[1][soff], u.y + o);
      cp_async16(&slot[2][soff], u.z + o);
    }
    cp_async_commit();
  };
  const int I = I0 + tx, J = J0 + ty;
  const bool inside = I <= g.nx && J <= g.ny;
  issue(K0 - 1);
  issue(K0);
  issue(K0 + 1);
  constexpr int SY = MP_X;
  const int h = (tx + 1) + SY * (ty + 1);
  const int sy = g.NX, sz = g.NX * g.NY;
  for (int K = K0; K <= K1; K++) {
    // q and p of this plane from HBM while the plane copies land
    MomNb nb;
    const int c0 = gidx(g, inside ? I : 1, inside ? J : 1, K);
    nb.qx0 = (inside && readq) ? q.x[c0] : 0.0;
    nb.qy0 = (inside && readq) ? q.y[c0] : 0.0;
    nb.qz0 = (inside && readq) ? q.z[c0] : 0.0;
    nb.p0 = nb.pE = nb.pN = nb.pT = 0.0;
    if (MODE == MOM_IMPLICIT && inside) {
      nb.p0 = __ldg(p + c0);
      nb.pE = __ldg(p + c0 + 1);
      nb.pN = __ldg(p + c0 + sy);
      nb.pT = __ldg(p + c0 + sz);
    }
    cp_async_wait<0>();  // planes up to K+1 have landed (this thread's copies)
    __syncthreads();     // ... everyone's, and plane K-2's slot is free
    if (K + 2 <= K1 + 1) issue(K + 2);
    if (inside) {
      const double *bx = ring[(K - 1) & 3][0] + h, *cx = ring[K & 3][0] + h, *tx_ = ring[(K + 1) & 3][0] + h;
      const double *by = ring[(K - 1) & 3][1] + h, *cy = ring[K & 3][1] + h, *ty_ = ring[(K + 1) & 3][1] + h;
      const double *bz = ring[(K - 1) & 3][2] + h, *cz = ring[K & 3][2] + h, *tz_ = ring[(K + 1) & 3][2] + h;
      nb.ux0 = cx[0]; nb.uxE = cx[1]; nb.uxW = cx[-1]; nb.uxN = cx[SY]; nb.uxS = cx[-SY];
      nb.uxT = tx_[0]; nb.uxB = bx[0]; nb.uxWN = cx[SY - 1]; nb.uxWT = tx_[-1];
      nb.uy0 = cy[0]; nb.uyE = cy[1]; nb.uyW = cy[-1]; nb.uyN = cy[SY]; nb.uyS = cy[-SY];
      nb.uyT = ty_[0]; nb.uyB = by[0]; nb.uySE = cy[1 - SY]; nb.uyST = ty_[-SY];
      nb.uz0 = cz[0]; nb.uzE = cz[1]; nb.uzW = cz[-1]; nb.uzN = cz[SY]; nb.uzS = cz[-SY];
      nb.uzT = tz_[0]; nb.uzB = bz[0]; nb.uzEB = bz[1]; nb.uzNB = bz[SY];
      const MomCell m = mom_compute<MODE == MOM_ONLY ? MOM_EXPLICIT : MODE>(
          g, J, nb, A, dt, B, adt, readq, ymet, theta);
      mom_store<MODE>(g, I, J, K, m, q, out);
    }
  }
  cp_async_wait<0>();
}

enum GradMode { GRAD_EXPLICIT = 0, GRAD_IMPLICIT = 1 };
constexpr int UMAX_SLOTS = 128;

__device__ __forceinline__ unsigned long long dbits(double v) {
  return (unsigned long long)__double_as_longlong(v);
}

// Projection update u = W - grad(psi) on active DOFs with ghost images
// (pressuregrad_update! + exchange_halo!, src/operators.jl:180-220,
// src/timestep.jl:28-30).  GRAD_IMPLICIT additionally does
// p += delta/(alpha dt) with images (src/timestep.jl:49-52).  W may alias u.
// If umax != nullptr, the block maxima of |u_c| over the interior are
// folded into umax[c] (as ordered bit patterns of non-negative doubles).
template <int MODE>
__global__ void __launch_bounds__(256) k_grad(Geo g, Fields3 u, CFields3 W,
                                              const double *__restrict__ psi, double *p,
                                              double radt, unsigned long long *umax) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  double m0 = 0, m1 = 0, m2 = 0;
  if (I <= g.nx && J <= g.ny) {
    const int sy = g.NX, sz = g.NX * g.NY;
    const int c0 = gidx(g, I, J, K);
    const bool yact = J <= g.jymax;
    // every load before the first store (u may alias W)
    const double *ps = psi + c0;
    const double s0 = ps[0], sE = ps[1], sN = ps[sy], sT = ps[sz];
    const double wx = W.x[c0], wy = W.y[c0], wz = W.z[c0];
    const double p0 = MODE == GRAD_IMPLICIT ? p[c0] : 0.0;
    const double ry = __ldg(g.rdyu + J);
    const double vx = wx - (sE - s0) * g.rdx;
    const double vy = wy - (sN - s0) * ry;
    const double vz = wz - (sT - s0) * g.rdz;
    store_img(u.x, g, I, J, K, vx, STAG_X);
    store_img(u.z, g, I, J, K, vz, STAG_Z);
    if (yact) store_img(u.y, g, I, J, K, vy, STAG_Y);
    if (MODE == GRAD_IMPLICIT) store_img(p, g, I, J, K, p0 + s0 * radt, STAG_P);
    m0 = fabs(vx);
    m1 = yact ? fabs(vy) : 0.0;
    m2 = fabs(vz);
  }
  if (umax) {
    // block maximum, then one atomic per block into one of UMAX_SLOTS slots
    // per component (spreads the contention; the host reduces the slots)
    __shared__ double red[3][8];
    for (int o = 16; o > 0; o >>= 1) {
      m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
      m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
      m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int w = tid >> 5, nw = (blockDim.x * blockDim.y + 31) >> 5;
    if ((tid & 31) == 0) { red[0][w] = m0; red[1][w] = m1; red[2][w] = m2; }
    __syncthreads();
    if (tid < 3) {
      double m = 0.0;
      for (int k = 0; k < nw; k++) m = fmax(m, red[tid][k]);
      const unsigned slot = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) % UMAX_SLOTS;
      atomicMax(umax + tid * UMAX_SLOTS + slot, dbits(m));
    }
  }
}

// pgrad{x,y,z}_kernel! (src/operators.jl:180-196): phi -= s * d_c p on
// ranges[c]; no halo update (as in the reference).
__global__ void k_pgrad(Geo g, double *phi, const double *__restrict__ p, int c, double s) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  const int jh = (c == STAG_Y) ? g.jymax : g.ny;
  if (I > g.nx || J > jh) return;
  const int c0 = gidx(g, I, J, K);
  const long long off = c == 0 ? 1 : c == 1 ? (long long)g.NX : (long long)g.NX * g.NY;
  const double r = c == 0 ? g.rdx : c == 1 ? __ldg(g.rdyu + J) : g.rdz;
  phi[c0] = phi[c0] - s * (p[c0 + off] - p[c0]) * r;
}

// ranges-wise register update u_c += B q_c then u_c -= s d_c p (the first
// half of imex_update!, src/ydiffusion.jl:133-135), writing into V the
// Crank-Nicolson right-hand side v + theta Dy u^n (see cn_rhs).
__global__ void k_vupdate(Geo g, Fields3 V, CFields3 u, CFields3 q, const double *__restrict__ p,
                          double B, double adt, const double2 *__restrict__ ymet, double theta) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  if (I > g.nx || J > g.ny) return;
  const int sy = g.NX, sz = g.NX * g.NY;
  const int c0 = gidx(g, I, J, K);
  const double p0 = p[c0];
  const double ux0 = u.x[c0], uy0 = u.y[c0], uz0 = u.z[c0];
  const double vx = (ux0 + B * q.x[c0]) - adt * (p[c0 + 1] - p0) * g.rdx;
  const double vy = J <= g.jymax ? (uy0 + B * q.y[c0]) - adt * (p[c0 + sy] - p0) * __ldg(g.rdyu + J)
                                 : uy0;
  const double vz = (uz0 + B * q.z[c0]) - adt * (p[c0 + sz] - p0) * g.rdz;
  const double2 *ym = ymet + YMET * J;
  const double2 m3 = ym[3], m4 = ym[4], m5 = ym[5];
  V.x[c0] = cn_rhs(m3.x, m3.y, m4.x, vx, theta, u.x[c0 - sy], ux0, u.x[c0 + sy]);
  V.y[c0] = cn_rhs(m4.y, m5.x, m5.y, vy, theta, u.y[c0 - sy], uy0, u.y[c0 + sy]);
  V.z[c0] = cn_rhs(m3.x, m3.y, m4.x, vz, theta, u.z[c0 - sy], uz0, u.z[c0 + sy]);
}

// divergence_kernel! (src/operators.jl:10-26) into the ghost-free r.
__global__ void k_divergence(Geo g, double *r, CFields3 u) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  if (I > g.nx || J > g.ny) return;
  const int sy = g.NX, sz = g.NX * g.NY;
  const int c0 = gidx(g, I, J, K);
  r[(I - 1) + (long long)g.nx * ((J - 1) + (long long)g.ny * (K - 1))] =
      (u.x[c0] - u.x[c0 - 1]) * g.rdx + (u.y[c0] - u.y[c0 - sy]) * __ldg(g.rdy + J) +
      (u.z[c0] - u.z[c0 - sz]) * g.rdz;
}

// exchange_halo! on one rank: every ghost cell (and, for the wall-normal
// component, the wall faces) from its interior source.
__global__ void k_fill_ghosts(Geo g, double *phi, int stag) {
  long long n = (long long)g.NX * g.NY * g.NZ;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int I = (int)(t % g.NX);
    long long r = t / g.NX;
    int J = (int)(r % g.NY);
    int K = (int)(r / g.NY);
    bool ghost = I == 0 || I == g.nx + 1 || J == 0 || J == g.ny + 1 || K == 0 || K == g.nz + 1 ||
                 (g.wall && stag == STAG_Y && J == g.ny);
    if (!ghost) continue;
    int Is = I, Js = J, Ks = K;
    double s;
    bool nz = ghost_src(g, stag, Is, Js, Ks, s);
    phi[t] = nz ? s * phi[gidx(g, Is, Js, Ks)] : 0.0;
  }
}

}  // namespace dnsb
