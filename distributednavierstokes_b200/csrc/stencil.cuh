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
#define LDG(p, o) __ldg((p) + (o))
  const double ux0 = LDG(ux, c0), uxE = LDG(ux, c0 + 1), uxW = LDG(ux, c0 - 1);
  const double uxN = LDG(ux, c0 + sy), uxS = LDG(ux, c0 - sy);
  const double uxT = LDG(ux, c0 + sz), uxB = LDG(ux, c0 - sz);
  const double uxWN = LDG(ux, c0 - 1 + sy), uxWT = LDG(ux, c0 - 1 + sz);
  const double uy0 = LDG(uy, c0), uyE = LDG(uy, c0 + 1), uyW = LDG(uy, c0 - 1);
  const double uyN = LDG(uy, c0 + sy), uyS = LDG(uy, c0 - sy);
  const double uyT = LDG(uy, c0 + sz), uyB = LDG(uy, c0 - sz);
  const double uySE = LDG(uy, c0 + 1 - sy), uyST = LDG(uy, c0 - sy + sz);
  const double uz0 = LDG(uz, c0), uzE = LDG(uz, c0 + 1), uzW = LDG(uz, c0 - 1);
  const double uzN = LDG(uz, c0 + sy), uzS = LDG(uz, c0 - sy);
  const double uzT = LDG(uz, c0 + sz), uzB = LDG(uz, c0 - sz);
  const double uzEB = LDG(uz, c0 + 1 - sz), uzNB = LDG(uz, c0 + sy - sz);
#undef LDG

  const double qx0 = readq ? q.x[c0] : 0.0, qy0 = readq ? q.y[c0] : 0.0;
  const double qz0 = readq ? q.z[c0] : 0.0;
  double pE = 0.0, pN = 0.0, pT = 0.0, p0 = 0.0;
  if (MODE == MOM_IMPLICIT) {
    p0 = __ldg(p + c0);
    pE = __ldg(p + c0 + 1);
    pN = __ldg(p + c0 + sy);
    pT = __ldg(p + c0 + sz);
  }
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
  const int c0 = gidx(g, I, J, K);
  const MomCell m = momentum_cell<MODE == MOM_ONLY ? MOM_EXPLICIT : MODE>(
      g, I, J, K, q, u, p, A, dt, B, adt, readq, ymet, theta);
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
