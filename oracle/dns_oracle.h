/*
 * dns_oracle.h -- CPU oracle (test infrastructure only).
 *
 * A plain-C restatement of the single-rank finite-volume time step of
 * DistributedNavierStokes (Julia).  It is the checker for the CUDA library:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  The product never links or calls it.
 *
 * Layout: every ghosted field is (nx+2) x (ny+2) x (nz+2) doubles,
 * column-major (x fastest), ghost width w = 1, exactly the reference's
 * `scalarfield` (src/fields.jl:4-5).  A C index I equals the reference's
 * cell index i (interior I = 1..nx, ghosts I = 0 and nx+1).
 *
 * Staggering codes: 0 = u.x, 1 = u.y, 2 = u.z, 3 = p (cell centred).
 */
#ifndef DNS_ORACLE_H
#define DNS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dnso dnso_t;

/* setup(; n, lims, bc, stretch, visc, bodyforce, ydiffusion)
 * (src/setup.jl:34-113).  `yf` holds the ny+1 global y faces
 * yface(j) = y0 + Ly*stretch(j/ny), j = 0..ny (src/setup.jl:155-156), so the
 * caller's stretch function is evaluated once, on the host, as in Julia. */
dnso_t *dnso_create(int nx, int ny, int nz, int wall, int implicit, double Lx,
                    double Lz, const double *yf, double visc, double fx,
                    double fy, double fz);
void dnso_destroy(dnso_t *s);
void dnso_set_threads(int n);

/* grid metrics (src/setup.jl:148-193): dy, dyu have ny+2 entries (ghosted
 * index J = 0..ny+1); lam1 nx/2+1, lam3 nz, lam2 ny (periodic y only). */
void dnso_grid(const dnso_t *s, double *dx, double *dz, double *dy,
               double *dyu, double *dymin);
void dnso_poisson_coeffs(const dnso_t *s, double *lam1, double *lam2,
                         double *lam3, double *ay, double *by, double *cy);
void dnso_ydiff_coeffs(const dnso_t *s, double *at, double *bt, double *ct,
                       double *an, double *bn, double *cn);

/* exchange_halo! single rank (src/halo.jl:26-45, 81-126) */
void dnso_fill_halo(const dnso_t *s, double *phi, int stag);
/* divergence! (src/operators.jl:10-42); r is ghost-free nx*ny*nz */
void dnso_divergence(const dnso_t *s, const double *ux, const double *uy,
                     const double *uz, double *r);
/* momentum! (src/operators.jl:44-178) */
void dnso_momentum(const dnso_t *s, double *qx, double *qy, double *qz,
                   const double *ux, const double *uy, const double *uz,
                   double A, double dt);
/* pressuregrad_component! (src/operators.jl:180-216) */
void dnso_pressuregrad(const dnso_t *s, double *phi, const double *p, int c,
                       double scale);
/* poisson! (src/poisson.jl:147-161): solves with r as the right-hand side
 * and writes the interior of the ghosted p (halos untouched). */
void dnso_poisson(dnso_t *s, const double *r, double *p);
/* project! (src/timestep.jl:25-31) */
void dnso_project(dnso_t *s, double *ux, double *uy, double *uz, double *psi);
/* imex_update! (src/ydiffusion.jl:119-154) */
void dnso_imex_update(dnso_t *s, double *ux, double *uy, double *uz,
                      const double *qx, const double *qy, const double *qz,
                      const double *p, double B, double alpha, double dt);
/* step! (src/timestep.jl:41-63) */
void dnso_step(dnso_t *s, double *ux, double *uy, double *uz, double *p,
               double *qx, double *qy, double *qz, double *delta, double dt);
/* cfl_timestep (src/timestep.jl:69-80) */
double dnso_cfl(const dnso_t *s, const double *ux, const double *uy,
                const double *uz, double cfl);
/* maxdiv, kinetic_energy (src/fields.jl:38-60) */
double dnso_maxdiv(dnso_t *s, const double *ux, const double *uy,
                   const double *uz);
double dnso_kinetic_energy(const dnso_t *s, const double *ux, const double *uy,
                           const double *uz);

/* sample_channelstats! plane sums (src/stats.jl:39-58).  acc holds
 * 8 arrays: Uc, Wc, uuc, wwc (ny each) then Vf, vvf, Uf, uvf (nf each),
 * nf = ny-1 (walls) or ny. */
void dnso_channel_sample(const dnso_t *s, const double *ux, const double *uy,
                         const double *uz, double *acc);
/* sample_spectrum! + binshells! (src/stats.jl:120-157); E has nbins entries */
void dnso_spectrum_sample(dnso_t *s, const double *ux, const double *uy,
                          const double *uz, double *E, int nbins);

/* FFT hooks for the oracle's own tests: forward unnormalised, inverse
 * normalised by 1/n (AbstractFFTs conventions). */
void dnso_cfft(int n, int howmany, int inverse, double _Complex *data);
void dnso_rfft(int n, int howmany, const double *in, double _Complex *out);
void dnso_irfft(int n, int howmany, const double _Complex *in, double *out);

/* splitmix64 counter-based noise after src/spectral/ic.jl:31-45, on the
 * active DOFs of component c: amp*(2U-1), U = ((r>>11)+0.5)*2^-53,
 * r = splitmix64(seed + key), key over global staggered indices. */
void dnso_noise(const dnso_t *s, double *phi, int c, unsigned long long seed,
                double amp);

#ifdef __cplusplus
}
#endif
#endif
