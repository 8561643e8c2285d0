/*
 * dnsb.h -- C ABI of libdnsb.so, the B200 (sm_100a) finite-volume time step.
 *
 * Drop-in for the single-GPU hot path of DistributedNavierStokes
 * (Julia): the functions below replace, one for one, the reference's
 * operator API for that path.  Each entry point cites the reference
 * function it stands in for (file:line in the reference repository).
 *
 * Fields are borrowed DEVICE pointers to the caller's ghosted arrays,
 * exactly the reference's `scalarfield` layout (src/fields.jl:4-5):
 * (nx+2) x (ny+2) x (nz+2) doubles, column-major (x fastest), ghost width 1.
 * A CuArray{Float64,3} from `scalarfield(setup)` can be passed as-is
 * (pointer(u.x)).  The library never frees them.  Scratch (spectrum, FFT
 * twiddles, coefficient tables, y-solve work) belongs to the context.
 *
 * Every call returns 0 on success or a DNSB_E* code; dnsb_last_error()
 * gives the message.  Work is enqueued on the context's stream; calls that
 * return a host scalar (dnsb_cfl, dnsb_maxdiv, dnsb_kinetic_energy)
 * synchronise that stream, as the reference's reductions do.  A context is
 * not re-entrant: one context per GPU and host thread.
 */
#ifndef DNSB_H
#define DNSB_H

#ifdef __cplusplus
extern "C" {
#endif

#define DNSB_VERSION 1

enum {
  DNSB_OK = 0,
  DNSB_EINVAL = 1,   /* bad configuration or argument */
  DNSB_ECUDA = 2,    /* CUDA runtime error */
  DNSB_EUNSUP = 3,   /* size the kernels do not support (e.g. FFT length) */
  DNSB_ENOMEM = 4
};

enum { DNSB_STAG_X = 0, DNSB_STAG_Y = 1, DNSB_STAG_Z = 2, DNSB_STAG_P = 3 };
enum { DNSB_BC_PERIODIC = 0, DNSB_BC_WALL = 1 };
enum { DNSB_YDIFF_EXPLICIT = 0, DNSB_YDIFF_IMPLICIT = 1 };

/* The problem description that setup() builds (src/setup.jl:34-113) and
 * that griddata() computes (src/setup.jl:148-193), single rank, w = 1.
 * dy/dyu are copied at create time. */
typedef struct {
  int nx, ny, nz;        /* cells; nx even; FFT lengths nx/2, nz (and ny when
                            periodic) must factor into 2, 3, 5 */
  int bc_y;              /* DNSB_BC_PERIODIC or DNSB_BC_WALL (bc[2]) */
  int ydiffusion;        /* DNSB_YDIFF_* (setup keyword ydiffusion) */
  double dx, dz;         /* grid.Δx, grid.Δz */
  const double *dy;      /* grid.Δy: ny+2 cell widths, ghosted index 0..ny+1 */
  const double *dyu;     /* grid.Δyu: ny+2 centre distances */
  double visc;           /* setup.visc */
  double bodyforce[3];   /* setup.bodyforce */
} dnsb_grid;

typedef struct dnsb_ctx dnsb_ctx;

/* Launch shapes of a context (no counterpart in the reference; the
 * autotuner of the batched ensemble picks them per grid).  0 keeps the
 * default (or the DNSB_* environment override): lines per CTA of the
 * Stockham x-, z- and y-transforms and of the four-step z-transform, the
 * block shape of the per-cell kernels (cell_bx a multiple of 32,
 * cell_bx * cell_by <= 256), z-planes per CTA of the fused projection +
 * momentum.  Results do not depend on them (every line and cell is computed
 * by the same arithmetic). */
typedef struct {
  int lines_x, lines_z, lines_y, lines_z4;
  int cell_bx, cell_by;
  int gm_planes;
} dnsb_tuning;

/* Library version (DNSB_VERSION). */
int dnsb_version(void);

/* setup(; ...) plans: plan_poisson (src/poisson.jl:56-120) and
 * plan_ydiffusion (src/ydiffusion.jl:54-68).  `stream` is a cudaStream_t
 * (NULL = legacy default stream) on device `device`. */
int dnsb_create(const dnsb_grid *grid, int device, void *stream, dnsb_ctx **out);
/* dnsb_create with explicit launch shapes (tuning may be NULL); the shapes
 * in effect (after the clamps to the grid) are read back by
 * dnsb_get_tuning. */
int dnsb_create_tuned(const dnsb_grid *grid, const dnsb_tuning *tuning, int device, void *stream,
                      dnsb_ctx **out);
int dnsb_get_tuning(const dnsb_ctx *ctx, dnsb_tuning *out);
void dnsb_destroy(dnsb_ctx *ctx);
/* Message of the last failed call on ctx (or of the last failed create when
 * ctx is NULL). */
const char *dnsb_last_error(const dnsb_ctx *ctx);
int dnsb_set_stream(dnsb_ctx *ctx, void *stream);
/* Synchronises the context's stream; returns DNSB_ECUDA if a kernel's
 * bounded device-side wait ran out since the last check (and clears it). */
int dnsb_sync(dnsb_ctx *ctx);
/* Poll limit of every device-side wait of this context's kernels (default
 * 2^26; 0 makes every such wait give up at once).  The only device-side
 * waits are the mbarrier waits of the opt-in persistent TMA z-transform
 * (DNSB_TMA=1); a wait that runs out makes its CTA drain its copies in
 * flight and return, and the next dnsb_sync reports it.  The reference's
 * FV path has no device-side waits (no counterpart). */
int dnsb_set_wait_limit(dnsb_ctx *ctx, unsigned long polls);

/* exchange_halo!(φ, stag, setup), single rank (src/halo.jl:81-126). */
int dnsb_fill_ghosts(dnsb_ctx *ctx, double *phi, int stag);

/* divergence!(r, u, setup) (src/operators.jl:29-42); r ghost-free
 * nx*ny*nz, x fastest. */
int dnsb_divergence(dnsb_ctx *ctx, double *r, const double *ux, const double *uy,
                    const double *uz);

/* momentum!(q, u, A, Δt, setup) (src/operators.jl:155-178). */
int dnsb_momentum(dnsb_ctx *ctx, double *qx, double *qy, double *qz, const double *ux,
                  const double *uy, const double *uz, double A, double dt);

/* pressuregrad_component!(φ, p, c, s, setup) (src/operators.jl:204-216). */
int dnsb_pressuregrad(dnsb_ctx *ctx, double *phi, const double *p, int c, double s);

/* poisson!(p, setup) (src/poisson.jl:147-161) with the right-hand side r
 * (the reference's setup.poisson.r): writes the interior of p, no halos. */
int dnsb_poisson(dnsb_ctx *ctx, const double *r, double *p);

/* z-slab decomposition (the reference's (P,1) process grid, z split over
 * ranks; transpose.jl:47-122 redistributes the spectrum between the FFT
 * directions): poisson! (src/poisson.jl:147-161) in three pieces between
 * which the caller moves the spectrum across ranks.
 * dnsb_poisson_x: rfft in x of the ghost-free local r (nx*ny*nz_local) into
 *   the context's spectrum, layout [kx][j][z] (z fastest), nx/2+1 kx planes;
 * dnsb_poisson_zy: on a context of the GLOBAL grid, the z-transform, the
 *   y-solve (solve_y!, poisson.jl:122-140, with the kx-dependent tables
 *   offset to kx0) and the inverse z-transform of the caller's kx-slab S
 *   holding planes kx0..kx0+nkx-1 with every z: [kx-kx0][j][z];
 * dnsb_poisson_xinv: the normalised inverse x-transform of the context's
 *   spectrum into p's interior with its x and y images (z ghosts are the
 *   caller's halo exchange);
 * dnsb_spectrum: the context's spectrum buffer and its dims;
 * dnsb_zblock_copy: dst[kx][j][z_dst + z] = src[kx][j][z_src + z] for
 *   z < nz_copy (complex values; lines of nz_dst and nz_src), the pack /
 *   unpack of the spectrum transposes.  Asynchronous on the context's
 *   stream. */
/* y += a x on the interior cells of two ghosted fields (the lagged-pressure
 * update p += delta / (alpha dt) of step!, src/timestep.jl:49-52, when the
 * stage is assembled from the pieces above); halos are the caller's. */
int dnsb_axpy(dnsb_ctx *ctx, double *y, const double *x, double a);
int dnsb_poisson_x(dnsb_ctx *ctx, const double *r);
int dnsb_poisson_zy(dnsb_ctx *ctx, void *S, int kx0, int nkx);
int dnsb_poisson_xinv(dnsb_ctx *ctx, double *p);
int dnsb_spectrum(dnsb_ctx *ctx, void **S, int *nkx, int *ny, int *nz);
int dnsb_zblock_copy(dnsb_ctx *ctx, void *dst, const void *src, int nkx, int ny, int nz_dst,
                     int z_dst, int nz_src, int z_src, int nz_copy);

/* project!(u, ψ, setup) (src/timestep.jl:25-31): u and ψ leave with valid
 * halos. */
int dnsb_project(dnsb_ctx *ctx, double *ux, double *uy, double *uz, double *psi);

/* The explicit stage of step! (src/timestep.jl:52-57, after momentum!
 * set q <- A q + dt F(u)) with a sub-filter-stress closure, on a periodic
 * box: q += dt f, f = -div(tau) on the staggered faces (normal stresses
 * differenced across each face, shear stresses averaged onto the cell
 * edges), then u += B q with the ghost images of u rewritten.  tau: DEVICE
 * [6][nz][ny][nx] cell-centred components xx, yy, zz, xy, yz, zx (e.g.
 * from dnsb_cnn_infer; periodic boxes only); NULL gives the plain stage
 * update (any box).  The reference has no SFS model. */
int dnsb_sfs_stage(dnsb_ctx *ctx, const double *tau, double *qx, double *qy, double *qz,
                   double *ux, double *uy, double *uz, double dt, double B);

/* imex_update!(u, q, p, B, α, Δt, setup) (src/ydiffusion.jl:119-154). */
int dnsb_imex_update(dnsb_ctx *ctx, double *ux, double *uy, double *uz, const double *qx,
                     const double *qy, const double *qz, const double *p, double B,
                     double alpha, double dt);

/* step!(u, p, q, δ, setup, Δt) (src/timestep.jl:41-63).  δ is scratch in
 * explicit mode (the reference aliases it to p there); pass p or NULL. */
int dnsb_step(dnsb_ctx *ctx, double *ux, double *uy, double *uz, double *p, double *qx,
              double *qy, double *qz, double *delta, double dt);

/* cfl_timestep(u, setup; cfl) (src/timestep.jl:69-80).  With
 * use_step_max != 0 the velocity maxima reduced by the last dnsb_step on
 * these same fields are reused (valid only if u was not modified since). */
int dnsb_cfl(dnsb_ctx *ctx, const double *ux, const double *uy, const double *uz, double cfl,
             int use_step_max, double *dt_out);

/* solve!(; u, setup, tlims, Δt, cfl) (src/timestep.jl:92-111) without
 * processors: initial halo + projection, then steps until t1 (or until
 * max_steps).  dt > 0 fixes the step, dt <= 0 is CFL-adaptive.  p, q and
 * delta are caller scratch fields (delta may be NULL in explicit mode).
 * Reports the final time and the number of steps. */
int dnsb_solve(dnsb_ctx *ctx, double *ux, double *uy, double *uz, double *p, double *qx,
               double *qy, double *qz, double *delta, double t0, double t1, double dt,
               double cfl, long max_steps, double *t_out, long *n_out);

/* The same with HOST arrays for u (in/out) and p (out): the velocity is
 * copied to the device, solved, and u, p copied back (for callers without
 * device arrays; pinned host memory makes the copies faster).  The device
 * fields (7-8 ghosted fields) are allocated on the first call and kept by
 * the context until dnsb_destroy. */
int dnsb_solve_host(dnsb_ctx *ctx, double *ux, double *uy, double *uz, double *p, double t0,
                    double t1, double dt, double cfl, long max_steps, double *t_out,
                    long *n_out);

/* maxdiv(u, setup) (src/fields.jl:38-42). */
int dnsb_maxdiv(dnsb_ctx *ctx, const double *ux, const double *uy, const double *uz,
                double *out);

/* kinetic_energy(u, setup) (src/fields.jl:45-60). */
int dnsb_kinetic_energy(dnsb_ctx *ctx, const double *ux, const double *uy, const double *uz,
                        double *out);

/* sample_channelstats! (src/stats.jl:39-58): adds the (x, z) plane sums of
 * (U, W, uu, ww) on the ny cell rows and (V, vv, Uf, uv) on the nf active
 * face rows (nf = ny-1 with walls) to the DEVICE accumulator acc
 * (4*ny + 4*nf doubles, in that order). */
int dnsb_channel_sample(dnsb_ctx *ctx, const double *ux, const double *uy, const double *uz,
                        double *acc);

/* sample_spectrum! + binshells! (src/stats.jl:120-157): adds the shell
 * energies of u to the DEVICE array E (nbins doubles); periodic boxes only. */
int dnsb_spectrum_sample(dnsb_ctx *ctx, const double *ux, const double *uy, const double *uz,
                         double *E, int nbins);

/* Counter-based noise on the active DOFs of component c (a channel initial
 * condition; hash after src/spectral/ic.jl:31-45): φ += amp*(2U-1) with
 * U = ((splitmix64(seed + key) >> 11) + 0.5) * 2^-53 and
 * key = ((c*nz + K-1)*ny + J-1)*nx + I-1. */
int dnsb_noise(dnsb_ctx *ctx, double *phi, int c, unsigned long long seed, double amp);

/* Integer-wavenumber shells of a fully periodic box (EINVAL with walls).
 * The reference defines them on its pseudo-spectral state
 * (src/spectral/forcing.jl:1-56, src/spectral/ic.jl:53-84); these are the
 * finite-volume counterparts, with no FV entry point in the reference to
 * replace.  Every velocity component is transformed on its own staggered
 * grid; shell s holds the modes with s <= |k| < s+1 (k the integer
 * wavenumber vector), energies are (1/2)|u_hat|^2 / N^2 with the rfft
 * double-counting weights, so their sum is the mean kinetic energy. */

/* Number of shells a box has: floor(|k|max) + 1, |k|max the Nyquist corner. */
int dnsb_shell_count(const dnsb_ctx *ctx);

/* shell_energies (src/spectral/forcing.jl:12-24) for shells 0..nshells-1
 * into the HOST array E; synchronises the stream. */
int dnsb_shell_energies(dnsb_ctx *ctx, const double *ux, const double *uy, const double *uz,
                        double *E, int nshells);

/* rescale_shell! (src/spectral/forcing.jl:26-35) for shells 0..nshells-1
 * at once: shell s times the HOST factor factors[s]; ghost images rewritten.
 * Real factors keep the discrete divergence. */
int dnsb_shell_rescale(dnsb_ctx *ctx, double *ux, double *uy, double *uz, const double *factors,
                       int nshells);

/* spectral_randomfield! (src/spectral/ic.jl:53-84): Gaussian counter-based
 * noise on the interior of every component (Box-Muller of two splitmix64
 * uniforms, key = ((c*nz + K-1)*ny + J-1)*nx + I-1 as in noise_kernel!,
 * src/spectral/ic.jl:37-51), ghosts filled, projected onto discretely
 * divergence-free fields, then every shell s < dnsb_shell_count rescaled
 * to energy totalenergy * profile[s] / sum(profile) (factor 0 where the
 * projected field has none).  profile = NULL uses k^4 exp(-2 (k/kpeak)^2);
 * otherwise profile[0..nprofile) (shells beyond are 0).  Synchronises. */
int dnsb_random_field(dnsb_ctx *ctx, double *ux, double *uy, double *uz, double totalenergy,
                      double kpeak, unsigned long long seed, const double *profile, int nprofile);

/* The distributed half of sfs_sample! (src/spectral/les.jl:313-334) on the
 * FV state of a periodic box: the cell-centred velocity v_c (average of the
 * two faces of each cell, as operators.jl:71-72; u needs valid halos), its
 * six products v_i v_j, their transforms scaled by 1/N (u_hat = F[u]/N),
 * and the LES cube |k_i| <= M/2 of each (lesboxes / lescoarse,
 * src/spectral/les.jl:146-168) written to the HOST array out as 9 coarse
 * rfft arrays of (M/2+1) x M x M complex values (interleaved re, im; kx
 * fastest, ky and kz wrapped 0..M/2-1 then -M/2..-1), in the order
 * u_hat x, y, z, sigma_hat xx, yy, zz, xy, yz, zx.  M even, M/2 <= n/2.
 * The reference gathers these to rank 0 and post-processes them on the
 * host (filter, truncation, coarse nonlinearity, tau); so does the mirror
 * (api.sfs_sample).  Synchronises. */
int dnsb_les_cube(dnsb_ctx *ctx, const double *ux, const double *uy, const double *uz, int M,
                  double *out);

/* The closure of shellforcing (src/spectral/forcing.jl:37-56): shells s
 * with eref[s] >= 0 are rescaled to energy eref[s] (unchanged where they
 * hold none), shells with eref[s] < 0 are not forced.  Energies, factors
 * and the rescale stay on the device (no host synchronisation once eref
 * is uploaded; a changed eref is uploaded synchronously, and the first call
 * allocates scratch that the context keeps: make it outside a stream
 * capture).  With nshells <= 4 the modes are formed by direct partial
 * Fourier sums (one read and one update pass per component); otherwise
 * each component is transformed once and back. */
int dnsb_shell_clamp(dnsb_ctx *ctx, double *ux, double *uy, double *uz, const double *eref,
                     int nshells);

/* Allocation-free Poisson solve (no counterpart in the reference): the same
 * computation as dnsb_poisson(ctx, r, p) for callers that cannot allocate
 * device memory -- e.g. callers whose device memory is held by a pooling
 * allocator with a hard cap (a foreign cudaMalloc may fail or force a pool
 * flush), or timed loops that cannot afford the implicit synchronisation of
 * cudaMalloc/cudaFree -- and that therefore cannot create a context.  It
 * needs no dnsb_ctx: the spectrum, the y-solve work array and all tables
 * live in one fixed file-scope device array (about 26 MB, held by every GPU
 * that loads the library until the process exits).  Limits: nx, ny, nz <=
 * 4096 and (nx/2+1)*ny*nz <= 1048576 (e.g. 96^3 or 128x128x64); larger
 * grids are rejected with DNSB_EUNSUP.  r (ghost-free nx*ny*nz) and p
 * (ghosted; its interior is written, no halos) are the caller's device
 * arrays on the current device; work is enqueued on `stream`.  The first
 * call on a device sets up: it resolves the scratch array's device address
 * (cudaGetSymbolAddress), sets kernel attributes and uploads the grid's
 * tables from host memory, synchronising `stream`; make that first call
 * before any stream capture.  A later call whose grid (sizes, boundary,
 * spacings, dy, dyu) differs from the previous call's on that device
 * uploads the tables again and synchronises `stream` as well; a call with
 * the same grid only enqueues its five kernels.  Every call reuses the same
 * scratch (nothing in it needs to start at zero; each call rewrites what it
 * reads): calls that overlap on the GPU (other streams, other host threads)
 * race.  The transforms are those of dnsb_poisson's Stockham path; with
 * walls the y-solve is the one-thread-per-line Thomas kernel.  Errors are
 * reported by dnsb_last_error(NULL). */
int dnsb_poisson_noalloc(const dnsb_grid *grid, const double *r, double *p, void *stream);

/* Ensembles (no counterpart in the reference; a batched ensemble of
 * periodic boxes): n independent members, each a context of its
 * own grid and viscosity with its own stream.  dnsb_ensemble_run advances
 * every member nsteps RK3 steps with a fixed step dts[i] (dnsb_step on each
 * member) in ONE graph launch: the graph is a conditional while loop whose
 * body is one step of all members (member branches concurrent, fork/join
 * from an internal stream ordered after and before the caller's stream)
 * followed by a countdown kernel.  fields holds 8 device pointers per
 * member: ux, uy, uz, p, qx, qy, qz, delta (delta NULL for an explicit
 * member).  The graph is captured again only when the pointers, steps or
 * forcing change (the step count is a device counter, set per call).
 * Results equal those of stepping each member alone.
 * dnsb_ensemble_create_tuned takes one launch-shape tuning per member
 * (NULL: defaults). */
typedef struct dnsb_ensemble dnsb_ensemble;
int dnsb_ensemble_create(int n, const dnsb_grid *grids, int device, void *stream,
                         dnsb_ensemble **out);
int dnsb_ensemble_create_tuned(int n, const dnsb_grid *grids, const dnsb_tuning *tunings,
                               int device, void *stream, dnsb_ensemble **out);
void dnsb_ensemble_destroy(dnsb_ensemble *ens);
const char *dnsb_ensemble_last_error(const dnsb_ensemble *ens);
/* Context of member i (for the per-member calls: cfl, noise, project, ...). */
dnsb_ctx *dnsb_ensemble_member(dnsb_ensemble *ens, int i);
int dnsb_ensemble_run(dnsb_ensemble *ens, double *const *fields, const double *dts, long nsteps);
/* Shell-clamp forcing of member i after each of its steps (as
 * dnsb_shell_clamp with the table eref[0..nshells), uploaded here; periodic
 * members only); eref = NULL removes it.  The graph is re-captured on the
 * next run when the forcing changes. */
int dnsb_ensemble_forcing(dnsb_ensemble *ens, int i, const double *eref, int nshells);

/* The pseudo-spectral solver of a periodic cube (the reference's second
 * solver, src/spectral/*.jl): transform grid n^3 (even; FFT lengths with
 * factors 2, 3, 5), side l, viscosity visc, truncation kcut (<= 0: n/3;
 * 3 kcut <= n).  The state uh is the reference's compact spectrum
 * (spectral_setup, src/spectral/setup.jl:62-73): 3 components, each
 * (kcut+1) x m x m complex values (interleaved re, im), m = 2 kcut + 1,
 * column-major with kx = 0..kcut fastest, ky and kz in compact fftfreq order
 * (0..kcut, then -kcut..-1); u_hat = F[u] / n^3.  Physical fields are 3
 * real n^3 arrays (x fastest) at the cell centres (i - 1/2) l / n.
 * Device pointers; work on the solver's stream; errors as elsewhere, with
 * dnsb_spectral_last_error. */
typedef struct dnsb_spectral dnsb_spectral;
int dnsb_spectral_create(int n, int kcut, double l, double visc, int device, void *stream,
                         dnsb_spectral **out);
void dnsb_spectral_destroy(dnsb_spectral *sp);
const char *dnsb_spectral_last_error(const dnsb_spectral *sp);
int dnsb_spectral_set_stream(dnsb_spectral *sp, void *stream);
/* Compact values per component, (kcut+1) m^2. */
long dnsb_spectral_size(const dnsb_spectral *sp);
/* spec_to_phys! (src/spectral/fft.jl): v = the physical velocity of uh. */
int dnsb_spectral_to_phys(dnsb_spectral *sp, const double *uh, double *v);
/* phys_to_spec! + truncation: uh = the retained modes of F[v] / n^3. */
int dnsb_spectral_from_phys(dnsb_spectral *sp, const double *v, double *uh);
/* spectral_rhs! (src/spectral/operators.jl:66-96): du = -i k_j F[v_i v_j] / n^3. */
int dnsb_spectral_rhs(dnsb_spectral *sp, const double *uh, double *du);
/* spectral_project! (src/spectral/operators.jl:10-29). */
int dnsb_spectral_project(dnsb_spectral *sp, double *uh);
/* spectral_step! (src/spectral/step.jl:60-92): one Wray RK3 step with the
 * integrating-factor viscosity, projected after every stage; vmax_out
 * (optional, synchronises) = vsummax of the first stage's velocity. */
int dnsb_spectral_step(dnsb_spectral *sp, double *uh, double dt, double *vmax_out);
/* vsummax of the physical velocity of uh (src/spectral/step.jl:45-58). */
int dnsb_spectral_vsummax(dnsb_spectral *sp, const double *uh, double *out);
/* Integer shells floor(|k|) of the spectral state (src/spectral/forcing.jl):
 * count = floor(sqrt(3) kcut) + 1; energies into the HOST array E (fixed
 * summation order); rescale by HOST factors; spectral_randomfield!
 * (src/spectral/ic.jl:53-84: Gaussian counter-based noise on the n^3 grid
 * with noise_kernel!'s key, phys_to_spec!, projection, every shell rescaled
 * to totalenergy * profile[s] / sum(profile), profile = NULL: k^4
 * exp(-2 (k/kpeak)^2)); and the closure of shellforcing (:37-56) with the
 * table eref (eref[s] < 0: shell s not forced), on the device. */
int dnsb_spectral_shell_count(const dnsb_spectral *sp);
int dnsb_spectral_shell_energies(dnsb_spectral *sp, const double *uh, double *E, int nshells);
int dnsb_spectral_shell_rescale(dnsb_spectral *sp, double *uh, const double *factors, int nshells);
int dnsb_spectral_random_field(dnsb_spectral *sp, double *uh, double totalenergy, double kpeak,
                               unsigned long long seed, const double *profile, int nprofile);
int dnsb_spectral_shell_clamp(dnsb_spectral *sp, double *uh, const double *eref, int nshells);
/* The distributed half of sfs_sample! (src/spectral/les.jl:313-334): the
 * LES cube |k_i| <= M/2 (M even, M/2 <= kcut) of u_hat (a truncation of
 * the state) and of sigma_hat = F[v_i v_j] / n^3 (products on the n^3
 * grid), into the HOST array out as in dnsb_les_cube.  Synchronises. */
int dnsb_spectral_les_cube(dnsb_spectral *sp, const double *uh, int M, double *out);
/* spectral_phaserandomize! (src/spectral/ic.jl:98-143): every retained
 * mode but the mean times a counter-based unit-modulus phase (Hermitian-safe
 * in the kx = 0 plane); |u_hat| and k . u_hat = 0 are preserved. */
int dnsb_spectral_phaserandomize(dnsb_spectral *sp, double *uh, unsigned long long seed);
/* which = 0: spectral_energy, 1: spectral_dissipation, 2: spectral_maxdiv
 * (src/spectral/operators.jl:98-110), single rank.  Synchronises. */
int dnsb_spectral_diagnostic(dnsb_spectral *sp, const double *uh, int which, double *out);

/* Instrumentation (no counterpart in the reference, which has no profiling
 * for the FV path): launches are counted always; with dnsb_profile(ctx, 1)
 * every launch of the step path is bracketed by CUDA events on the context's
 * stream and its device time is accumulated per kernel kind.  Enabling
 * resets the accumulators; dnsb_profile_read synchronises.  GRADMOM is the
 * projection of a semi-implicit stage fused with the next stage's momentum;
 * ZYZ the z-FFT, y-solve and inverse z-FFT of wall-bounded grids in one
 * kernel (one thread-block cluster per kx plane). */
enum {
  DNSB_KIND_MOMENTUM = 0, DNSB_KIND_CN = 1, DNSB_KIND_RFFTX = 2, DNSB_KIND_FFTZ = 3,
  DNSB_KIND_YSOLVE = 4, DNSB_KIND_IFFTZ = 5, DNSB_KIND_IRFFTX = 6, DNSB_KIND_GRAD = 7,
  DNSB_KIND_OTHER = 8, DNSB_KIND_GRADMOM = 9, DNSB_KIND_ZYZ = 10, DNSB_NKINDS = 11
};
int dnsb_profile(dnsb_ctx *ctx, int enable);
int dnsb_profile_read(dnsb_ctx *ctx, int kind, double *ms, long *launches);
long dnsb_launch_count(const dnsb_ctx *ctx);
const char *dnsb_kind_name(int kind);

#ifdef __cplusplus
}
#endif
#endif
