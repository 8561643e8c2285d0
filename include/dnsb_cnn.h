/*
 * dnsb_cnn.h -- C ABI of the sub-filter-stress CNN closure in libdnsb.so.
 *
 * No counterpart in the reference: DistributedNavierStokes has no learned
 * closure.  Its data pipeline is the reference's (filtered velocity u_bar and
 * trace-free sub-filter stress tau = filter(u u) - u_bar u_bar from
 * sfs_sample!, src/spectral/les.jl:302-370; Gaussian filter
 * exp(-Delta^2 k^2 / 24), :77), and its training pairs come from the
 * library's own DNS (dnsb_les_cube + the host half of the sampler).
 *
 * The network: 4 convolution layers, 3x3x3 kernels, channels 3 -> 32 -> 32
 * -> 32 -> 6, bias, GELU (tanh form) after the first three, periodic padding on
 * the full periodic field.  BF16 weights / activations / gradients, FP32
 * accumulation on the tensor cores (tcgen05.mma, accumulators in tensor
 * memory, operands staged by TMA), FP32 master weights and Adam state.
 * Training batches are `batch` crops of side `crop` taken with a halo of 4
 * cells from their periodic parent field, so a crop's outputs equal the
 * full field's.  Loss: mean squared error of the 6 stress components, each
 * normalised by the scale given to dnsb_cnn_set_scales.
 *
 * Parameters (FP32, dnsb_cnn_param_count values): per layer L = 1..4,
 * W[27][cout][cin] (tap t = (dz * 3 + dy) * 3 + dx, the input voxel of output
 * (x, y, z) for tap t being (x + dx - 1, y + dy - 1, z + dz - 1) on the
 * periodic field), then b[cout].
 *
 * Every call returns 0 or a DNSB_E* code (include/dnsb.h); the message is
 * dnsb_cnn_last_error().  Work is enqueued on the closure's stream; calls
 * returning host data synchronise it.  A device-side wait that runs out
 * (bounded mbarrier waits in the tensor-core kernels) is reported as
 * DNSB_ECUDA by the next synchronising call.
 */
#ifndef DNSB_CNN_H
#define DNSB_CNN_H

#include "dnsb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dnsb_cnn dnsb_cnn;

/* Training geometry: `batch` crops of side `crop`; inference geometry: a
 * periodic field of side `nfield` (0: none).  Either may be 0 to leave that
 * part out.  Sides from 8 to about 96 (a convolution's ring of at least 4
 * staged input planes, each 4 chunks x 5-12 rows x (side + 8) voxels x 16
 * bytes, plus the layer's 55 KB of weights must fit in shared memory):
 * DNSB_EUNSUP otherwise. */
int dnsb_cnn_create(int device, void *stream, int batch, int crop, int nfield, dnsb_cnn **out);
void dnsb_cnn_destroy(dnsb_cnn *cnn);
const char *dnsb_cnn_last_error(const dnsb_cnn *cnn);
int dnsb_cnn_set_stream(dnsb_cnn *cnn, void *stream);
int dnsb_cnn_sync(dnsb_cnn *cnn);
long dnsb_cnn_launch_count(const dnsb_cnn *cnn);

/* Number of FP32 parameters (63174). */
int dnsb_cnn_param_count(const dnsb_cnn *cnn);
/* Uniform(-1/sqrt(27 cin), +1/sqrt(27 cin)) weights and biases from the
 * splitmix64 stream of `seed` (key = parameter index, the uniform mapping
 * of src/spectral/ic.jl:31-45); resets Adam. */
int dnsb_cnn_init(dnsb_cnn *cnn, unsigned long long seed);
/* HOST arrays of dnsb_cnn_param_count floats; set resets Adam. */
int dnsb_cnn_set_params(dnsb_cnn *cnn, const float *params);
int dnsb_cnn_get_params(dnsb_cnn *cnn, float *params);
/* Input scale (multiplies u_bar's 3 components before the network) and
 * output scale (multiplies the network's 6 outputs to give tau). */
int dnsb_cnn_set_scales(dnsb_cnn *cnn, const float *in_scale3, const float *out_scale6);

/* Training data: DEVICE array [nsnap][9][n][n][n] FP32 (x fastest): per
 * snapshot the normalised u_bar x, y, z and tau xx, yy, zz, xy, yz, zx at the
 * cell centres of the periodic n^3 grid.  Borrowed until replaced. */
int dnsb_cnn_set_dataset(dnsb_cnn *cnn, const float *data, int nsnap, int n);
/* nsteps Adam steps (lr; beta1 0.9, beta2 0.999, eps 1e-8) on random crops
 * of the dataset (snapshot and origin from splitmix64 of (seed, step,
 * sample)); each step's loss goes to the loss history.  Asynchronous. */
int dnsb_cnn_train(dnsb_cnn *cnn, int nsteps, float lr, unsigned long long seed);
/* Steps taken so far, and the loss history (HOST out, losses of steps
 * first .. first+count-1).  Synchronise. */
int dnsb_cnn_steps(dnsb_cnn *cnn, long *steps);
int dnsb_cnn_losses(dnsb_cnn *cnn, float *out, long first, long count);

/* One forward + backward pass on a caller batch (DEVICE arrays: x
 * [batch][3][P][P][P] FP32 with P = crop + 8, the crops with their halo; t
 * [batch][6][crop][crop][crop] FP32 normalised targets): the loss (HOST)
 * and the gradient of every parameter (HOST, dnsb_cnn_param_count floats;
 * NULL to skip).  With nadam > 0 it also takes nadam Adam steps on that
 * batch (loss and gradients of the first).  Synchronises. */
int dnsb_cnn_batch(dnsb_cnn *cnn, const float *x, const float *t, int nadam, float lr,
                   float *loss_out, float *grads_out);

/* The network on the periodic field of side nfield.  dnsb_cnn_infer_cells:
 * DEVICE v[3][n][n][n] (FP64 cell-centred velocity, x fastest); the FV form:
 * the staggered ghosted fields of a periodic box (the reference's layout,
 * include/dnsb.h), averaged onto the cell centres (operators.jl:71-72).
 * tau: DEVICE [6][n][n][n] FP64, components xx, yy, zz, xy, yz, zx at the
 * cell centres.  Asynchronous. */
int dnsb_cnn_infer_cells(dnsb_cnn *cnn, const double *v, double *tau);
int dnsb_cnn_infer(dnsb_cnn *cnn, const double *ux, const double *uy, const double *uz,
                   double *tau);

/* The closed LES step on a periodic box (an explicit-mode context whose
 * grid side is the closure's nfield): the RK3 stages of step!
 * (src/timestep.jl:41-63), each evaluating tau(u) with dnsb_cnn_infer and
 * adding its -div(tau) in the stage update (dnsb_momentum, dnsb_sfs_stage,
 * dnsb_project).  tau: DEVICE scratch [6][n][n][n].  cnn NULL: the same
 * three stages without the closure.  The closure is switched to the
 * context's stream.  Asynchronous. */
int dnsb_les_step(dnsb_ctx *ctx, dnsb_cnn *cnn, double *ux, double *uy, double *uz, double *p,
                  double *qx, double *qy, double *qz, double *tau, double dt);
/* CFL-adaptive steps from t0 to exactly t1 (cfl_timestep, timestep.jl:69-80,
 * the last step shortened to land on t1): dnsb_les_step with the closure,
 * or the library's fused dnsb_step when cnn is NULL (the unclosed
 * fallback); after each step the shell-energy clamp dnsb_shell_clamp with
 * the HOST table eref[0..nshells) when eref is not NULL.  Reports t1 and the
 * number of steps.  Where the fields are 16-byte aligned, the box explicit,
 * the clamp the direct one (at most 4 shells) and per-launch timing off, the
 * whole run is one launch of a CUDA graph (a conditional loop whose body
 * computes the CFL step on the device, with the same operations as
 * cfl_timestep here, and runs the step reading it from device memory):
 * the call synchronises once, at the end.  The context keeps the graphs
 * of its last four argument sets (fields, tau, closure, cfl, shell count)
 * and relaunches one for any later interval (a closure created at a
 * destroyed one's address is told apart; fields are matched by address
 * and are the context's shape by contract).  Otherwise (or with the environment variable
 * DNSB_LESGRAPH=0) a host loop synchronises once per step for the CFL
 * maximum.  Both give the same bits. */
int dnsb_les_advance(dnsb_ctx *ctx, dnsb_cnn *cnn, double *ux, double *uy, double *uz, double *p,
                     double *qx, double *qy, double *qz, double *tau, double t0, double t1,
                     double cfl, const double *eref, int nshells, double *t_out, long *n_out);

/* Instrumentation: with enable != 0, CUDA events bracket every tensor-core
 * launch; kind 0 = forward convolutions, 1 = transposed (backward-data)
 * convolutions, 2 = weight gradients, 3 = the rest.  Read synchronises. */
int dnsb_cnn_profile(dnsb_cnn *cnn, int enable);
int dnsb_cnn_profile_read(dnsb_cnn *cnn, int kind, double *ms, long *launches, double *flops);

#ifdef __cplusplus
}
#endif
#endif
