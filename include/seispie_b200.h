/*
 * seispie_b200.h -- C ABI of the B200 (sm_100a) FWI solver library
 * libseispie_b200.so.
 *
 * The library replaces the Numba @cuda.jit kernels and device-side time loops
 * of icui/seispie's fd2d solver plugin (seispie/solver/fd2d/solver.py,
 * seispie/solver/fd2d/fd2d.py, seispie/solver/misfit/waveform.py,
 * seispie/solver/source/ricker.py).  Each entry point below names the
 * reference code it replaces.  All paths in citations are relative to the
 * seispie project root.
 *
 * Conventions
 *   - Every pointer argument is a DEVICE pointer unless stated otherwise.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  All work is enqueued on it; nothing synchronises the host.
 *   - Every function returns 0 on success or a negative FWI_E* code; the
 *     message of the last failure on the calling thread is available from
 *     fwi_last_error().  No function allocates device memory: every buffer,
 *     scratch included, is owned by the caller.
 *   - Wavefield layout: z is contiguous.  A field of one shot is nx rows of
 *     `pitch` floats (pitch >= nz, pitch % 4 == 0, cells [nz, pitch) of a row
 *     are padding that must be zero and stay zero).  A batch stores its shots
 *     back to back: element (shot, i, j) is at shot*nx*pitch + i*pitch + j.
 *     Point positions (sources, receivers) use the reference's cell number
 *     k = i*nz + j (fd2d.py:134, 159).
 */
#ifndef SEISPIE_B200_H
#define SEISPIE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FWI_ABI_VERSION 7

/* status codes */
#define FWI_OK 0
#define FWI_EINVAL (-1)   /* bad argument (null pointer, size, alignment)   */
#define FWI_ECUDA (-2)    /* a CUDA runtime call or kernel launch failed     */
#define FWI_ERANGE (-3)   /* size beyond a documented maximum                */

/* wave types, solver.py:205-234 */
#define FWI_SH 0          /* SH: vy, uy, sxy, szy                            */
#define FWI_PSV 1         /* P-SV: vx, vz, ux, uz, sxx, szz, sxz             */
#define FWI_SPIN 2        /* P-SV plus micropolar spin vy_c, uy_c, sy*_c     */

/*
 * One batch of shots that share a model and a grid.  Field slots:
 *   sig[2][6]  stress, ping-pong pair; SH: {sxy, szy}; P-SV: {sxx, szz, sxz};
 *              spin adds {syx_c, syy_c, syz_c} in slots 3..5
 *   vel[2][3]  velocity, ping-pong pair; SH: {vy}; P-SV: {vx, vz};
 *              spin adds vy_c in slot 2
 *   disp[3]    displacement, updated in place, same slots as vel; all NULL
 *              for a displacement-free batch (fwi_run)
 * `cur` selects which half of each pair holds the current state; fwi_run
 * flips it once per step.
 * Model (shared by all shots, [nx][pitch]; prepared by fwi_prepare_model):
 *   buo = dt/rho, buo_j = dt/j (spin), bound (sponge), lam, mu,
 *   nu, mnc = mu_c + nu_c (spin).
 * Injection (per shot, CSR): the entries of shot s are inj_ptr[s] ..
 *   inj_ptr[s+1]-1; entry e adds stf_c[inj_row[e]*nt + it] to the stress
 *   divergence of component c at cell inj_cell[e] (reference numbering)
 *   before the velocity update, in entry order (stf_dsy / stf_dsxz,
 *   solver.py:78-93).  Component pointers: SH uses stf[1] (y); P-SV uses
 *   stf[0] (x) and stf[2] (z).
 * Receivers: rec_cell[nrec] (reference numbering), recorded into
 *   obs[c][(shot*nrec + r)*nt + it] after each forward step (save_obs,
 *   solver.py:151-156); obs[c] may be NULL to skip a component.
 *   Components: SH obs[1] = uy; P-SV obs[0] = ux, obs[2] = uz;
 *   spin also obs[1] = uy_c.
 * Snapshots (forward; sae > 0): snap_u[c] is [nsa][nshots][nx][pitch]; slot
 *   nsa-(it+1)/sae receives u as it is before step it whenever
 *   (it+1) % sae == 0 (solver.py:193-203).  snap_v[c] (optional) receives v
 *   after that step (solver.py:236-242).  NULL skips.
 * Sensitivity kernels (adjoint; FP64, [nx][pitch], accumulated over every
 *   shot of the batch): k_mu for SH (interaction_muy, solver.py:159-163,
 *   315-321); k_lam, k_mu, k_rho for P-SV.  NULL skips.
 */
typedef struct fwi_batch {
    int mode;                 /* FWI_SH, FWI_PSV or FWI_SPIN                 */
    int nx, nz, pitch;        /* grid; pitch = padded z length               */
    int nshots;               /* shots in this batch                         */
    int nt;                   /* samples per source / receiver trace         */
    float dx, dz;             /* grid spacing (fd2d.py:195-196)              */
    double dt;                /* time step                                   */
    int cur;                  /* current half of the ping-pong pairs (0/1)   */
    int tile;                 /* tile variant (0 = library default)          */
    float *sig[2][6];
    float *vel[2][3];
    float *disp[3];
    const float *buo, *buo_j, *bound, *lam, *mu, *nu, *mnc;
    const int *inj_ptr, *inj_cell, *inj_row;
    const float *stf[3];
    int nrec;
    const int *rec_cell;
    float *obs[3];
    int sae, nsa;
    float *snap_u[3];
    float *snap_v[3];
    double *k_lam, *k_mu, *k_rho;
    /* Exact discrete adjoint (fwi_run_transposed).  Forward runs with these
     * set also store, for every step it with 0 <= it-seg0 < nseg, at slot
     * it-seg0 of [nseg][nshots][nx][pitch] buffers: the terms of the stress
     * update that the new velocity v(it+1) enters through (D+ of it, masked
     * as the stress update uses it) into seg_e[k] -- SH: exy, ezy; P-SV: exx,
     * ezz, exz+ezx; spin: exx, ezz, exz+ezx, -vy_c - (ezx-exz)/2, Dx+ vy_c,
     * Dz+ vy_c -- and the stress divergence including the sources of step it
     * into seg_ds[c] (component slots as obs).  NULL skips. */
    float *seg_e[6];
    float *seg_ds[3];
    int seg0, nseg;
    /* Spin gradients of fwi_run_transposed (FP64 [nx][pitch], NULL skips):
     * dL/dnu, dL/d(mu_c+nu_c), dL/d(dt/j). */
    double *k_nu, *k_mnc, *k_buoj;
    /* Receivers listed by cell: a permutation of 0 .. nrec-1 with
     * rec_cell[rec_order[i]] non-decreasing.  Required by displacement-free
     * forward runs that record traces (see fwi_run). */
    const int *rec_order;
    /* Displacement-free batches: row slots of the row-marching kernel's
     * staging ring, 3, 4, 6 or 8 (0 = chosen from the row length). */
    int ring;
    /* Row-marching step: resident CTAs per SM its grid is sized for (0 =
     * as many as fit).  A smaller grid leaves room on every SM for another
     * kernel running concurrently on a second stream. */
    int ctas_per_sm;
    /* P-SV transposed step (fwi_run_transposed): 0 = tiles of 32 x 64 cells,
     * two z columns per thread; 1 = tiles of 32 x 32 cells, one column per
     * thread.  Same adjoint fields bit for bit. */
    int adj_tile;
    /* 1: programmatic dependent launch between the steps of one fwi_run
     * (row-marching steps) or fwi_run_transposed (P-SV wide tiles) call --
     * each step's kernel is scheduled while the previous step is finishing,
     * hiding launch latency and set-up; every access to the state still
     * waits for the previous step to complete, so the results are
     * bit-identical to 0, which serialises the launches.  Worth it for a
     * time loop that has the GPU to itself; a loop that shares the SMs with
     * another stream's kernels runs faster with 0 (the early CTAs hold SM
     * slots while they wait).  No counterpart in the reference (its steps
     * are separate Numba launches, solver.py:205-234). */
    int step_overlap;
} fwi_batch;

/* ABI version of the loaded library (FWI_ABI_VERSION). */
int fwi_abi_version(void);

/* Binary version (major*10 + minor) of the device code the library runs on
 * the current device, from cudaFuncGetAttributes: 100 for sm_100a.  A
 * negative FWI_ECUDA code without a usable device.  No counterpart in the
 * reference. */
int fwi_binary_version(void);

/* Number of kernels this library has launched in the process so far (for
 * launch accounting by benchmarks).  No counterpart in the reference. */
long long fwi_launch_count(void);

/* Device-side status of the kernels whose waits are bounded (TMA and
 * tensor-core pipelines): *status gets bit 0 if a step or transposed-step
 * kernel gave up a wait, bit 1 if a U-Net kernel did (its outputs are then
 * invalid); clear != 0 resets both.  Synchronous (reads device memory).  No
 * counterpart in the reference. */
int fwi_device_status(int *status, int clear);

/* Poll limit of every bounded wait in the library's kernels (0 restores the
 * default of 2^22 polls, seconds on a B200).  A wait that runs out ends its
 * kernel, which sets bit 0 (step kernels) or bit 1 (U-Net kernels) of
 * fwi_device_status.  Synchronous; process-wide for the current device.  No
 * counterpart in the reference. */
int fwi_set_wait_limit(int polls);

/* Launch a one-thread kernel whose bounded wait runs out (an mbarrier nothing
 * completes; no copy in flight): it sets bit 0 of fwi_device_status and
 * returns.  Tests the failure path without faulting or hanging the GPU.  No
 * counterpart in the reference. */
int fwi_wait_selftest(void *stream);

/* Copy the last error message of the calling thread into buf (always NUL
 * terminated); returns the status code of that error (0 if none). */
int fwi_last_error(char *buf, size_t len);

/* Interior tile (x rows, z columns) of step-kernel variant `tile`
 * (fwi_batch.tile); returns FWI_EINVAL for an unknown variant.  Variant 0
 * is the library default.  No counterpart in the reference (its kernels use
 * a 1-D grid of threads_per_block threads, fd2d.py:184-187). */
int fwi_tile_shape(int tile, int *tx, int *tz);

/* Kind of step-kernel variant `tile`: 0 = one thread per cell walking the
 * tile, staged with cp.async; 1 = lane per z column with an x register
 * window, staged with cp.async; 2 = the same staged with TMA tensor copies
 * (cp.async.bulk.tensor, mbarrier completion).  FWI_EINVAL if unknown.  No
 * counterpart in the reference. */
int fwi_tile_kind(int tile);

/* vp/vs -> lambda/mu in place: lam_io holds vp and mu_io holds vs on entry.
 * Replaces vps2lm, seispie/solver/fd2d/fd2d.py:21-33 (launched at
 * fd2d.py:216).  n elements, any layout. */
int fwi_vps2lm(float *lam_io, float *mu_io, const float *rho, long long n, void *stream);

/* lambda/mu -> vp/vs in place.  Replaces lm2vps, fd2d.py:36-44. */
int fwi_lm2vps(float *vp_io, float *vs_io, const float *rho, long long n, void *stream);

/* Gaussian sponge weights, [nx][pitch].  Replaces set_bound,
 * fd2d.py:47-68 (launched at fd2d.py:225-228). */
int fwi_set_bound(float *bound, int nx, int nz, int pitch, int width, double alpha,
                  int left, int right, int bottom, int top, void *stream);

/* Ricker source-time functions, FP64 arithmetic rounded to float32.
 * params (device, nsrc x 4 doubles: f0, t0, ang [deg], amp) ->
 * stf_x/stf_y/stf_z [nsrc*nt].  Replaces ricker, ricker.py:7-11, and the
 * host loop of import_sources, fd2d.py:136-138. */
int fwi_ricker(const double *params, int nsrc, int nt, double dt,
               float *stf_x, float *stf_y, float *stf_z, void *stream);

/* Derived per-cell model arrays used by fwi_run: buo = dt/rho,
 * buo_j = dt/j, mnc = mu_c + nu_c (the last two only when j / mu_c are
 * non-NULL).  n elements, any layout.  Replaces the per-step divisions of
 * add_vy / add_vxz (solver.py:95-109) and the sum in add_sy_c
 * (solver.py:140-141). */
int fwi_prepare_model(const float *rho, const float *j, const float *mu_c, const float *nu_c,
                      double dt, long long n, float *buo, float *buo_j, float *mnc, void *stream);

/* Advance every shot of the batch by nsteps time steps starting at step it0.
 * adjoint = 0: forward modelling; replaces the time loop of run_forward,
 *   solver.py:192-242 (div_sy/div_sxz/div_sxyz_c, stf_dsy/stf_dsxz,
 *   add_vy/add_vxz, div_vy/div_vxz, add_sy/add_sxz/add_sy_c, save_obs and
 *   the snapshot copies), fused into one kernel launch per step.
 * adjoint = 1: adjoint modelling; replaces run_adjoint, solver.py:290-321
 *   (same step with the adjoint source, plus the interaction kernels every
 *   sae steps with ndt = sae*dt).  Requires the forward snapshots.
 * The caller clears the wavefields first (fwi_clear or cudaMemsetAsync),
 * as clear_wavefields does (fd2d.py:318-341).  b->cur is updated.
 * Displacement-free batches (disp[] all NULL; SH or P-SV forward, nz <= 1024,
 * no snapshots): the displacement, which the reference keeps as a field only
 * to feed save_obs, is not stored.  The step runs on the row-marching kernel
 * and each recorded trace is the running sum u(it) = u(it-1) + v(it) dt of
 * the velocity at its receiver, evaluated in the same float operations as
 * add_vy / add_vxz (solver.py:95-109), so the traces are bit-identical to a
 * run with displacement fields.  Such batches need rec_order when they
 * record, and the injection entries of each shot sorted by cell (entries at
 * one cell keep their relative order, which fixes their summation order). */
int fwi_run(fwi_batch *b, int adjoint, int it0, int nsteps, void *stream);

/* Uneven batches: n independent forward batches of one mode (each with its
 * own grid, model, shots, sources, receivers and nt) stepped together, one
 * launch per time step covering every tile of every running instance.  All
 * start at the same step with the same `cur`; an instance stops after its
 * own nt steps.  workspace: caller device buffer of
 * fwi_multi_workspace_bytes(n) bytes; fwi_multi_prepare uploads the
 * per-instance step arguments into it (synchronously; call it outside stream
 * capture, again whenever a pointer changes) and fwi_multi_run enqueues
 * steps [it0, it0+nsteps) and updates each batch's cur.  Tile variants:
 * 0 or a 32-column register-window variant.  No counterpart in the reference,
 * which runs one model at a time (solver.py:352-373). */
long long fwi_multi_workspace_bytes(int n);
int fwi_multi_prepare(fwi_batch *const *batches, int n, void *workspace);
int fwi_multi_run(fwi_batch *const *batches, int n, void *workspace, int it0, int nsteps, void *stream);

/* Exact discrete adjoint of fwi_run's SH / P-SV / spin forward step, run backwards
 * over forward steps it = it_hi-1 down to it_hi-nsteps on the adjoint state
 * held in the batch's stress and velocity buffers (sig~, v~; cleared by the
 * caller before the last step; disp is not used).  The adjoint displacement
 * u~ is nonzero only at the receivers, where it is the suffix sum over the
 * steps s >= it of dL/d trace(s): stf_c[inj_row[e]*nt + it] holds that value
 * for entry e (fwi_trace_suffix_sum of the trace gradients; rows as for
 * fwi_run's injection, typically one per receiver and shot) and enters v~ as
 * dt * u~ at inj_cell[e].  Each step also accumulates, over every shot, into
 * the FP64 arrays: dL/dlam (k_lam, P-SV and spin), dL/dmu (k_mu), dL/dbuo
 * with buo = dt/rho (k_rho), and for spin k_nu, k_mnc, k_buoj; NULL skips an
 * array.  Needs the forward strain of v(it+1) in seg_e for every step of the
 * range (written by a forward fwi_run over the same segment), and the
 * divergence of step it in seg_ds when k_rho (spin: or k_buoj) is set; a
 * forward run without seg_ds stores 40 % fewer bytes per P-SV step.  No counterpart in
 * the reference, whose adjoint (solver.py:290-329) is the continuous-adjoint
 * approximation fwi_run's adjoint = 1 reproduces. */
int fwi_run_transposed(fwi_batch *b, int it_hi, int nsteps, void *stream);

/* L2 waveform misfit and adjoint source for nshots x nrec traces of nt
 * samples (receiver-major, [shot][rec][t]).  data = observed traces (the
 * reference's `syn`), syn = synthetics (its `obs`).  Writes the
 * time-reversed adjoint source adstf = 2 taper^2 (data - syn) and
 * misfit[shot] = || taper (data - syn) ||_2 accumulated in FP64.
 * partial is caller scratch of fwi_misfit_partials(nrec, nt) doubles per
 * shot.  Replaces diff + waveform, seispie/solver/misfit/waveform.py:5-34. */
int fwi_misfit(const float *data, const float *syn, float *adstf, double *misfit,
               double *partial, int nshots, int nrec, int nt, double dt, void *stream);
long long fwi_misfit_partials(int nrec, int nt);

/* fwi_misfit writing, instead of the time-reversed adjoint source, the
 * derivative of chi = sum taper^2 (syn - data)^2 with respect to every trace
 * sample, in forward time order: grad = 2 taper^2 (syn - data) -- the input
 * of fwi_run_transposed.  misfit[shot] is the same norm as fwi_misfit's.
 * Same taper as waveform.py:11-21. */
int fwi_misfit_tracegrad(const float *data, const float *syn, float *grad, double *misfit, double *partial,
                         int nshots, int nrec, int nt, double dt, void *stream);

/* Suffix sums along time of ntraces traces of nt samples ([trace][t]):
 * out[t] = sum over s >= t of g[s], accumulated in FP64; out may alias g.
 * Turns trace gradients (fwi_misfit_tracegrad) into the injection values of
 * fwi_run_transposed. */
int fwi_trace_suffix_sum(const float *g, float *out, long long ntraces, int nt, void *stream);

/* Source illumination for the learned preconditioner: acc[i] += sum over
 * the nshots fields of f ([nshots][field]) of f^2, accumulated in FP64 in
 * shot order.  No counterpart in the reference. */
int fwi_energy_accumulate(const float *f, int nshots, long long field, double *acc, void *stream);

/* Optimizer vector kernels (float32 vectors of n elements, FP64 arithmetic).
 * fwi_dot: *out = sum x[i]*y[i] in FP64, deterministic; partial is caller
 *   scratch of fwi_reduce_partials() doubles.  Replaces np.dot of
 *   lbfgs.py:37-45, cg.py:20-29, bracket.py:23-30,49-50.
 * fwi_absmax: *out = max |x[i]| (partial: fwi_reduce_partials() floats).
 *   Replaces np.amax(abs(.)), bracket.py:48-49.
 * fwi_axpby: out = a*x + b*y evaluated in FP64, stored float32 (y may be
 *   NULL); out may alias x or y.  Replaces the float64-scalar updates
 *   q -= al*y, q += s*(al-be), m + alpha*p (lbfgs.py:40-46, bracket.py:59). */
long long fwi_reduce_partials(void);
int fwi_dot(const float *x, const float *y, long long n, double *out, double *partial, void *stream);
int fwi_absmax(const float *x, long long n, float *out, float *partial, void *stream);
int fwi_axpby(float *out, double a, const float *x, double b, const float *y, long long n, void *stream);

/* Capacity, in FP64 partial sums, of the fixed scratch of fwi_misfit_noalloc
 * (1 MiB): nshots * fwi_misfit_partials(nrec, nt) must not exceed it. */
#define FWI_MISFIT_NOALLOC_MAX_PARTIALS (1 << 17)

/* fwi_misfit for callers that cannot allocate device memory while they run
 * (an application whose pool owns all device memory after start-up, or a
 * time-critical loop where cudaMalloc/cudaFree would synchronise the device):
 * same arguments and results as fwi_misfit minus `partial`, whose role is
 * taken by a fixed array inside the library (FWI_MISFIT_NOALLOC_MAX_PARTIALS
 * doubles on every device that loads the library, until exit).  Larger
 * batches are rejected with FWI_ERANGE.  Each call looks up the array's
 * address on the current device; the first call on a device may load the
 * library's device code there, so make it outside stream capture.
 * All calls share the array: calls that overlap on the GPU race, so keep them
 * in order on one stream.  It allocates nothing.  No counterpart in the
 * reference. */
int fwi_misfit_noalloc(const float *data, const float *syn, float *adstf, double *misfit, int nshots, int nrec,
                       int nt, double dt, void *stream);

/* Separable Gaussian smoothing of an FP64 kernel ([nx][in_pitch]) into a
 * float32 field ([nx][out_pitch]), normalised by the Gaussian mass inside
 * the grid as init_gausian does; taps beyond 6 sigma (relative weight
 * < 2e-8) are dropped.  tmp: caller scratch of nx*nz doubles.  sigma > 0.
 * Replaces init_gausian / apply_gauxxian_x / apply_gauxxian_z and smooth,
 * fd2d.py:76-108, 349-352. */
int fwi_smooth(const double *in, int in_pitch, float *out, int out_pitch, double *tmp,
               int nx, int nz, int sigma, void *stream);

/*
 * Learned preconditioner: kernels of a small U-Net (training and inference).
 * No counterpart in the reference, which has no learned component.
 * Activations are NHWC bf16 ([n][h][w][c], c a multiple of 16, 16-byte
 * aligned); 3x3 weights [9][cout][cin] bf16 (tap = 3*(dy+1)+(dx+1), input
 * channel innermost); biases and gradients FP32.  Arithmetic: bf16 products,
 * FP32 accumulation on the tensor cores.
 */

/* out = act(conv3x3(concat(in0, in1), w) + bias), zero padding; channel
 * counts c0, c1 (c1 = 0: in1 unused), cout = d0 + d1 output channels split
 * between out0 (first d0) and out1; bias may be NULL; relu != 0 applies
 * max(., 0).  The data gradient of a layer is this call on the gradient of
 * its output, with the weights of fwi_unet_flip_weights, no bias and no
 * relu, splitting the result back into the layer's two inputs. */
int fwi_unet_conv3x3(const void *in0, int c0, const void *in1, int c1, const void *w, const float *bias,
                     int cout, void *out0, int d0, void *out1, int d1, int n, int h, int wd, int relu,
                     void *stream);

/* Kernel of fwi_unet_conv3x3: path 0 (default) uses the tcgen05 tensor-core
 * kernel where wd >= 64 and the mma.sync kernel elsewhere;
 * path 1 uses the mma.sync kernel everywhere.  Other values only query.
 * Returns the previous path.  Process-wide; not thread-safe against
 * concurrent convolution calls. */
int fwi_unet_conv_path(int path);

/* wd[8-tap][ci][co] = w[tap][co][ci]: the weights of the data gradient. */
int fwi_unet_flip_weights(const void *w, void *wd, int cout, int cin, void *stream);

/* g[i] = 0 where y[i] <= 0 (gradient through a ReLU whose output is y). */
int fwi_unet_relu_bwd(void *g, const void *y, long long count, void *stream);

/* Weight and bias gradients of a 3x3 layer: dw[9][cout][c0+c1] = sum over
 * pixels of g (x) shifted input, db[cout] = sum over pixels of g (db may be
 * NULL), both summed in a fixed block order.  part: caller scratch of
 * fwi_unet_wgrad_partials(cout, c0+c1, n, h, w) floats. */
long long fwi_unet_wgrad_partials(int cout, int cin, int n, int h, int w);
int fwi_unet_conv3x3_wgrad(const void *g, int cout, const void *in0, int c0, const void *in1, int c1, int n,
                           int h, int wd, float *part, float *dw, float *db, void *stream);

/* 2x2 average pooling [n][h][w][c] -> [n][h/2][w/2][c] (h, w even) and its
 * adjoint (accumulate != 0 adds into gin); nearest 2x upsampling
 * [n][h][w][c] -> [n][2h][2w][c] and its adjoint (h, w of the smaller
 * image). */
int fwi_unet_pool2(const void *in, void *out, int c, int n, int h, int w, void *stream);
int fwi_unet_pool2_bwd(const void *gout, void *gin, int c, int n, int h, int w, int accumulate, void *stream);
int fwi_unet_up2(const void *in, void *out, int c, int n, int h, int w, void *stream);
int fwi_unet_up2_bwd(const void *gout, void *gin, int c, int n, int h, int w, void *stream);

/* 1x1 output head from 16 channels: out[p] = sum_c w[c] x[p][c] + b[0]
 * (FP32), and its adjoint: gx = w gout, gwb[0..15] = dL/dw, gwb[16] = dL/db;
 * part: caller scratch of 17 * ceil(n*h*w / 4096) floats. */
int fwi_unet_head(const void *x, const float *w, const float *b, float *out, int n, int h, int wd, void *stream);
int fwi_unet_head_bwd(const void *x, const float *w, const float *gout, void *gx, float *part, float *gwb, int n,
                      int h, int wd, void *stream);

/* Network input: three FP32 planes [n][3][h][w] -> [n][h][w][16] bf16, the
 * channels past the third zero. */
int fwi_unet_pack(const float *planes, void *x, int n, int h, int w, void *stream);

/* One Adam step on FP32 master weights w with moments m, v and gradient g;
 * wb (may be NULL) receives the bf16 copy.  step counts from 1. */
int fwi_unet_adam(float *w, float *m, float *v, const float *g, void *wb, long long count, double lr,
                  double beta1, double beta2, double eps, int step, void *stream);

/* Mean squared error of out against tgt: *loss (FP64) and gout = dloss/dout.
 * part: caller scratch of fwi_unet_mse_partials() doubles. */
long long fwi_unet_mse_partials(void);
int fwi_unet_mse(const float *out, const float *tgt, float *gout, double *loss, double *part, long long count,
                 void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SEISPIE_B200_H */
