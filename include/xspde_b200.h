/* xspde_b200.h -- C ABI of the B200-native xSPDE ensemble-integration path.
 *
 * The library replaces the hooks through which xSPDE 4.21 drives one ensemble
 * block (reference paths are relative to the xspde_matlab project root):
 *
 *   xs_run_path   replaces  p.path(a,nc,p)        Simulator/xpath.m:1, called at
 *                           Simulator/xensemble.m:79, default set at
 *                           Simulator/xpreferences.m:62.  The whole time loop
 *                           (noise, method, observables) runs on the GPU.
 *   xs_step       replaces  p.method(a,w,p)       Applications/SDE/MP.m:1, RK4.m:1,
 *                           Euler.m:1, RK2.m:1, Implicit.m:1, called at
 *                           Simulator/xpath.m:42.
 *   xs_noise      replaces  p.noisegen(w1,nc,s,p) Simulator/xnoise.m:1 (one draw,
 *                           before the coarse average of xnoise.m:33-35).
 *   xs_random     replaces  p.randomgen(p)        Simulator/xrandom.m:1.
 *
 * The problem description mirrors the input struct fields of
 * Simulator/xpreferences.m (dimensions, fields, points, ranges, origins,
 * steps, checks, ensembles, noises, inrandoms, iterations, ipsteps, seed,
 * boundaries, linear, deriv, initial, observe) after xSPDE's defaults have
 * been applied.  Function-valued fields are passed as the text of the MATLAB
 * anonymous function (what func2str returns), e.g.
 *   deriv  = "@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)"
 * The text is compiled into the fused kernel (NVRTC, sm_100a).  Expressions
 * outside the supported grammar make xs_create fail with XS_ERR_GRAMMAR:
 * there is no CPU fallback.
 *
 * Conventions: all host arrays are caller-owned, complex values are
 * interleaved (re, im) FP64, and array layout is MATLAB column-major with the
 * field index fastest and the ensemble index slowest: a(fields, space..., ens).
 * The library owns its device buffers.  Every call returns XS_OK (0) or a
 * negative XS_ERR_* code and never aborts; xs_last_error() gives the message
 * of the calling thread's last failure.  One handle per host thread.
 */
#ifndef XSPDE_B200_H
#define XSPDE_B200_H

#include <stddef.h>

#ifdef __cplusplus
#define XS_EXTERN extern "C"
#else
#define XS_EXTERN extern
#endif
#define XS_API XS_EXTERN __attribute__((visibility("default")))

typedef struct xs_handle xs_handle;
typedef int xs_status;

enum {
  XS_OK = 0,
  XS_ERR_SHAPE = -1,       /* sizes or layout not supported / inconsistent */
  XS_ERR_GRAMMAR = -2,     /* MATLAB expression outside the device grammar */
  XS_ERR_NVRTC = -3,       /* runtime compilation failed */
  XS_ERR_CUDA = -4,        /* CUDA runtime/driver error */
  XS_ERR_NAN = -5,         /* a trajectory produced a non-finite value */
  XS_ERR_TIMEOUT = -6,     /* a bounded device wait gave up */
  XS_ERR_ARG = -7,         /* invalid argument */
  XS_ERR_NODEVICE = -8,    /* no CUDA device */
  XS_ERR_UNSUPPORTED = -9  /* valid xSPDE input that this path does not cover */
};

enum { XS_METHOD_MP = 0, XS_METHOD_RK4 = 1, XS_METHOD_EULER = 2, XS_METHOD_RK2 = 3, XS_METHOD_IMPLICIT = 4 };
enum { XS_PREC_FP64 = 0, XS_PREC_FP32 = 1 };

#define XS_MAXDIM 4 /* p.dimensions up to 4: time + 3 space dimensions */

typedef struct xs_problem {
  int dimensions;              /* p.dimensions: 1 = SDE, 2..4 = SPDE with 1..3 space dims */
  int fields;                  /* components of the single field cell, p.fields */
  int noises;                  /* Gaussian x-space noises, p.noises */
  int inrandoms;               /* initial Gaussian randoms, p.inrandoms */
  int points[XS_MAXDIM];       /* p.points after space steps (xpreferences.m:137) */
  double ranges[XS_MAXDIM];    /* p.ranges */
  double origins[XS_MAXDIM];   /* p.origins */
  int steps;                   /* p.steps(1) */
  int checks;                  /* p.checks(1): 1 = step-halving fine/coarse passes */
  int ensembles[3];            /* p.ensembles */
  int method;                  /* XS_METHOD_* (p.method) */
  int iterations;              /* p.iterations (MP, Implicit) */
  int ipsteps;                 /* p.ipsteps: propagator is exp(L dtr/ipsteps) */
  int precision;               /* XS_PREC_FP64 or XS_PREC_FP32 (fields/transforms/drift) */
  unsigned long long seed;     /* p.seed */
  const int* boundaries;       /* NULL: periodic; else [dimensions-1][fields][2] of p.boundaries{1,d}(i,b) */
  const char* deriv;           /* p.deriv text, "@(a,w,p) ..." */
  const char* initial;         /* p.initial text, "@(v,p) ..." */
  const char* linear;          /* p.linear text "@(p) ..." or NULL/"" for none */
  int nobserve;                /* number of observe functions (0 -> default "a") */
  const char* const* observe;  /* p.observe texts, "@(a,p) ..." */
  int nparams;                 /* named scalar constants readable as p.<name> */
  const char* const* param_names;
  const double* param_values;
  int path_kind;               /* 0 = automatic, 1 = resident, 2 = streaming */
  int runtime_params;          /* 1: named scalars are read at run time (per batch item; param_values are
                                  the defaults), so one compiled kernel serves many parameter values.
                                  p.linear always uses param_values. */
  const int* transforms;       /* NULL: every observable in x space; else [nobserve][4] flags of
                                  p.transforms{n} (time, x, y, z): 1 = the observable sees the field
                                  Fourier-transformed along that space dimension (xnft.m, periodic
                                  dimensions only); the time flag evaluates the observable on the time
                                  spectrum of the field (Simulator/xpath.m:90-106) */
  int sequence;                /* index of this input in a sequence (xensemble.m:36-62): part of the
                                  Philox counter, so every sequence draws its own noise */
  int boundary_values;         /* 1: p.boundfun gives boundary values (MP only); the caller supplies
                                  them per check pass with xs_set_boundary_values before each path */
  int knoises;                 /* p.knoises: k-filtered noise components (Simulator/xnoise.m:39-50), the
                                  drift's next noise argument after w: @(a,w,z,p), or @(a,z,p) when
                                  noises = 0; every space dimension periodic */
  int krandoms;                /* p.krandoms: k-filtered initial randoms (Simulator/xrandom.m:24-29), the
                                  initial function's next argument after v */
  const double* nfilter;       /* NULL (p.nfilter = identity) or [knoises][space] complex FP64: the factor
                                  p.nfilter multiplies each k-space noise value by, the k lattice in FFT
                                  order (p.kx ... in propagation order, Simulator/xgrid.m) */
  const double* rfilter;       /* the same for p.rfilter and krandoms */
  int auxfields;               /* p.auxfields: components of the auxiliary cell (Simulator/xpath.m:36-45),
                                  0 for none; observe functions then take (a, x, p) */
  const char* define;          /* p.define text "@(a,w,p) ...": the auxiliary cell from the field and
                                  the step's noise, averaged over the start and end of each step */
} xs_problem;

/* Create a handle: parse, generate and compile the kernels (NVRTC, cached).
 * Replaces no single reference function: it is the one-time set-up that
 * Simulator/xensemble.m:47 (p.propfactor) and the per-call evaluation of the
 * user's handles amount to. */
XS_API xs_status xs_create(const xs_problem* prob, xs_handle** out);
XS_API void xs_destroy(xs_handle* h);

/* Message of the calling thread's last failed call (truncated to n bytes).
 * Returns the full message length. */
XS_API size_t xs_last_error(char* buf, size_t n);

/* Library version string. */
XS_API const char* xs_version(void);

/* Shape of observable o (0-based): lines, and spatial = 1 when the ensemble
 * average keeps the lattice (av{o} is [lines, time, space...]) or 0 when it is
 * [lines, time] (Int/Ave over all space).  Mirrors the observe sizing of
 * Simulator/xpreferences.m:262-343. */
XS_API xs_status xs_observe_info(const xs_handle* h, int o, int* lines, int* spatial);

/* Space sizes of av{o} for a spatial observable: dims[d] (d = 0, 1, 2 for x, y, z)
 * is the lattice's points, 1 for a dimension that an observable of the form
 * Int(f, dx, [bounds,] p) or Ave(f, v, p) over a subset of the dimensions reduces
 * (Applications/SPDE/Int.m:48-70, Ave.m), and 1 beyond the lattice's dimensions.
 * Such an observable is evaluated per site on the device and summed over its
 * reduced dimensions on the host when the means are copied out (xs_run_path,
 * xs_batch_results); xs_run_path_device returns the unreduced site means. */
XS_API xs_status xs_observe_shape(const xs_handle* h, int o, int* dims);

/* Bytes of av_out for nblocks blocks: sum over observables of
 * lines*points(1)*(spatial ? nspace : 1) complex doubles, per block. */
XS_API size_t xs_av_doubles_per_block(const xs_handle* h);

/* Which device path integrates this problem: 1 resident (one CTA per group of
 * trajectories), 2 streaming 2D (row and column passes), 3 streaming 3D
 * (plane and z-line passes, DST/DCT in every dimension); 0 for a null handle.
 * Chosen at xs_create (no GPU needed). */
XS_API int xs_path_kind(const xs_handle* h);

/* p.path replacement (Simulator/xpath.m): integrate ensemble blocks
 * first_block .. first_block+nblocks-1 (global block index
 * npar-1 + (j-1)*ensembles(3), Simulator/xensemble.m:26) for check pass nc
 * (1 = fine, 2 = coarse; Simulator/xensemble.m:27).
 *   a_in   NULL: the initial field is p.initial(p.randomgen(p)) evaluated on the
 *          device (Simulator/xensemble.m:53-64); else [fields, space, ens1*nblocks]
 *          complex FP64 (the `a` that xensemble passes to p.path).
 *   av_out per block, per observable o in order, the block mean av{o}
 *          [lines, points(1), space] complex FP64 (Simulator/xpath.m:81).
 *   a_out  NULL or the final field, same layout as a_in.
 * Host pointers; copies are synchronous with respect to the caller. */
XS_API xs_status xs_run_path(xs_handle* h, int first_block, int nblocks, int nc, const double* a_in,
                             double* av_out, double* a_out);

/* xs_run_path that also returns p.path's third output `raw` when p.rawdata is
 * set (Simulator/xpath.m:73-78, stored at xensemble.m:79 and returned by
 * xsim.m:1): raw_out is the field at every output time, [fields, points(1),
 * space, ens1*nblocks] complex FP64 (raw{l} of Simulator/xpreferences.m:148 for
 * consecutive blocks).  Resident path only (XS_ERR_UNSUPPORTED on the
 * streaming path); XS_ERR_SHAPE when the record exceeds free device memory.
 * raw_out NULL is xs_run_path. */
XS_API xs_status xs_run_path_raw(xs_handle* h, int first_block, int nblocks, int nc, const double* a_in,
                                 double* av_out, double* a_out, double* raw_out);

/* Same as xs_run_path with device pointers and a caller stream (cudaStream_t
 * passed as void*; NULL is the default stream, as in CUDA); nothing is copied
 * to or from the host and the call returns without synchronising.  a_in_dev/a_out_dev use the device layout
 * [ens][fields][space] (identical to the host layout when fields == 1) and
 * may be NULL.  av_dev receives, per block and output time, one row of
 * complex FP64 values: site observables' lines k at k*nspace + s (s the
 * column-major lattice index), then the non-spatial lines. */
XS_API xs_status xs_run_path_device(xs_handle* h, int first_block, int nblocks, int nc, const double* a_in_dev,
                                    double* av_dev, double* a_out_dev, void* stream);

/* xs_run_path_device for callers that cannot allocate device memory: no
 * counterpart in the reference.  A MATLAB MEX function that must leave device
 * memory to MATLAB's own gpuArray allocator, code recorded into a CUDA graph,
 * or a service whose memory budget is fixed after start-up may not call
 * cudaMalloc; this entry point calls no cudaMalloc, cudaFree or allocating
 * library routine.  It runs the resident path (problems whose per-trajectory
 * field fits in shared memory) with the observable partial sums in a fixed
 * 16 MiB device array inside the library (1,048,576 complex FP64 values);
 * launches that need more -- points(1) x (trajectories / trajectories per
 * CTA) x row length -- are rejected with XS_ERR_SHAPE, and a streaming-path
 * handle with XS_ERR_UNSUPPORTED.  The handle must already hold its tables
 * for check pass nc: call xs_run_path or xs_run_path_device once with the
 * same nc first (those calls allocate).  The first call on each device looks
 * up the array's device address (cudaGetSymbolAddress) and should come before
 * any stream capture; the address is kept for the life of the process, so do
 * not call this entry point again on a device after resetting it
 * (cudaDeviceReset).  Its launches are not counted by xs_kernel_stats.  Every call shares the one array per device, so calls
 * that overlap on the GPU race; nothing in it needs to start at zero, since
 * each call writes every element it later reads.  The initial field comes
 * from p.initial on the device; av_dev is as for xs_run_path_device. */
XS_API xs_status xs_run_path_device_noalloc(xs_handle* h, int first_block, int nblocks, int nc, double* av_dev,
                                            void* stream);

/* Wait for the handle's work and report device-side status (XS_ERR_NAN when a
 * trajectory became non-finite in the last run). */
XS_API xs_status xs_sync(xs_handle* h);

/* p.noisegen replacement, one draw (Simulator/xnoise.m:29-32): w_out =
 * randn * sqrt(scale * noisefactor) as [noises, space, ens1] real FP64 for
 * block `block`, draw index `draw` (1 = first call of a path).  The coarse
 * average (xnoise.m:33-35) stays with the caller. */
XS_API xs_status xs_noise(xs_handle* h, int block, int draw, double scale, double* w_out);

/* p.randomgen replacement (Simulator/xrandom.m:20-23): [inrandoms, space, ens1]
 * real FP64, randn * sqrt(noisefactor), Philox draw 0. */
XS_API xs_status xs_random(xs_handle* h, int block, double* v_out);

/* p.method replacement (Applications/SDE/<method>.m): one step of length dtr
 * from time t on a [fields, space, ens1] complex FP64 field, in place, with
 * the pre-scaled noise w [noises, space, ens1] (NULL: zero noise). */
XS_API xs_status xs_step(xs_handle* h, double* a_inout, const double* w, double t, double dtr);

/* Inputs of the learned control variate (no counterpart in the reference):
 * coarse space-time projections of the Wiener increments that p.noisegen
 * feeds the trajectories of blocks first_block .. first_block+nblocks-1
 * (fine pass; lattices of up to two space dimensions, an SDE being a single
 * site).  region = {i1lo, i2lo, bw, bh, nbx, nby}: nbx x nby lattice
 * blocks of bw x bh sites starting at x index i1lo, y index i2lo (<= 16 x 16
 * blocks); windows of draws_per_window consecutive draws starting at
 * first_draw (>= 1); within a window the draws are weighted by
 * exp(-decay * (last draw of the window - draw)).  out_dev[traj][comp][window]
 * [by][bx] (FP32, device): the weighted sum of the standard normals over the
 * block and window divided by sqrt(sum of squared weights * sites), so each
 * feature is N(0,1) and independent of the others.  Asynchronous on `stream` (a cudaStream_t; NULL is the default stream). */
XS_API xs_status xs_noise_features(xs_handle* h, int first_block, int nblocks, const int* region, int first_draw,
                                   int draws_per_window, int windows, double decay, float* out_dev, void* stream);

/* Learned control variate network (no counterpart in the reference): MLP
 * in -> hidden -> hidden -> hidden -> 1 with GELU, BF16 tensor-core operands
 * and FP32 accumulation.  All pointers are device pointers (FP32); work is
 * the activation workspace.  xs_mlp_sizes returns the workspace floats for a
 * batch and the parameter count (W1[h][in], b1, W2[h][h], b2, W3[h][h], b3,
 * w4[h], b4).  xs_mlp_train_grad runs the forward pass, the MSE loss against
 * target (*loss_dev, FP64) and the backward pass into grad.  xs_mlp_adam
 * applies one Adam step (step >= 1) with decoupled weight decay. */
XS_API size_t xs_mlp_sizes(int in, int hidden, int batch, size_t* nparams);
XS_API xs_status xs_mlp_forward(int batch, int in, int hidden, const float* x, const float* params, float* work,
                                float* y, void* stream);
XS_API xs_status xs_mlp_train_grad(int batch, int in, int hidden, const float* x, const float* params, float* work,
                                   const float* target, float* grad, double* loss_dev, void* stream);
XS_API xs_status xs_mlp_adam(size_t n, float* params, const float* grad, float* m, float* v, float lr, float beta1,
                             float beta2, float eps, int step, float weight_decay, void* stream);

/* Ensemble moments of block means on the device (Simulator/xensemble.m:98-101,
 * where xSPDE accumulates data(:,1) += D*nes and data(:,m1) += D.^2*nes with
 * D = real(output(av)) and nes = 1/(ensembles(2)*ensembles(3))): av_dev holds
 * nblocks consecutive blocks of n complex FP64 means (as xs_run_path_device
 * writes them); mom_dev[k] = scale * sum_b Re(av[b][k]) and
 * mom_dev[n + k] = scale * sum_b Re(av[b][k])^2 (FP64, compensated sums over
 * the blocks in order), added to mom_dev's contents when accumulate != 0.
 * Asynchronous on `stream` (NULL: the default stream); allocates nothing. */
XS_API xs_status xs_block_moments(const double* av_dev, int nblocks, long long n, double scale, double* mom_dev,
                                  int accumulate, void* stream);

/* Kernel kinds counted by xs_kernel_stats. */
enum {
  XS_KERNEL_RESIDENT = 0, /* whole path with fields in shared memory */
  XS_KERNEL_OBS_REDUCE,   /* block means of the resident path */
  XS_KERNEL_X_INIT,       /* streaming: initial field -> K state */
  XS_KERNEL_X_STEP,       /* streaming: row pass (IFFT_x, drift + noise, FFT_x); 3D: plane pass */
  XS_KERNEL_X_FINAL,      /* streaming: K state -> x-space field */
  XS_KERNEL_Y_PASS,       /* streaming: column pass (FFT_y, exp(L dt), IFFT_y); 3D: z-line pass */
  XS_KERNEL_X_OBS,        /* streaming: observables */
  XS_KERNEL_SCALAR,       /* streaming: Int/Ave scalar observables */
  XS_KERNEL_RC_PASS,      /* streaming: row pass of one half of the trajectories fused with the
                             column pass of the other half */
  XS_KERNEL_KINDS
};

/* Instrumentation (no counterpart in the reference, which has only tic/toc,
 * Simulator/xsim.m:28): with timing on, every launch of the handle is
 * bracketed by CUDA events on its stream.  xs_kernel_stats synchronises
 * that stream and returns, per kernel kind, the launches and the summed
 * device milliseconds since the last reset (arrays of XS_KERNEL_KINDS). */
XS_API xs_status xs_set_kernel_timing(xs_handle* h, int on);
XS_API xs_status xs_kernel_stats(xs_handle* h, int reset, double* ms_out, long long* launches_out);

/* Uneven batch (no counterpart in the reference): many independent problems,
 * each one ensemble block (ensembles(2) = ensembles(3) = 1), integrated by
 * ONE CUDA-graph launch.  An item with checks = 1 runs both check passes of
 * xensemble.m:41-45 (fine, nc = 1, and coarse, nc = 2) inside the same graph.  Items whose generated kernels agree
 * (same lattice, fields, expressions, method, precision; set runtime_params
 * so that named scalars differ per item) share a persistent kernel that pulls
 * (item, trajectory tile) units from a longest-first queue; items too large
 * for shared memory run their streaming launches inside the same graph.
 *   xs_batch_create  groups the items (host only; copies everything it needs)
 *   xs_batch_tune    picks each variant's tile: mode 0 heuristic, mode 1 times
 *                    the candidates on the device (cached per source and GPU)
 *   xs_batch_run     captures the graph on first use, then launches it on
 *                    `stream` (NULL: the batch's own stream); asynchronous
 *   xs_batch_sync    waits for the device and reports kernel status
 *   xs_batch_results item means in the layout of xs_run_path's av_out, the
 *                    fine pass followed (checks = 1) by the coarse pass
 *                    (xs_batch_av_doubles doubles in all)
 *   xs_batch_info    item >= 0: {variant, path (1 resident, 2 streaming), G,
 *                    threads, CTAs, units}; item < 0: {items, variants,
 *                    streaming items, kernel launches per run} */
typedef struct xs_batch xs_batch;
XS_API xs_status xs_batch_create(const xs_problem* items, int nitems, xs_batch** out);
XS_API void xs_batch_destroy(xs_batch* b);
XS_API xs_status xs_batch_tune(xs_batch* b, int mode);
XS_API xs_status xs_batch_run(xs_batch* b, void* stream);
XS_API xs_status xs_batch_sync(xs_batch* b);
XS_API size_t xs_batch_av_doubles(const xs_batch* b, int item);
XS_API xs_status xs_batch_results(xs_batch* b, int item, double* av_out);
XS_API xs_status xs_batch_info(const xs_batch* b, int item, int* info, int ninfo);

/* Boundary values of p.boundfun for one check pass nc (xpatch.m, xsetbound.m;
 * problems created with boundary_values = 1): values = complex FP64
 * [ntimes][space dims][fields][2] (lower, upper end) at t = origins(1) +
 * k dtr/2, k = 0..ntimes-1, dtr the pass's step; the host evaluates the user's
 * p.boundfun there (it may be any function of t and the parameters). */
XS_API xs_status xs_set_boundary_values(xs_handle* h, int nc, int ntimes, const double* values);

/* Compile-only check (no device needed): parse and NVRTC-compile the kernels
 * of a problem for sm_100a.  Writes the compile log (truncated to n). */
XS_API xs_status xs_compile_check(const xs_problem* prob, char* log, size_t n);

#endif /* XSPDE_B200_H */
