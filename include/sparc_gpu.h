/*
 * sparc_gpu.h -- C ABI of the B200 implementation of SPARC's linear wave
 * time step (libsparc_gpu.so).
 *
 * The reference (damoprz/SPARC2, Fortran 90 + MPI) keeps every quantity in
 * module globals and calls argument-less subroutines from driver.f90.  This
 * header replaces those calls with handle-based entry points that take plain
 * pointers and sizes, so a Fortran ISO_C_BINDING shim (or ctypes, or C++) can
 * bind them.  Every entry point returns an int status: SPARC_OK (0) or a
 * negative SPARC_ERR_* code.  No exception crosses the ABI.
 *
 * Layout conventions: every 3-D array is Fortran order (x fastest, then y,
 * then z), exactly as the reference's a(dim1,dim2,dim3,l).  Host buffers are
 * owned by the caller and copied; device memory is owned by the library.
 * A handle is not thread safe: use one host thread per handle.
 */
#ifndef SPARC_GPU_H
#define SPARC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define SPARC_OK               0
#define SPARC_ERR_INVALID     -1  /* bad argument or unsupported option      */
#define SPARC_ERR_CUDA        -2  /* a CUDA runtime call failed              */
#define SPARC_ERR_NOMEM       -3  /* device allocation failed                */
#define SPARC_ERR_UNSTABLE    -4  /* driver.f90:175-183 fail criterion hit   */
#define SPARC_ERR_ORDER       -5  /* call made before its prerequisites      */
#define SPARC_ERR_TIMEOUT     -6  /* a bounded device wait gave up           */
#define SPARC_ERR_NODEVICE    -7  /* no usable sm_100 device                 */

/* precision of the device state */
#define SPARC_FP64 0   /* plain form: FP64 state, coefficients and arithmetic */
#define SPARC_FP32 1   /* precision form: FP32 state/coefficients, FP64 setup */

/* source kinds (driver.f90:130-155) */
#define SPARC_SRC_NONE  0
#define SPARC_SRC_PULSE 1  /* PULSE = 1: one analytic pulse                   */
#define SPARC_SRC_PSR   2  /* PULSE = 2: table of "random-ish" pulses         */
#define SPARC_SRC_RANDOM 3 /* PULSE = 0: forcing series vr(x, y, t), 7-point
                              Lagrange in time (all_modules.f90:1892-1950)   */

/*
 * Run parameters: the subset of the .trol keys (initialize.f90:1385-1924)
 * that the time step reads.  Units are the .trol units (cgs, seconds).
 */
typedef struct sparc_params {
    int32_t nx, ny, nz;            /* global grid                            */
    int32_t magnetic;              /* MAGNETIC: 0 quiet, 1 thermal, 2 MHD    */
    int32_t periodic;              /* PERIODIC (x,y)                          */
    int32_t use_pml;               /* USE_PML  (z CPML)                       */
    int32_t use_hpml;              /* USE_HPML (x,y CPML)                     */
    int32_t stabilise;             /* STABILISE                               */
    int32_t filter_mode_xy;        /* 1: 11-pt filter, 2: 7-pt filter         */
    int32_t filter_mode_z;
    int32_t block_x, block_y, block_z; /* reference MPI block counts; fix the
                                          rank-local quirks that the oracle
                                          and the kernels reproduce          */
    int32_t npml_xb, npml_xt, npml_yb, npml_yt, npml_zb, npml_zt;
    double  pml_xb[4], pml_xt[4];  /* RC, n, kappa, sponge (xpmlb, xpmlt)    */
    double  pml_yb[4], pml_yt[4];
    double  pml_zb[4], pml_zt[4];
    double  xlength, ylength;      /* cm                                      */
    double  timestep;              /* s                                       */
    double  s_xy, s_z;             /* 7-pt filter strengths                   */
    double  t_xy, t_z;             /* filter cadences, s                      */
    double  maxva;                 /* Alfven limiter, cm/s                    */
    double  sp_str, sp_length, sp_decay; /* horizontal sponge (no HPML)      */
    int32_t precision;             /* SPARC_FP64 or SPARC_FP32                */
    int32_t damping;               /* DAMPING: FFT horizontal damping of the
                                      velocities in every RHS evaluation
                                      (all_modules.f90:1803-1888; FP64
                                      plain form only)                      */
    int32_t reserved[6];
} sparc_params;

/* One entry of a PULSE = 2 table: the reference's psr_* arrays
 * (all_modules.f90:159-160, drawn at all_modules.f90:566-586), code units:
 * px, py in [0,1) of the box, pz, sr, sz in solar radii, t0, t1 in s. */
typedef struct sparc_pulse {
    double px, py, pz, sr, sz, amp, t0, t1;
} sparc_pulse;

typedef struct sparc_source {
    int32_t kind;        /* SPARC_SRC_*                                      */
    int32_t dir;         /* pulse_dir: 1 v_x, 2 v_y, 3 v_z                   */
    int64_t init;        /* first driver iteration of the run (driver init);
                            PULSE = 2 adds every pulse twice at this step    */
    /* SPARC_SRC_PULSE, .trol units (driver.f90:140-145) */
    double  amp, t0, t1, st, px, py, pz, sr, sz;
    /* SPARC_SRC_PSR */
    double  psr_st;      /* time width, 120 s in the reference               */
    int32_t npulses;
    int32_t pad;
    const sparc_pulse *pulses;
    /* SPARC_SRC_RANDOM (driver.f90:73-81, 130-132): the series replaces the
     * forcingfunc FITS cube; it is copied, times rnd_ampl / dimc.  The
     * forcing acts on v_z (dir is ignored). */
    double  cadforcing;  /* s between two samples of the series              */
    double  rnd_ampl;    /* randomexciteampl, cm/s                           */
    double  rnd_depth;   /* randomexcitedepth, cm (centre of source_dep)     */
    double  rnd_sigma;   /* randomexcitesigma, cm                            */
    int32_t nseries;     /* num_steps: samples in the series (>= 1)          */
    int32_t pad2;
    const double *series; /* nx*ny*nseries, x fastest, then y, then sample   */
} sparc_source;

typedef struct sparc_handle sparc_handle;

/* Diagnostics of the last completed driver iteration (driver.f90:161-183). */
typedef struct sparc_diag {
    double  ke_norm;     /* norm((rho0+rho)|v|^2/2)*dimc^2*dimrho            */
    double  min_rho;     /* min(rho + rho0) over the stage-5 fields          */
    double  min_p;       /* min(p + p0) over the stage-5 fields              */
    int64_t iteration;   /* driver iteration these belong to (-1: none)      */
    int64_t fail_iteration; /* first iteration that failed, -1 if none      */
} sparc_diag;

/* ------------------------------------------------------------- lifecycle */

/* Replaces INIT_MPI + INITANDALLOCATE (initialize.f90:12, 463): validates
 * the parameters, allocates the device state on CUDA device `device`. */
int sparc_create(const sparc_params *p, int device, sparc_handle **out);

/* Frees all device memory of the handle. */
int sparc_destroy(sparc_handle *h);

/* Replaces READ_IN_HDF5 (all_modules.f90:179-416) + INITIALISE_RHS
 * (initialize.f90:883-1273) + INITIALIZE_STEP (initialize.f90:1366):
 * the background arrays in dimensional cgs units, nx*ny*nz each (bx0, by0,
 * bz0 may be NULL unless magnetic == 2), zaxis in Mm and grav in cm/s^2
 * (nz each).  The FP64 coefficient setup runs on the device.  Resets the
 * state and the CPML auxiliary fields to zero. */
int sparc_set_background(sparc_handle *h,
                         const double *rho0, const double *pre0,
                         const double *cs0, const double *bx0,
                         const double *by0, const double *bz0,
                         const double *zaxis_mm, const double *grav);

/* Replaces the forcing fill of driver.f90:130-155 / RUN_PSR_PULSE
 * (all_modules.f90:521-663); the forcing is evaluated inside the kernels. */
int sparc_set_source(sparc_handle *h, const sparc_source *src);

/* Number of doubles of the state (V*nx*ny*nz, V = 5 or 8) and of the
 * concatenated CPML auxiliary state [z-bot, z-top, x-bot, x-top, y-bot,
 * y-top], each face in the reference's (dim1,dim2,npml,P) /
 * (npml,dim2,dim3,P) / (dim1,npml,dim3,P) layout, P = 2 or 6. */
int sparc_sizes(const sparc_handle *h, int64_t *n_state, int64_t *n_psi);

/* Checkpoint / restart of a(:,:,:,l) and zpmlvars/xpmlvars/ypmlvars
 * (all_modules.f90:741-1562 without the HDF5 container). psi may be NULL. */
int sparc_set_state(sparc_handle *h, const double *a, const double *psi);
int sparc_get_state(sparc_handle *h, double *a, double *psi);

/* ------------------------------------------------------------ time step */

/* One call of STEP (step.f90:20-63) for driver iteration nn: the forcing
 * of iteration nn, five RK stages with fused derivatives, CPML and RHS,
 * the final update, and the diagnostics of driver.f90:161-183.  Asynchronous
 * on the handle's stream. */
int sparc_step(sparc_handle *h, int64_t nn);

/* FILTER_VARS (derivatives.f90:659-703) as called at driver.f90:200 after
 * iteration nn (nothing happens at nn == 0 or off cadence).  Asynchronous. */
int sparc_filter_vars(sparc_handle *h, int64_t nn);

/* Iterations first .. first+count-1 of the driver loop (driver.f90:123-202:
 * step, diagnostics, filter at cadence), launched as CUDA graphs.
 * Asynchronous; errors of the fail criterion surface in sparc_diagnostics. */
int sparc_run(sparc_handle *h, int64_t first, int64_t count);

/* z extent of the stage kernels' work items (a work item is a 32 x 8
 * column tile over zchunk layers; each item pays 10 layers of z-window
 * warm-up).  No counterpart in the reference.  11 <= zchunk (clamped to
 * nz); set up from the grid size, changed by sparc_set_zchunk or
 * sparc_tune.  Results do not depend on it. */
int sparc_set_zchunk(sparc_handle *h, int zchunk);
int sparc_get_zchunk(const sparc_handle *h, int *zchunk);

/* Autotuner of the z extent: runs iterations first, first+1, ... of the
 * driver loop exactly as sparc_run would (they are real iterations of the
 * simulation), giving each candidate extent (16 .. 150 layers) one untimed
 * iteration and then `steps_per_trial` iterations off the filter cadence
 * timed with CUDA events; keeps the fastest.  *next receives the first
 * iteration not yet run, *best the extent chosen.  Synchronous. */
int sparc_tune(sparc_handle *h, int64_t first, int steps_per_trial, int64_t *next,
               int *best);

/* Waits for the handle's stream and returns the diagnostics of the last
 * iteration.  Returns SPARC_ERR_UNSTABLE when an iteration met the fail
 * criterion of driver.f90:175-183 (the diagnostics are still filled). */
int sparc_diagnostics(sparc_handle *h, sparc_diag *out);

/* Waits for all work queued on the handle. */
int sparc_synchronize(sparc_handle *h);

/* The cudaStream_t the handle launches on (for event timing by callers). */
int sparc_stream(sparc_handle *h, void **stream);

/* Number of kernels the library has launched on this handle so far
 * (graph launches count every kernel node). */
int sparc_launch_count(const sparc_handle *h, int64_t *count);

/* ----------------------------------------------------- unit primitives */

/* ddx/ddy/ddz (derivatives.f90:10-116, 226-341, 451-562) of one host field
 * with boundary flag bc (1 or 5), on the device; dir 0 = x, 1 = y, 2 = z.
 * Needs sparc_set_background (for the z metric). */
int sparc_derivative(sparc_handle *h, int dir, int bc,
                     const double *in, double *out);

/* filtx/filty/filtz (derivatives.f90:119-223, 345-447, 565-642) of one host
 * field (no edge pre-averaging; that belongs to FILTER_VARS). */
int sparc_filter_field(sparc_handle *h, int dir, const double *in,
                       double *out);

/* Copies one FP64 coefficient array of the setup to the host, by the
 * reference's variable name ("rho0", "gradp0_z", "spongexyz", "reduction",
 * "curlbox", "stretch", "g", "az_bot", ...).  *count is the element count
 * on return; out may be NULL to query it. */
int sparc_get_coeff(sparc_handle *h, const char *name, double *out,
                    int64_t *count);

/* Scalars of the setup: dimc, dimrho, diml, dimb, deltat, stretchx,
 * stretchy, betas[5] (12 doubles in that order). */
int sparc_get_scalars(sparc_handle *h, double *out12);

/* Human-readable text of the last error on this handle (or of the last
 * failed sparc_create when h is NULL). */
const char *sparc_last_error(const sparc_handle *h);

/* ------------------------------------------------ allocation-free path
 * No counterpart in the reference.  The kinetic-energy norm of the handle's
 * current state (norm() of all_modules.f90:684-706 as driver.f90:161 uses
 * it) computed without allocating memory: the reduction's scratch is a
 * static device array of 33,024 bytes, so grids above 67,108,864 points are
 * rejected (SPARC_ERR_INVALID).  For callers that must not allocate, e.g. a
 * monitor polling a simulation whose device memory is fully committed to
 * the serving loop's budget.  It equals sparc_diagnostics' ke_norm only
 * when called right after an iteration's stages, before that iteration's
 * filter (sparc_filter_vars, or a filter iteration inside sparc_run) or a
 * sparc_set_state replaces the state; sparc_diagnostics keeps the norm of
 * the stage-5 state as driver.f90:161 does before FILTER_VARS.  Works on a
 * batch member too (it reads the member's live state buffer, ordered on the
 * batch's stream).  The scratch is shared by every call on a device: calls
 * that overlap in time race and must be serialised by the caller.  The
 * first call on a device looks up the scratch address; make it before any
 * stream capture, and not after cudaDeviceReset (the cached address does
 * not survive a reset).  Waits for the handle's (or batch's) stream. */
int sparc_ke_norm_noalloc(sparc_handle *h, double *ke_norm);

/* ---------------------------------------------------- failure injection
 * No counterpart in the reference.  For failure-detection tests: launches on
 * the handle's stream a kernel whose bounded wait on an mbarrier that nothing
 * completes gives up after `polls` polls (1 <= polls <= 2^20) or 10 ms of
 * the GPU's global timer, whichever comes first, and raises the handle's
 * device error flag, as a stage kernel's gave-up wait does.  The GPU
 * neither hangs nor faults.  The next sparc_diagnostics returns
 * SPARC_ERR_TIMEOUT; sparc_set_state (a restart from saved state) clears
 * the flag. */
int sparc_inject_wait_timeout(sparc_handle *h, int64_t polls);

/* -------------------------------------------------------- batched engine
 * No counterpart in the reference, which runs one simulation per MPI job.
 * A batch advances many SPARC_FP32 handles of any grid sizes together: each
 * step of all members is one CUDA-graph launch of persistent kernels (one
 * per RK stage) over a device (simulation, tile, z-chunk) work-list.  While
 * a handle is in a batch the batch owns its buffer roles, iteration and
 * stream order: sparc_step/run/filter_vars/set_state/get_state/set_source/
 * destroy on it return SPARC_ERR_ORDER; sparc_diagnostics works. */
typedef struct sparc_batch sparc_batch;

/* A batch of up to `capacity` simulations on CUDA device `device`. */
int sparc_batch_create(int device, int capacity, sparc_batch **out);

/* Removes the remaining members (they keep their state) and frees. */
int sparc_batch_destroy(sparc_batch *b);

/* Adds a SPARC_FP32 handle (background and source set) that will run
 * driver iterations first .. first+count-1; *slot receives its slot. */
int sparc_batch_add(sparc_batch *b, sparc_handle *h, int64_t first,
                    int64_t count, int *slot);

/* Takes a member out (after the queued steps); the handle is usable alone
 * again with its state as the batch left it. */
int sparc_batch_remove(sparc_batch *b, int slot);

/* Enqueues `steps` batched steps.  Each step advances every member with
 * iterations left by one driver iteration (forcing, five RK stages,
 * diagnostics, FILTER_VARS at its own cadence).  Asynchronous. */
int sparc_batch_run(sparc_batch *b, int64_t steps);

/* Waits, then writes each slot's iterations left (-1: free slot),
 * `capacity` entries. */
int sparc_batch_remaining(sparc_batch *b, int64_t *remaining);

/* z extent of the work items of MHD and quiet members (>= 11 layers);
 * the autotuner's knob.  Results do not depend on it. */
int sparc_batch_set_tiles(sparc_batch *b, int zchunk_mhd, int zchunk_quiet);
int sparc_batch_get_tiles(const sparc_batch *b, int *zchunk_mhd,
                          int *zchunk_quiet);

/* Autotuner: times `steps_per_trial` batched steps per candidate z extent
 * of the work items (one axis at a time, MHD then quiet; their column
 * shapes, 32x8 MHD and 32x16 quiet, are fixed by the kernels' thread
 * layout) and keeps the fastest; returns the z extents.  The trial steps
 * advance the members like sparc_batch_run. */
int sparc_batch_tune(sparc_batch *b, int steps_per_trial, int *best_mhd,
                     int *best_quiet);

int sparc_batch_synchronize(sparc_batch *b);
int sparc_batch_stream(sparc_batch *b, void **stream);
int sparc_batch_launch_count(const sparc_batch *b, int64_t *count);
const char *sparc_batch_last_error(const sparc_batch *b);

/* ----------------------------------------------------------- serving
 * No counterpart in the reference.  A server runs a worker thread over one
 * batch: solve requests (SPARC_FP32 parameters and a duration) queue first
 * in first out, are admitted by a device-memory budget and a slot count,
 * built by the client once admitted, and run as batch members while later
 * requests are admitted and set up.  Ticket states: */
#define SPARC_REQ_QUEUED    0  /* submitted, nothing allocated             */
#define SPARC_REQ_ADMITTED  1  /* budget reserved; client builds the handle */
#define SPARC_REQ_RUNNING   2  /* attached; advancing in the batch          */
#define SPARC_REQ_DONE      3  /* all iterations done; out of the batch     */
#define SPARC_REQ_FAILED    4  /* the batch reported an error               */
#define SPARC_REQ_COLLECTED 5  /* handle handed back by sparc_serve_result  */

typedef struct sparc_server sparc_server;

/* Device bytes of a SPARC_FP32 handle for `p`: resident while it runs, and
 * at the peak of its set-up (FP64 setup arrays included). */
int sparc_estimate_bytes(const sparc_params *p, int64_t *resident,
                         int64_t *peak);

/* A server on `device` with up to `capacity` concurrent requests, a device
 * memory budget in bytes, and `quantum` batched steps per service round. */
int sparc_server_create(int device, int capacity, int64_t budget_bytes,
                        int quantum, sparc_server **out);

/* Stops the worker; running requests end FAILED, their handles stay the
 * client's. */
int sparc_server_destroy(sparc_server *s);

/* Queues a request for driver iterations first .. first+steps-1;
 * SPARC_ERR_NOMEM if its peak size exceeds the whole budget. */
int sparc_serve_submit(sparc_server *s, const sparc_params *p, int64_t first,
                       int64_t steps, int64_t *ticket);

/* Waits up to timeout_ms for a not yet taken ticket in `state`
 * (SPARC_REQ_ADMITTED: to build; SPARC_REQ_DONE: to collect, FAILED ones
 * included); SPARC_ERR_TIMEOUT if none. */
int sparc_serve_next(sparc_server *s, int state, int64_t timeout_ms,
                     int64_t *ticket);

/* The parameters and iteration range a ticket was submitted with. */
int sparc_serve_params(sparc_server *s, int64_t ticket, sparc_params *p,
                       int64_t *first, int64_t *steps);

/* Hands the built handle (background and source set) of an ADMITTED
 * ticket to the server, which adds it to the batch. */
int sparc_serve_attach(sparc_server *s, int64_t ticket, sparc_handle *h);

/* The handle of a DONE or FAILED ticket and its timestamps (seconds since
 * the server started: submit, admit, start, done). */
int sparc_serve_result(sparc_server *s, int64_t ticket, sparc_handle **h,
                       double *times4, int *state);

/* Ends a ticket and returns its budget (after the client destroyed or
 * took over the handle, or gave up building it). */
int sparc_serve_release(sparc_server *s, int64_t ticket);

int sparc_serve_state(sparc_server *s, int64_t ticket, int *state);

/* stats[0..11]: queued, admitted, running, done, budget bytes in use, max
 * concurrent requests (admitted or running), batched steps run, service
 * rounds, grid-point updates, seconds the worker waited on batched steps,
 * max requests running in the batch at once, requests attached while
 * others were running (their work joined a batch already on the device). */
int sparc_serve_stats(sparc_server *s, double *stats12);

const char *sparc_server_last_error(const sparc_server *s);

#ifdef __cplusplus
}
#endif

#endif /* SPARC_GPU_H */
