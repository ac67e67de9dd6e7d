/*
 * libgray_cuda -- B200 (sm_100a) geodesic hot path of GRay2 behind a C ABI.
 *
 * The reference (luxsrc/gray) reaches its OpenCL kernels through the lux
 * opencl module: sim-org/build.c:30-143 JIT-builds the program,
 * sim-org/icond.c:29-86 launches icond_drv, sim-org/evolve.c:28-67 launches
 * evolve_drv once per dump interval and returns the kernel time in ns, and
 * sim-org/io.c:39-72 maps the ray buffers back to the host.  In the new lux
 * tree (sim/gray.c:116-176) the same steps are dmk() of real[8] rays,
 * ic->init(), the planner's exec (a TODO at sim/gray.c:168) and ocl->d2h().
 * This header replaces that glue with plain C entry points: no CUDA or
 * torch types cross it; the context owns every device allocation, and hosts
 * pass host pointers with explicit byte counts.
 *
 * Errors: every entry point returns an int status (0 = GRAY_OK, negative =
 * GRAY_E*), never aborts; gray_strerror() names it.  Threading: one context
 * per host thread, except gray_serve_submit / gray_serve_poll, which lock.
 */
#ifndef GRAY_CUDA_H
#define GRAY_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRAY_ABI_VERSION 3
#define GRAY_MAX_FREQ    8

enum gray_status {
	GRAY_OK        =  0,
	GRAY_EINVAL    = -1,  /* bad argument or configuration        */
	GRAY_ENOMEM    = -2,  /* device or host allocation failed      */
	GRAY_ECUDA     = -3,  /* CUDA runtime error                    */
	GRAY_ENODEV    = -4,  /* no usable sm_100 device               */
	GRAY_EBUDGET   = -5,  /* request exceeds the HBM budget        */
	GRAY_ETIMEOUT  = -6,  /* reserved: no kernel here waits on a
	                         flag, so no entry point returns it     */
	GRAY_ENOTFOUND = -7,  /* unknown render / request id           */
	GRAY_ESTATE    = -8,  /* call out of order (e.g. no icond yet) */
	GRAY_ESIZE     = -9,  /* host buffer size does not match       */
	GRAY_ESOURCE   = -10  /* a caller callback reported failure    */
};

enum gray_precision {
	GRAY_PREC_FP64  = 0,  /* plain FP64 (sim-org/setup.opts:11 precision=8) */
	GRAY_PREC_MIXED = 1   /* FP32 bulk, FP64 islands, compensated update    */
};

enum gray_spacetime {
	GRAY_ST_KERR      = 0, /* analytic Cartesian Kerr-Schild (KS.cl)         */
	GRAY_ST_NUMERICAL = 1  /* interpolated grid (dyst.cl + interp.cl)        */
};

enum gray_flow {
	GRAY_FLOW_NONE    = 0, /* geodesics only (n_freq ignored)               */
	GRAY_FLOW_TORUS   = 1, /* analytic power-law torus feeding rt.cl form   */
	GRAY_FLOW_THERMAL = 2  /* the reference's template flow (flow.cl:36-58):
	                          n_e = rho of the grid, T_e = flow_te, |b| =
	                          flow_b along z, fluid at rest; thermal
	                          bremsstrahlung + synchrotron of rt.cl:28-198
	                          (numerical spacetimes)                       */
};

enum gray_term {
	GRAY_TERM_EPS   = 0,   /* reference: stop when r - r_+ < 0.01 (phys.cl:54) */
	GRAY_TERM_RPLUS = 1    /* stop when r < 1.01 r_+                          */
};

enum gray_layout {
	GRAY_LAYOUT_SOA = 0,   /* data[s * n_rays + g]  (sim-org/SoA.cl:29)      */
	GRAY_LAYOUT_AOS = 1    /* data[g * n_data + s]  (sim-org/AoS.cl:29)      */
};

/* One render: the run-time parameters of sim/gray.opts, sim/Kerr.opts,
 * sim/infcam.opts, sim-org/setup.opts and sim-org/param.opts that the hot
 * path reads, with the reference's names. */
typedef struct gray_render_desc {
	/* Kerr.opts */
	double   m_bh;            /* m_bh:M   solar masses (transfer units only) */
	double   a_spin;          /* a_spin:a dimensionless spin                  */
	/* infcam.opts */
	double   w_img, h_img;    /* w_img:w, h_img:h   image size in GM/c^2      */
	double   r_obs;           /* r_obs:r  camera distance                     */
	double   i_obs, j_obs;    /* i_obs:i, j_obs:j   degrees                   */
	uint64_t n_width;         /* n_width:W  rays along the width             */
	uint64_t n_height;        /* n_height:H rays along the height            */
	/* gray.opts / setup.opts step control and output times */
	double   t_init;          /* t_init:t0                                    */
	double   dt_dump;         /* dt_dump:dt  affine interval between dumps    */
	uint64_t n_sub;           /* n_sub:n  substeps per dump (step-size cap)   */
	uint64_t n_dump;          /* n_dump:N number of dump intervals            */
	int32_t  term;            /* enum gray_term                               */
	/* radiative transfer (param.opts nu list) */
	int32_t  n_freq;          /* 0 .. GRAY_MAX_FREQ                            */
	double   nu[GRAY_MAX_FREQ];
	int32_t  flow;            /* enum gray_flow                               */
	double   torus_n0;        /* density normalisation                        */
	double   torus_kappa;     /* absorption normalisation                     */
	double   torus_hr;        /* scale height over radius                     */
	/* selection */
	int32_t  spacetime;       /* enum gray_spacetime                          */
	int32_t  precision;       /* enum gray_precision                          */
	/* thermal flow (GRAY_FLOW_THERMAL) */
	double   m_adm;           /* param.opts M_ADM:m, solar masses            */
	double   flow_te;         /* electron temperature kT/(m_e c^2) (1e12)     */
	double   flow_b;          /* magnetic field magnitude, along z (0)        */
	/* camera row window (no reference counterpart): the render integrates
	 * rows [row_begin, row_begin + n_rows) of the n_height-row image, with
	 * the pixel map of the whole image (driver.cl:47-51), so that row
	 * blocks of one render can run on different GPUs.  n_rows = 0 means
	 * every row (row_begin must then be 0).  Ray r of the render is pixel
	 * (r % n_width, row_begin + r / n_width). */
	uint64_t row_begin;
	uint64_t n_rows;
} gray_render_desc;

typedef struct gray_ctx gray_ctx;

/* ---- context ------------------------------------------------------- */

const char *gray_strerror(int status);
int         gray_abi_version(void);

/* Replaces lux_load("opencl", &opts) (sim/gray.c:88-95; sim-org/build.c:134-142):
 * binds CUDA device `device` (the i_device:id option) and caps the HBM the
 * context may allocate at hbm_budget bytes (0 = 90% of free memory). */
gray_ctx   *gray_create(int device, size_t hbm_budget, int *status);
void        gray_destroy(gray_ctx *ctx);

/* Launch on a caller-provided cudaStream_t (passed as void *); NULL returns
 * to the context's own stream. */
int         gray_set_stream(gray_ctx *ctx, void *cuda_stream);
int         gray_sync(gray_ctx *ctx);
size_t      gray_hbm_used(const gray_ctx *ctx);

/* ---- renders ------------------------------------------------------- */

/* Replaces the buffer set-up of sim-org/gray.c:113-145 (_init: data and
 * info buffers of n_rays * n_data reals) and sim/gray.c:115-117 (dmk of
 * real[8] rays).  State is kept on the device in SoA order. */
int gray_render_create(gray_ctx *ctx, const gray_render_desc *desc, int *render_id);
int gray_render_destroy(gray_ctx *ctx, int render_id);

/* Replaces icond() (sim-org/icond.c:29-86 -> driver.cl:36-67 icond_drv) and
 * the infcam initcond plug-in's init (sim/gray/infcam.c:37-42). */
int gray_icond(gray_ctx *ctx, int render_id);

/* Replaces evolve() (sim-org/evolve.c:28-67 -> driver.cl:69-108 evolve_drv):
 * integrates every ray over one dump interval of affine length target - t
 * with n_sub substeps (target == t leaves the state unchanged).  If ns is
 * non-NULL the call waits and stores the kernel time in ns (what ocl->exec
 * returns); otherwise it only enqueues. */
int gray_evolve(gray_ctx *ctx, int render_id, double t, double target,
                uint64_t n_sub, double *ns);

/* icond + all n_dump intervals of the render (the sim-org/gray.c:243-294
 * loop without the intermediate dumps).  FP64 renders run the per-interval
 * kernel like the reference; mixed renders run one persistent launch. */
int gray_run(gray_ctx *ctx, int render_id, double *ns);

/* The evolve part of gray_run alone: all n_dump intervals from the current
 * state (after gray_icond or gray_write_state). */
int gray_evolve_all(gray_ctx *ctx, int render_id, double *ns);

/* Replaces dump()'s ocl->mmap (sim-org/io.c:39-72) and sim/gray.c:170-172
 * d2h: copies the FP64 state (n_rays * n_data doubles) and the getuu()
 * diagnostic (n_rays doubles) to host memory in the requested layout.
 * Either pointer may be NULL. */
int gray_read_state(gray_ctx *ctx, int render_id, void *data, size_t data_bytes,
                    void *info, size_t info_bytes, int layout);

/* Upload a state (resume from a dump; io.c:37 leaves load() as a TODO). */
int gray_write_state(gray_ctx *ctx, int render_id, const void *data,
                     size_t data_bytes, int layout);

/* Covariant momentum k_mu = g_mu_nu u^nu per ray (KS.cl:91-114 down()),
 * n_rays * 4 doubles in SoA order. */
int gray_read_kdown(gray_ctx *ctx, int render_id, double *k, size_t bytes);

/* Output coordinates of an analytic render's state (KS.cl:63-153), n_rays
 * * 8 doubles in SoA order: t, r, theta, phi, then u^t, u^r, u^theta,
 * u^phi.  GRAY_COORDS_SPH_KS is getsphKS/getsphKSu; GRAY_COORDS_BL is
 * getBL/getBLu with t_BL = t_KS at r_match (> r_+; the reference leaves
 * r_match undefined) and phi matched at infinity.  Two lines of KS.cl
 * disagree with the metric the path integrates (down(), KS.cl:91-114):
 * phi is taken with (r - i a) where the metric's event is x + i y =
 * (r + i a) e^(i phi) sin(theta) (KS.cl:68-69, 130), and getBLu multiplies
 * u^phi and u^t where the change of coordinates has u^r (KS.cl:148-151).
 * By default both follow the metric, so a null ray stays null in the
 * Boyer-Lindquist metric; GRAY_COORDS_AS_WRITTEN reproduces the lines. */
enum gray_coords {
	GRAY_COORDS_SPH_KS = 0,
	GRAY_COORDS_BL     = 1
};
#define GRAY_COORDS_AS_WRITTEN 1
int gray_read_coords(gray_ctx *ctx, int render_id, int system, double r_match, int flags,
                     double *out, size_t bytes);

/* Accepted RK4 steps summed over the render's rays since the last icond. */
int gray_ray_steps(gray_ctx *ctx, int render_id, uint64_t *steps);

/* Of those, the steps that interpolated the numerical grid (mixed
 * numerical renders; in physics mode steps outside the box do not). */
int gray_gather_steps(gray_ctx *ctx, int render_id, uint64_t *steps);

/* ---- batches, launch plans, graphs ---------------------------------- */

/* A batch is many mixed-precision renders integrated by ONE persistent
 * launch (a render table; rays of every render share the warp-refilled ray
 * queue).  The first gray_batch_run captures the sequence -- per-render
 * initial conditions, queue reset, persistent kernel -- into a CUDA graph;
 * later runs replay it.  All renders of a batch use the same spacetime;
 * analytic ones also the same n_freq.  Renders stay owned by the context
 * and must outlive the batch. */
int gray_batch_create(gray_ctx *ctx, const int *render_ids, int n, int *batch_id);
int gray_batch_destroy(gray_ctx *ctx, int batch_id);
int gray_batch_run(gray_ctx *ctx, int batch_id, double *ns);
int gray_batch_steps(gray_ctx *ctx, int batch_id, uint64_t *steps);

/* Launch shape of the persistent kernels. */
typedef struct gray_launch_plan {
	int32_t block;            /* threads per block                          */
	int32_t blocks_per_sm;    /* 0 = as many as fit                         */
	int32_t rays_per_thread;  /* 1 (scalar FP32) or 2 (packed f32x2)         */
	int32_t rk4_rolled;       /* 0: the four RK4 stages unrolled (one RHS
	                             body each), 1: one RHS body in a loop     */
	double  ns;               /* measured trial time (gray_plan output)      */
} gray_launch_plan;

enum gray_plan_flags {
	GRAY_PLAN_ESTIMATE = 0,   /* choose by rule, no trial launches          */
	GRAY_PLAN_MEASURE  = 1    /* time every candidate on the batch           */
};

/* Autotuner replacing the lux planner of sim/gray/Kerr/ocl.c:41-75 and
 * tests/ck_sample.c:84-104 (7 work-group sizes, estimate or measure): picks
 * block size, blocks per SM, rays per thread and RK4 stage unrolling for
 * the batch's kernel,
 * installs it in the context and returns it.  MEASURE runs trial launches
 * over the first dump intervals of the batch, leaving the renders' state
 * undefined (gray_batch_run / gray_run start from icond again). */
int gray_plan(gray_ctx *ctx, int batch_id, int flags, gray_launch_plan *best);
int gray_set_plan(gray_ctx *ctx, const gray_launch_plan *plan);
int gray_get_plan(const gray_ctx *ctx, gray_launch_plan *plan);

/* ---- serving: continuous batching (no reference counterpart) -------- */

/* A scheduler thread owned by the context admits submitted renders as HBM
 * (the configured budget) and table slots free up, and advances every
 * admitted render by a window of dump intervals per iteration: one
 * persistent launch per kind (analytic by n_freq, numerical), so renders
 * that arrived while others run share the device with them.  An iteration
 * lasts dumps_per_iter intervals of the admitted render whose interval is
 * estimated to take longest (and at least 50 ms); every other render
 * advances as many intervals as fit in that time, so small renders finish
 * within an iteration or two and a newcomer waits about one iteration at
 * most for admission.  The estimates (steps per interval times the longer
 * of one ray's step latency and the rays' share of the device) size the
 * windows only; results do not depend on them.  With analytic and
 * numerical renders in flight at once, their two launches run together on
 * a split of the SMs.  Request state comes from a device memory pool that
 * the server keeps until it stops (its size never exceeds the budget).
 * Finished renders are copied to host memory (a 2 GiB pinned pool while it
 * has room) and their device state returns to the pool.  Only
 * mixed-precision renders are served; numerical ones use the context's
 * grid, which must be loaded before gray_serve_start.  While the server
 * runs, only gray_serve_* may be called on the context (they are
 * thread-safe). */
enum gray_req_state {
	GRAY_REQ_QUEUED    = 0,
	GRAY_REQ_RUNNING   = 1,
	GRAY_REQ_DONE      = 2,
	GRAY_REQ_FAILED    = 3,
	GRAY_REQ_CANCELLED = 4
};

typedef struct gray_serve_config {
	size_t  hbm_budget;      /* bytes of admitted render state (0: the context's) */
	int32_t max_inflight;    /* renders admitted at once (0: 1024)              */
	int32_t dumps_per_iter;  /* dump intervals per iteration (0: 1)             */
} gray_serve_config;

typedef struct gray_request_status {
	int32_t  state;          /* enum gray_req_state                        */
	int32_t  status;         /* GRAY_E* of a failed request                */
	double   t_submit;       /* gray_serve_clock() seconds                 */
	double   t_admit;
	double   t_done;
	uint64_t n_rays;
} gray_request_status;

typedef struct gray_serve_stats {
	uint64_t iterations;
	uint64_t ray_steps[2];   /* [0] analytic, [1] numerical                */
	uint64_t completed, failed, cancelled;
	double   busy_s;         /* device time of the iterations (events)    */
} gray_serve_stats;

double gray_serve_clock(void);
int gray_serve_start(gray_ctx *ctx, const gray_serve_config *cfg);
int gray_serve_submit(gray_ctx *ctx, const gray_render_desc *desc, uint64_t *request_id);
int gray_serve_poll(gray_ctx *ctx, uint64_t request_id, gray_request_status *out);
/* Copy a finished request's state (SoA, as gray_read_state) and release it. */
int gray_serve_result(gray_ctx *ctx, uint64_t request_id, void *data, size_t data_bytes,
                      void *info, size_t info_bytes);
int gray_serve_cancel(gray_ctx *ctx, uint64_t request_id);
int gray_serve_get_stats(gray_ctx *ctx, gray_serve_stats *out);
/* drain != 0: finish every submitted request first; else drop them. */
int gray_serve_stop(gray_ctx *ctx, int drain);

/* ---- numerical spacetime (sim-org/io.c:302-533, interp.cl, dyst.cl) - */

typedef struct gray_grid_desc {
	int32_t nx, ny, nz;  /* points along x, y, z (num_points.s123)         */
	float   box[8];      /* {t1, xmin, ymin, zmin, t2, xmax, ymax, zmax}     */
	int32_t bug_gzz;     /* 1: read g_zz from g_yz as dyst.cl:283 does      */
	int32_t physics;     /* 1: flat outside the box, time factor in [0,1]   */
} gray_grid_desc;

/* Upload one time level (0 = t1, 1 = t2) of 51 FP32 fields, each nz*ny*nx
 * in [z][y][x] order, in the order of io.c:356-428: Gamma_ijk (i-major,
 * j <= k; 40), g_ij (i <= j; 10), rho.  fields[51] are host pointers. */
int gray_load_spacetime(gray_ctx *ctx, const gray_grid_desc *grid,
                        const float *const *fields, int level);

/* Same, but the fields are already interleaved [z][y][x][51] in one host
 * array of nz*ny*nx*51 floats. */
int gray_load_spacetime_interleaved(gray_ctx *ctx, const gray_grid_desc *grid,
                                    const float *fields, int level);

/* Sample boosted Kerr-Schild (mass 1, spin a, speed v along axis 1..3) on
 * the device at time t into level `level` of the context's grid: the
 * generator of tools/generate_data.py + tools/boosted_ks.py run as a kernel. */
int gray_make_boosted_ks(gray_ctx *ctx, const gray_grid_desc *grid, double a,
                         double v, int axis, double t, int level);

/* Swap the two time levels (io.c:279-300 copy_snapshot). */
int gray_swap_levels(gray_ctx *ctx);

/* Copy one time level back to the host, interleaved [z][y][x][51] floats
 * (nz*ny*nx*51*4 bytes): inspection of a loaded or generated grid. */
int gray_read_spacetime(gray_ctx *ctx, int level, float *fields, size_t bytes);

/* ---- time series of snapshots (sim-org/gray.c:147-294) --------------- */

/* The snapshots of a dynamic spacetime: what the reference lists from the
 * groups of its HDF5 file (io.c:150-230) and reads one at a time
 * (load_snapshot, io.c:302-533).  load() fills `fields` -- nz*ny*nx*51
 * floats, interleaved [z][y][x][51] in the field order of
 * gray_load_spacetime -- with snapshot k and returns 0, or nonzero on
 * failure.  It is called on the thread that called gray_run_series. */
typedef struct gray_snapshot_source {
	uint64_t      n_times;  /* snapshots available (>= 1)                   */
	const double *times;    /* their times, strictly increasing             */
	void         *user;
	int         (*load)(void *user, uint64_t k, float *fields);
} gray_snapshot_source;

/* The snapshot pair (k, k+1) each dump interval integrates on, chosen as
 * sim-org/gray.c:41-57 and 183-293 choose it: first the pair bracketing
 * t_init, then, after each interval whose end time leaves [t_k, t_k+1],
 * the pair bracketing that time.  pairs[i] is the pair of interval i + 1
 * (from t_init + i dt_dump to t_init + (i+1) dt_dump).  With fast_light
 * (param.opts enable_fast_light) or a single snapshot the spacetime is
 * frozen: every entry is the snapshot bracketing t_init (0 for a single
 * one) and the run interpolates in space only.  GRAY_EINVAL where the
 * reference stops: t_init or the final time outside the series
 * (sim-org/gray.c:193-205), times not increasing.  Host code only. */
int gray_series_schedule(const double *times, uint64_t n_times, double t_init,
                         double dt_dump, uint64_t n_dump, int fast_light,
                         int64_t *pairs);

/* Replaces the dynamic-spacetime loop of sim-org/gray.c:147-294 for a
 * numerical render: icond at t_init, then its n_dump intervals, each on
 * the snapshot pair of gray_series_schedule, with the level times of that
 * pair.  `grid` gives the shape, spatial box and flags (its box times are
 * ignored).  Snapshots stream: while an interval runs, the snapshot the
 * next one needs is read (src->load) and copied to the device into a third
 * level, and a pair that moves by one snapshot keeps the level it shares
 * (copy_snapshot, io.c:279-300, becomes a relabelling).  after_dump
 * (nullable) is called as after_dump(src->user, i) after interval
 * i = 1..n_dump with the render's state readable, where the reference
 * dumps (sim-org/gray.c:255); nonzero stops the run with
 * GRAY_ESOURCE, as does a failing load().  *loads (nullable) receives the
 * number of load() calls, *ns the elapsed device time.  The grid keeps the
 * last pair as levels 0 and 1.  GRAY_ESTATE while the server runs. */
int gray_run_series(gray_ctx *ctx, int render, const gray_grid_desc *grid,
                    const gray_snapshot_source *src, int fast_light,
                    int (*after_dump)(void *user, uint64_t i), double *ns,
                    uint64_t *loads);

/* ---- allocation-free entry point ----------------------------------- */

/* No counterpart in the reference.  For callers that cannot call
 * cudaMalloc -- hosts whose own allocator already owns the device memory
 * and forbids side allocations, or latency-critical loops that cannot take
 * the device-wide synchronisation cudaMalloc/cudaFree imply -- this runs
 * gray_icond + gray_evolve_all of up to GRAY_NOALLOC_MAX_RENDERS analytic
 * Kerr-Schild renders in mixed precision without allocating anything.
 *
 *  - state_dev[i] / info_dev[i]: device buffers the caller owns, of
 *    n_width*n_height*(8 + 2 n_freq) and n_width*n_height doubles (SoA,
 *    as gray_read_state returns them); they are written.
 *  - All renders of one call share n_freq and flow; rays over all renders
 *    must not exceed 2^31.  More renders, or more rays, return GRAY_EINVAL.
 *  - The kernel's scratch (render table, ray queue, step counter:
 *    GRAY_NOALLOC_SCRATCH_BYTES) is a static device array that every GPU
 *    loading this library holds until exit.  The first call on a device
 *    looks up its address (cudaGetSymbolAddress).  Every call shares the
 *    array: calls that overlap on the GPU (other streams, other host
 *    threads) race.
 *  - Work is enqueued on cuda_stream (a cudaStream_t, NULL = legacy default
 *    stream).  If steps_host is non-NULL the call waits and stores the
 *    accepted ray-steps there; otherwise it returns after enqueueing. */
#define GRAY_NOALLOC_MAX_RENDERS   32
#define GRAY_NOALLOC_SCRATCH_BYTES 16384
int gray_run_mixed_noalloc(int device, const gray_render_desc *descs, int n_renders,
                           double *const *state_dev, double *const *info_dev,
                           void *cuda_stream, uint64_t *steps_host);

/* ---- measurement (no reference counterpart) ------------------------ */

/* CUDA-core FMA-loop peak of the context's device in FLOP/s (FMA = 2):
 * the roofline denominator of the geodesic kernels.  precision selects
 * FP64 or FP32 (best of scalar and packed f32x2 FMA).  With
 * GRAY_PEAK_L1_GATHER it is instead the L1 load bandwidth in bytes/s with
 * the numerical kernel's 32-byte loads, all hits and fully used lines: the
 * ceiling of the grid gathers, which hit L1 for 95% of their sectors. */
#define GRAY_PEAK_L1_GATHER 2
int gray_measure_peak(gray_ctx *ctx, int precision, double *flops);

#ifdef __cplusplus
}
#endif

#endif /* GRAY_CUDA_H */
