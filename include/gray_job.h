/*
 * gray_job -- the GRay2 lux-job surface in C, on top of libgray_cuda.
 *
 * The reference is a lux job module: LUX_MKMOD builds a struct gray whose
 * Lux_job vtable is {conf, init, exec} (sim/gray.c:37-216,
 * sim-org/gray.c:62-346); conf(arg) consumes one "name=value" run-time
 * option from the .opts tables (sim/gray.opts, sim/Kerr.opts,
 * sim/infcam.opts, sim-org/setup.opts, sim-org/param.opts) and returns 0
 * when it recognised it; init builds the device state; exec runs the dump
 * loop.  The lux runtime itself is not available, so this header carries
 * the same vtable and option names with a gray_ prefix; a lux build would
 * alias LUX_MKMOD / LUX_RMMOD to gray_job_mkmod / gray_job_rmmod.
 *
 * Errors are returned (never lux_fatal/abort).
 */
#ifndef GRAY_JOB_H
#define GRAY_JOB_H

#include <stddef.h>
#include <stdint.h>

#include "gray_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gray_lux_job gray_lux_job;

/* lux's Lux_job vtable (lux/job.h as used by sim/gray.c:196-198) */
struct gray_lux_job {
	int (*conf)(gray_lux_job *ego, const char *arg);
	int (*init)(gray_lux_job *ego);
	int (*exec)(gray_lux_job *ego);
};

/* LUX_MKMOD (sim/gray.c:187-204): a job with every option at its default. */
gray_lux_job *gray_job_mkmod(const void *opts);
/* LUX_RMMOD (sim/gray.c:206-216) */
void          gray_job_rmmod(gray_lux_job *ego);

/* conf() return values: 0 = consumed; GRAY_JOB_UNKNOWN = no such option
 * (lux's non-zero "not mine"); negative GRAY_E* = recognised but invalid. */
#define GRAY_JOB_UNKNOWN 1

/* Inspection for tests and hosts: the render the current options describe,
 * the dump file pattern, and the option value as text. */
int gray_job_desc(const gray_lux_job *ego, gray_render_desc *out);
int gray_job_get(const gray_lux_job *ego, const char *name, char *buf, size_t len);

/* After exec: accepted ray-steps and summed kernel ns over all dumps. */
int gray_job_stats(const gray_lux_job *ego, uint64_t *ray_steps, double *kernel_ns);

/* Raw dump writer of sim-org/io.c:39-72: header {sz, n_data, W, H} as
 * size_t, then W*H*n_data reals, then W*H*n_info reals (AoS).  sz is 8. */
int gray_write_raw(const char *path, const double *data, const double *info,
                   size_t n_data, size_t w, size_t h);

/* Reads a dump gray_write_raw wrote, after checking that its header is
 * {8, n_data, w, h}: the load path sim-org/io.c:37 leaves as a TODO.
 * GRAY_ENOTFOUND when the file does not open, GRAY_ESIZE on a header or
 * length mismatch. */
int gray_read_raw(const char *path, double *data, double *info, size_t n_data, size_t w,
                  size_t h);

#ifdef __cplusplus
}
#endif

#endif /* GRAY_JOB_H */
