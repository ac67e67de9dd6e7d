/*
 * Internal declarations shared by the libgray_cuda translation units.
 * Not part of the public ABI (include/gray_cuda.h is).
 */
#ifndef GRAY_INTERNAL_H
#define GRAY_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gray_cuda.h"

#define GRAY_NCOMP 51        /* 40 Gamma + 10 g + rho per grid point      */
#define GRAY_EPSILON 1e-28   /* sim-org/preamble.cl:30                    */

/* Per-render constants, computed once on the host (FP64, libm) and passed
 * by value to every kernel.  Host-side evaluation of the camera angles'
 * sin/cos (KS.cl:195-197) and of r_+, r_isco and nu^-0.7 keeps all device
 * arithmetic to +, *, fma, /, sqrt, which round identically in the CPU
 * oracle. */
/* libm-derived constants of the thermal emissivities (rt.cl:95-143),
 * evaluated once on the host from volatile inputs exactly as the oracle
 * does, so that no compile-time folding differs between the two. */
struct ThermalConsts {
	double g1;        /* sqrt(3/pi)                               */
	double g2;        /* sqrt(3)/pi                               */
	double g3;        /* log(4/1.78107241799)                     */
	double g4;        /* log(4/1.78107241799^2.5)                 */
	double g5;        /* sqrt(12)                                 */
	double ff_f;      /* bremsstrahlung normalisation (rt.cl:135) */
	double lk_scale;  /* T_GRID / log(T_MAX/T_MIN)                */
};

struct RenderParams {
	double a, aa;            /* spin and its square                      */
	double rp, risco;        /* horizon and prograde ISCO radii          */
	double eps_stop;         /* stop when r - r_+ < eps_stop             */
	double ci, si, cj, sj;   /* camera angle cosines and sines           */
	double w_img, h_img, r_obs;
	long long w_rays, h_rays, n_rays;
	long long row0;          /* first camera row of the render's rays    */
	int    n_freq, flow, n_data, spacetime;
	double torus_n0, torus_kappa, torus_hr;
	double nupow[GRAY_MAX_FREQ];   /* nu_i^-0.7 */
	double nuinv2[GRAY_MAX_FREQ];  /* nu_i^-2   */
	float  nupow_f[GRAY_MAX_FREQ];
	float  nuinv2_f[GRAY_MAX_FREQ];
	/* thermal flow */
	double nu[GRAY_MAX_FREQ];      /* frequencies (Hz for the thermal flow) */
	double m_adm, flow_te, flow_b;
	ThermalConsts th;
};

void gray_thermal_consts(ThermalConsts *t);

/* Numerical spacetime on the device: two time levels, each interleaved
 * [z][y][x][GRAY_NSTRIDE] floats, plus per-axis fisheye node tables. */
#define GRAY_NSTRIDE 56      /* 51 fields padded to a 32-byte multiple    */
struct GridParams {
	int    nx, ny, nz;
	float  box[8];
	int    bug_gzz, physics;
	double A[3], B[3];       /* fisheye constants per axis (interp.cl:116-117) */
	const double *nodes[3];  /* node coordinates per axis, n+1 entries (FP64) */
	const float  *nodes_f[3];
	const float  *lvl[2];
	int    single;           /* t1 == t2: use level 0 only               */
};

/* descriptor validation and per-render constants (gray_api.cu) */
int  gray_internal_check_desc(const gray_render_desc *d);
void gray_internal_make_params(const gray_render_desc *d, RenderParams *p);

/* ---- launchers (one per translation unit) ---- */
cudaError_t launch_icond64(const RenderParams &p, double *data, double *info,
                           cudaStream_t st);
cudaError_t launch_evolve64(const RenderParams &p, double *data, double *info,
                            double dt, long long n_sub,
                            unsigned long long *steps, cudaStream_t st,
                            int block);
cudaError_t launch_kdown64(const RenderParams &p, const double *data, double *k,
                           cudaStream_t st);
cudaError_t launch_getuu64(const RenderParams &p, const double *data, double *info,
                           cudaStream_t st);
cudaError_t launch_coords64(const RenderParams &p, const double *data, double *out,
                            int system, double r_match, int as_written, cudaStream_t st);
cudaError_t launch_transpose(const double *src, double *dst, long long n_rays,
                             int n_data, int to_aos, cudaStream_t st);

/* launch shape of the persistent kernels */
struct MixedLaunch {
	int block;        /* threads per block                              */
	int blocks_per_sm;/* 0: from the occupancy calculator               */
	int sms;
	int rays_per_thread; /* 1 or 2 (analytic kernel only)               */
	int rk4_rolled;      /* 0: RK4 stages unrolled; 1: one stage body looped */
};

/* numerical spacetime */
cudaError_t launch_dyst_icond(const RenderParams &p, const GridParams &g, double *data,
                              double *info, cudaStream_t st);
cudaError_t launch_dyst_evolve64(const RenderParams &p, const GridParams &g, double *data,
                                 double *info, double dt, long long n_sub,
                                 unsigned long long *steps, cudaStream_t st);
size_t      mixed_render_bytes(void); /* sizeof(MixedRender) */
cudaError_t launch_boosted_ks(const GridParams &g, float *lvl, double a, double v,
                              int axis, double t, cudaStream_t st);

#endif /* GRAY_INTERNAL_H */
