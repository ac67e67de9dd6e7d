/*
 * Render table of the mixed-precision persistent kernels.  One entry per
 * render: FP32 constants for the bulk arithmetic, FP64 copies for the FP64
 * islands, the render's state buffers and its dump schedule.  A batch of
 * renders (many cameras, spins, resolutions) is one table and one launch.
 */
#ifndef GRAY_MIXED_TABLE_H
#define GRAY_MIXED_TABLE_H

#include "gray_internal.h"

struct MixedRender {
	float  a, aa, rp, risco, eps_stop;
	float  cdt_scale;          /* 0.01: the step fraction of phys.cl:60-61     */
	float  kappa, n0_rp15, ihr2_log2e;
	float  nupow[GRAY_MAX_FREQ];
	float  nuinv2[GRAY_MAX_FREQ];
	int    flow;
	int    dump_begin;         /* integrate dump intervals [dump_begin,        */
	int    dump_end;           /*   dump_end) of the render's schedule          */
	double a_d, aa_d, rp_d;    /* FP64 islands                                */
	double *data, *info;       /* SoA FP64 state and getuu diagnostic         */
	long long n_rays;
	double t_init, dt_dump;    /* dump i covers [t_init + i dt, t_init + (i+1) dt] */
	long long n_sub;
	/* thermal flow of numerical renders (FP64 transfer) */
	double nu_hz[GRAY_MAX_FREQ];
	double m_adm, flow_te, flow_b;
	ThermalConsts th;
	int    thermal;
};

struct MixedTable {
	const MixedRender *renders;        /* device array [n_renders]           */
	const unsigned long long *prefix;  /* device array: first global index   */
	int n_renders;
	unsigned long long total;          /* rays over all renders              */
};

void fill_mixed_render(const RenderParams &p, double *data, double *info,
                       double t_init, double dt_dump, long long n_dump,
                       long long n_sub, MixedRender *m);

/* rays_per_thread: 1 (scalar FP32) or 2 (two rays per thread in f32x2) */
cudaError_t launch_mixed_table(const MixedTable &T, int n_freq, unsigned int *queue,
                               unsigned long long *steps, cudaStream_t st,
                               const MixedLaunch &cfg);

/* numerical spacetime: every render of the table on the same grid and with
 * the same n_freq; inbox (nullable) accumulates the steps that interpolate
 * the grid */
cudaError_t launch_dyst_mixed_table(const MixedTable &T, const GridParams &g, int n_freq,
                                    unsigned int *queue, unsigned long long *steps,
                                    cudaStream_t st, const MixedLaunch &cfg,
                                    unsigned long long *inbox = nullptr);

/* resident blocks per SM of the mixed kernel for a launch shape */
cudaError_t mixed_occupancy(int n_freq, const MixedLaunch &cfg, int *blocks_per_sm);

#endif /* GRAY_MIXED_TABLE_H */
