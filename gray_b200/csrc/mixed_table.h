/*
 * Render table of the mixed-precision persistent kernels.  One entry per
 * render: FP32 constants for the bulk arithmetic, FP64 copies for the FP64
 * islands, the render's state buffers and its dump schedule.  A batch of
 * renders (many cameras, spins, resolutions) is one table and one launch.
 */
#ifndef GRAY_MIXED_TABLE_H
#define GRAY_MIXED_TABLE_H

#include "gray_internal.h"

/* The thermal emissivities of rt.cl:80-170 with everything that depends
 * only on the render's temperature, field and mass folded into per-render
 * constants (FP64, on the host), so that per frequency and RHS only the
 * frequency-dependent part is evaluated. */
struct ThermalFast {
	double kf2;       /* B_Planck: f2 = h nu / (m_e c^2 te) = nu kf2          */
	double kB;        /* B = kB nu^3 / (e^f2 - 1), kB = 2 h / c^2              */
	double kB2;       /* f2 <= 1e-5: B = kB2 nu^2 / (1 + f2/2 + f2^2/6)        */
	double ky;        /* Gaunt y = nu ky                                      */
	double xg, sxg;   /* Gaunt x (te only) and sqrt(x)                        */
	double g1, g2, g3, g4, g5;
	double kff;       /* L_ff = kff ne^2 G / (sqrt(te) e^y + EPS)              */
	double sqte;      /* sqrt(te)                                             */
	double knus;      /* nu_s = knus sin(theta)                               */
	double ksyn;      /* L_syn = ksyn xx^2 e^-cbrt(x) ne nu_s                  */
	double b;         /* field magnitude                                      */
	int    syn;       /* te > T_MIN and b != 0 (else L_syn is exactly 0)      */
};

struct MixedRender {
	float  a, aa, rp, risco, eps_stop;
	float  cdt_scale;          /* 0.01: the step fraction of phys.cl:60-61     */
	float  kappa, n0_rp15, ihr2_log2e;
	float  nupow[GRAY_MAX_FREQ];
	float  nuinv2[GRAY_MAX_FREQ];
	/* the analytic torus folded for the Hamiltonian kernel: log2 of the
	 * density scale n0 r_+^1.5 (-inf without the torus flow),
	 * -kappa nu_0^-2 n0 r_+^1.5, and -log2(e) (nu_0/nu_i)^2, which turns
	 * tau_0 into -log2(e) tau_i */
	float  ln0t, ktau;
	float  tcoef[GRAY_MAX_FREQ];
	int    flow;
	int    dump_begin;         /* integrate dump intervals [dump_begin,        */
	int    dump_end;           /*   dump_end) of the render's schedule          */
	int    n_ticks;            /* ticks per dump interval: a multiple of n_sub */
	double a_d, aa_d, rp_d;    /* FP64 islands                                */
	double *data, *info;       /* SoA FP64 state and getuu diagnostic         */
	long long n_rays;
	double t_init, dt_dump;    /* dump i covers [t_init + i dt, t_init + (i+1) dt] */
	long long n_sub;
	/* thermal flow of numerical renders */
	double nu_hz[GRAY_MAX_FREQ];
	ThermalFast tf;
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

/* rays_per_thread: 1 (scalar FP32) or 2 (two rays per thread in f32x2).
 * one (nullable): a host copy of the table's only render; with it, a
 * one-render launch passes the render as a kernel parameter, so that its
 * constants are read from the constant bank instead of held in registers
 * per ray. */
cudaError_t launch_mixed_table(const MixedTable &T, int n_freq, unsigned int *queue,
                               unsigned long long *steps, cudaStream_t st,
                               const MixedLaunch &cfg, const MixedRender *one = nullptr);

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
