/*
 * CPU oracle for the GRay2 geodesic hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C FP64 restatement of the reference arithmetic
 * (luxsrc/gray, the sim-org OpenCL kernels).  It exists so that tests, the smoke check
 * and the CPU-baseline leg of the benchmark can check the CUDA path.  It is
 * never linked into, loaded by or called from the product library.
 *
 * Parity pins: the reference ships no golden vectors for this path (its
 * only test, tests/ck_sample.c, checks the lux planner).  The oracle is
 * pinned instead against vectors produced by the reference's own Python
 * spacetime code (tools/boosted_ks.py: metric and Christoffel symbols),
 * generated by tests/golden/make_golden.py, and against physics invariants
 * derived from the cited formulas.
 *
 * Rounding contract: compiled with -ffp-contract=off; every fused
 * multiply-add is an explicit fma() call, placed exactly where the FP64 CUDA
 * kernel places it, so both sides round identically.
 */
#ifndef GRAY_ORACLE_H
#define GRAY_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_FREQ 8

/* Termination rules. ORC_TERM_EPS is the reference rule
 * (sim-org/phys.cl:54, stop when r - r_+ < 0.01); ORC_TERM_RPLUS stops at
 * r < 1.01 r_+. */
enum { ORC_TERM_EPS = 0, ORC_TERM_RPLUS = 1 };

/* Flow models feeding the transfer equation. ORC_FLOW_THERMAL is the
 * reference's template flow (flow.cl:36-58) with rt.cl's emissivities. */
enum { ORC_FLOW_NONE = 0, ORC_FLOW_TORUS = 1, ORC_FLOW_THERMAL = 2 };

typedef struct {
	/* Kerr.opts */
	double a_spin;
	/* infcam.opts */
	double w_img, h_img, r_obs, i_obs, j_obs;
	int64_t w_rays, h_rays;
	/* gray.opts / setup.opts step control and output times */
	double  t_init, dt_dump;
	int64_t n_sub, n_dump;
	int     term;
	/* radiative transfer */
	int     n_freq;
	double  nu[ORC_MAX_FREQ];
	int     flow;
	double  torus_n0, torus_kappa, torus_hr;
	/* thermal flow: M_ADM (param.opts:5), T_e (flow.cl:49), |b| along z */
	double  m_adm, flow_te, flow_b;
} orc_desc;

/* Numerical spacetime grid (interp.cl / dyst.cl).  fields[lvl] points to
 * nz*ny*nx*51 floats stored [z][y][x][comp] with comps ordered Gamma (40,
 * i-major then j<=k), g (10, i<=j), rho (1).  Coordinates are given by the
 * bounding box and the n=3 fisheye map of interp.cl:89-96. */
typedef struct {
	int    nx, ny, nz;
	float  box[8];             /* {t1, xmin, ymin, zmin, t2, xmax, ymax, zmax} */
	const float *fields[2];    /* time levels t1, t2 */
	int    bug_gzz;            /* 1: reproduce dyst.cl:78 (g_zz read as g_yz) */
	int    physics;            /* 1: flat outside the box, time factor in [0,1] */
} orc_grid;

/* ---- analytic Kerr-Schild pieces (KS.cl) ---- */
double orc_getrr(double a, const double q[4]);
double orc_geteps(double a, const double q[4]);
void   orc_down(double a, const double q[4], const double u[4], double k[4]);
double orc_getuu(double a, const double s[8]);
/* KS.cl:63-153 output coordinates: spherical Kerr-Schild and
 * Boyer-Lindquist events and vectors; r_match is where t_BL = t_KS;
 * as_written = 1 reproduces KS.cl's phi convention and getBLu terms */
void   orc_getsphKS(double a, const double q[4], int as_written, double out[4]);
void   orc_getBL(double a, double r_match, const double q[4], int as_written,
                 double out[4]);
void   orc_getsphKSu(double a, const double q[4], const double u[4], int as_written,
                     double out[4]);
void   orc_getBLu(double a, const double q[4], const double u[4], int as_written,
                  double out[4]);
void   orc_ks_rhs(double a, const double s[8], double ds[8]);

/* Per-render camera constants computed once on the host:
 * {cos i, sin i, cos j, sin j} (KS.cl:195-197). */
void   orc_camera(const orc_desc *d, double cam[4]);
void   orc_icond(const orc_desc *d, const double cam[4], int64_t ray, double *state);

/* step control (phys.cl:48-64) */
double orc_getdt(const orc_desc *d, const double q[4], double dt);

/* full right-hand side (phys.cl:66-74) for KS + optional torus transfer */
void   orc_rhs(const orc_desc *d, const double *s, double *ds);

/* one RK4 step (RK4.cl:37-47) on n_data = 8 + 2 n_freq reals */
void   orc_integrate(const orc_desc *d, double *s, double dt);

/* one dump interval of the integer-tick substep loop (driver.cl:69-108);
 * returns the number of accepted RK4 steps */
int64_t orc_evolve_ray(const orc_desc *d, double *s, double dt, int64_t n_sub);

/* icond + all n_dump intervals for a list of rays.  out is [k][n_data],
 * info is [k], steps is [k]. */
int    orc_trace(const orc_desc *d, const int64_t *rays, int64_t n,
                 double *out, double *info, int64_t *steps, int nthreads);

/* the same trace with every real in float (the reference's default
 * precision, sim-org/setup.opts:6), gray_oracle32.c: the single-precision
 * CPU baseline; out is [k][n_data] doubles, steps is [k] */
int    orc32_trace(const orc_desc *d, const int64_t *rays, int64_t n,
                   double *out, int64_t *steps, int nthreads);

/* same, but only n_dump intervals starting from given states (in/out). */
int    orc_evolve_states(const orc_desc *d, double *states, int64_t n,
                         double *info, int64_t *steps, int nthreads);

/* ---- torus constants ---- */
double orc_rplus(double a);
double orc_risco(double a);

/* ---- thermal emissivities (rt.cl:28-170) ---- */
double orc_log_K2it(double te);
double orc_B_Planck(double nu, double te);
double orc_Gaunt(double x, double y);
double orc_L_j_ff(double m_adm, double nu, double te, double ne);
double orc_L_j_syn(double m_adm, double nu, double te, double ne, double b, double cos_theta);

/* ---- numerical spacetime (interp.cl, dyst.cl) ---- */
double orc_interp(const orc_grid *g, const double q[4], int comp);
void   orc_dyst_rhs(const orc_grid *g, const double s[8], double ds[8]);
/* geodesic + thermal transfer on n_data = 8 + 2 n_freq reals (phys.cl:66-74) */
void   orc_dyst_rhs_rt(const orc_desc *d, const orc_grid *g, const double *s, double *ds);
void   orc_dyst_down(const orc_grid *g, const double q[4], const double u[4], double k[4]);
void   orc_dyst_icond(const orc_desc *d, const double cam[4], int64_t ray, double s[8]);
double orc_dyst_getdt(double dt);
int64_t orc_dyst_evolve_ray(const orc_desc *d, const orc_grid *g, double *s,
                            double dt, int64_t n_sub);
/* sim-org/gray.c:41-57 + 183-293: the snapshot pair of t_init (*first)
 * and of every dump interval (pairs[n_dump]); -1 where the reference stops */
int    orc_series_schedule(const double *times, int64_t n_times, double t_init,
                           double dt_dump, int64_t n_dump, int fast_light,
                           int64_t *first, int64_t *pairs);
/* the dyst trace across a snapshot series: g gives shape, box and flags;
 * snaps[k] are interleaved [z][y][x][51] levels at times[k] */
int    orc_dyst_series_trace(const orc_desc *d, const orc_grid *g,
                             const float *const *snaps, const double *times,
                             int64_t n_times, int fast_light, const int64_t *rays,
                             int64_t n, double *out, double *info, int64_t *steps,
                             int nthreads);
int    orc_dyst_trace(const orc_desc *d, const orc_grid *g, const int64_t *rays,
                      int64_t n, double *out, double *info, int64_t *steps,
                      int nthreads);

/* boosted Kerr-Schild sampler (restates tools/boosted_ks.py:120-186 and its
 * dual-number Christoffel construction :191-275 with closed-form derivatives).
 * out[0..39] = Gamma^i_jk (i-major, j<=k), out[40..49] = g_ij (i<=j). */
void   orc_boosted_ks(double m, double a, double v, int axis,
                      const double q[4], double out[50]);

#ifdef __cplusplus
}
#endif

#endif /* GRAY_ORACLE_H */
