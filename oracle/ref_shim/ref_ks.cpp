/*
 * The reference's analytic Kerr-Schild program (sim-org: preamble.cl, KS.cl,
 * flow.cl, rt.cl, AoS.cl, phys.cl, RK4.cl, driver.cl -- the source list of
 * sim-org/build.c:85-95 with coordinates = KS.cl), compiled from the
 * reference's own files with opencl_shim.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Two things the sources leave open are supplied here, and nothing else:
 *  - the build-time definitions sim-org/build.c:100-122 prepends (n_freq,
 *    n_data, n_info, the ray counts, n_chunk, realE, nus, M_ADM), and the
 *    constants KS.cl uses but never defines (a_spin, r_match);
 *  - KS.cl's functions take no spacetime arguments while phys.cl and
 *    driver.cl pass them (phys.cl:70-72, driver.cl:65): forwarding overloads
 *    drop them, which is what a working build of the sources would need.
 *    getflow (flow.cl) reads the numerical grid's rho, which the analytic
 *    spacetime does not have: the overload here returns a flow with no
 *    electrons (n_e = 0), so the transfer state stays zero.
 * The entry points run icond_drv and evolve_drv over a list of rays, one
 * work-item at a time per host thread, as the reference's host loop
 * (sim-org/gray.c:243-294) drives them dump by dump.
 */
#define GRAY_SHIM_NO_IMAGES /* the analytic program reads no image */
#include "opencl_shim.h"

#include <cstdlib>
#include <vector>

thread_local size_t gray_shim_gid[2];

namespace ref_ks {

/* sim-org/build.c:100-122.  One frequency with no emission (the flow
 * below has n_e = 0), so the transfer state stays zero: OpenCL C has no
 * zero-length arrays for n_freq = 0, and the geodesic does not depend on it */
#define n_freq 1
#define n_data 10
#define n_info 1
static size_t w_rays_v, h_rays_v;
#define w_rays w_rays_v
#define h_rays h_rays_v
#define n_rays (w_rays_v * h_rays_v)
#define n_chunk 5
typedef real2 realE;
static real nus[1] = {1};
static real M_ADM = 0;
static real a_spin, r_match = 10;

#include "preamble.cl"
#include "interp.cl"
#include "KS.cl"

template <typename... A> real4 down(real4 q, real4 u, A...) { return down(q, u); }
template <typename... A> real getuu(struct gr g, A...) { return getuu(g); }
template <typename... A> struct gr gr_rhs(struct gr g, A...) { return gr_rhs(g); }

#define getflow getflow_grid /* flow.cl's grid flow: needs the grid's rho */
#include "flow.cl"
#undef getflow
template <typename... A> struct flow getflow(real4, real4, A...)
{
	struct flow f = {0, 1e12, 0, 0, 1}; /* ne, te, b, bkcos, shift */
	return f;
}

#include "rt.cl"
#include "AoS.cl"
#include "phys.cl"

/* RK4.cl's integrate() under another name, and a forwarding integrate()
 * that counts the calls: driver.cl calls it once per accepted step, so the
 * count is the ray-steps of the reference's own loop */
thread_local long long ref_steps;
#define integrate ref_integrate
#include "RK4.cl"
#undef integrate
template <typename... A> struct state integrate(struct state s, real dt, A... a)
{
	++ref_steps;
	return ref_integrate(s, dt, a...);
}

#include "driver.cl"

} /* namespace ref_ks */

using namespace ref_ks;

/* a render's camera and step control, as the host passes them */
struct ref_ks_desc {
	double a_spin, w_img, h_img, r_obs, i_obs, j_obs;
	int64_t w_rays, h_rays;
	double t_init, dt_dump;
	int64_t n_sub, n_dump;
};

extern "C" {

/* KS.cl functions one at a time: q[4], u[4] in, results out */
double ref_ks_getrr(double a, const double *q)
{
	a_spin = a;
	return getrr(real4{q[0], q[1], q[2], q[3]});
}
double ref_ks_geteps(double a, const double *q)
{
	a_spin = a;
	return geteps(real4{q[0], q[1], q[2], q[3]});
}
void ref_ks_down(double a, const double *q, const double *u, double *k)
{
	a_spin = a;
	real4 r = down(real4{q[0], q[1], q[2], q[3]}, real4{u[0], u[1], u[2], u[3]});
	for(int i = 0; i < 4; ++i)
		k[i] = r.v[i];
}
void ref_ks_rhs(double a, const double *s, double *ds)
{
	a_spin = a;
	struct gr g = {real4{s[0], s[1], s[2], s[3]}, real4{s[4], s[5], s[6], s[7]}};
	struct gr d = gr_rhs(g);
	for(int i = 0; i < 4; ++i) {
		ds[i] = d.q.v[i];
		ds[4 + i] = d.u.v[i];
	}
}

/* icond_drv + evolve_drv per dump for the listed rays: out [n][8] (x^mu,
 * u^mu), info [n], the state after n_dump intervals; steps [n] (nullable)
 * the accepted RK4 steps of each ray.  nthreads host threads share the
 * list (at least one). */
int ref_ks_trace(const ref_ks_desc *d, const int64_t *rays, int64_t n, double *out,
                 double *info, int64_t *steps, int nthreads)
{
	a_spin = d->a_spin;
	w_rays_v = (size_t)d->w_rays;
	h_rays_v = (size_t)d->h_rays;
	real8 bounding_box = {};
	int4 num_points = {};
	image3d_t Gamma_ttt_t1 = {}, Gamma_ttx_t1 = {}, Gamma_tty_t1 = {}, Gamma_ttz_t1 = {},
	          Gamma_txx_t1 = {}, Gamma_txy_t1 = {}, Gamma_txz_t1 = {}, Gamma_tyy_t1 = {},
	          Gamma_tyz_t1 = {}, Gamma_tzz_t1 = {}, Gamma_xtt_t1 = {}, Gamma_xtx_t1 = {},
	          Gamma_xty_t1 = {}, Gamma_xtz_t1 = {}, Gamma_xxx_t1 = {}, Gamma_xxy_t1 = {},
	          Gamma_xxz_t1 = {}, Gamma_xyy_t1 = {}, Gamma_xyz_t1 = {}, Gamma_xzz_t1 = {},
	          Gamma_ytt_t1 = {}, Gamma_ytx_t1 = {}, Gamma_yty_t1 = {}, Gamma_ytz_t1 = {},
	          Gamma_yxx_t1 = {}, Gamma_yxy_t1 = {}, Gamma_yxz_t1 = {}, Gamma_yyy_t1 = {},
	          Gamma_yyz_t1 = {}, Gamma_yzz_t1 = {}, Gamma_ztt_t1 = {}, Gamma_ztx_t1 = {},
	          Gamma_zty_t1 = {}, Gamma_ztz_t1 = {}, Gamma_zxx_t1 = {}, Gamma_zxy_t1 = {},
	          Gamma_zxz_t1 = {}, Gamma_zyy_t1 = {}, Gamma_zyz_t1 = {}, Gamma_zzz_t1 = {},
	          g_tt_t1 = {}, g_tx_t1 = {}, g_ty_t1 = {}, g_tz_t1 = {}, g_xx_t1 = {},
	          g_xy_t1 = {}, g_xz_t1 = {}, g_yy_t1 = {}, g_yz_t1 = {}, g_zz_t1 = {},
	          rho_t1 = {};
	image3d_t Gamma_ttt_t2 = {}, Gamma_ttx_t2 = {}, Gamma_tty_t2 = {}, Gamma_ttz_t2 = {},
	          Gamma_txx_t2 = {}, Gamma_txy_t2 = {}, Gamma_txz_t2 = {}, Gamma_tyy_t2 = {},
	          Gamma_tyz_t2 = {}, Gamma_tzz_t2 = {}, Gamma_xtt_t2 = {}, Gamma_xtx_t2 = {},
	          Gamma_xty_t2 = {}, Gamma_xtz_t2 = {}, Gamma_xxx_t2 = {}, Gamma_xxy_t2 = {},
	          Gamma_xxz_t2 = {}, Gamma_xyy_t2 = {}, Gamma_xyz_t2 = {}, Gamma_xzz_t2 = {},
	          Gamma_ytt_t2 = {}, Gamma_ytx_t2 = {}, Gamma_yty_t2 = {}, Gamma_ytz_t2 = {},
	          Gamma_yxx_t2 = {}, Gamma_yxy_t2 = {}, Gamma_yxz_t2 = {}, Gamma_yyy_t2 = {},
	          Gamma_yyz_t2 = {}, Gamma_yzz_t2 = {}, Gamma_ztt_t2 = {}, Gamma_ztx_t2 = {},
	          Gamma_zty_t2 = {}, Gamma_ztz_t2 = {}, Gamma_zxx_t2 = {}, Gamma_zxy_t2 = {},
	          Gamma_zxz_t2 = {}, Gamma_zyy_t2 = {}, Gamma_zyz_t2 = {}, Gamma_zzz_t2 = {},
	          g_tt_t2 = {}, g_tx_t2 = {}, g_ty_t2 = {}, g_tz_t2 = {}, g_xx_t2 = {},
	          g_xy_t2 = {}, g_xz_t2 = {}, g_yy_t2 = {}, g_yz_t2 = {}, g_zz_t2 = {},
	          rho_t2 = {};
	for(int64_t j = 0; j < n; ++j)
		if(rays[j] < 0 || (size_t)rays[j] >= n_rays)
			return -1;
	/* the whole render's arrays, as the reference allocates them; each
	 * work-item touches only its own ray's slots, so the listed rays can
	 * run on several threads at once */
	std::vector<real> data((size_t)n_data * n_rays), inf((size_t)n_info * n_rays);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
	for(int64_t j = 0; j < n; ++j) {
		const int64_t g = rays[j];
		gray_shim_gid[0] = (size_t)(g / d->w_rays); /* gj: row    */
		gray_shim_gid[1] = (size_t)(g % d->w_rays); /* gi: column */
		const long long s0 = ref_steps;
		icond_drv(data.data(), inf.data(), d->w_img, d->h_img, d->r_obs, d->i_obs, d->j_obs,
		          nullptr, SPACETIME_ARGS);
		/* sim-org/gray.c:248-257: one evolve per dump interval */
		for(int64_t i = 0; i < d->n_dump;) {
			const real t = d->t_init + (real)i * d->dt_dump;
			const real target = d->t_init + (real)(++i) * d->dt_dump;
			evolve_drv(data.data(), inf.data(), target - t, (whole)d->n_sub, nullptr,
			           SPACETIME_ARGS);
		}
		for(int s = 0; s < 8; ++s)
			out[j * 8 + s] = data[(size_t)g * n_data + s];
		info[j] = inf[(size_t)g];
		if(steps)
			steps[j] = (int64_t)(ref_steps - s0);
	}
	return 0;
}

} /* extern "C" */
