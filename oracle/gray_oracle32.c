/*
 * FP32 build of the CPU restatement -- TEST AND BASELINE INFRASTRUCTURE ONLY.
 * Only bench.py's CPU legs and tests/ load it (through liborc.so).
 *
 * The reference's default build computes in single precision: `real` is
 * float unless precision:p asks otherwise (sim-org/setup.opts:6, size of
 * float; the kernels are built with that real type, sim-org/build.c:138).
 * This file is the analytic Kerr-Schild + torus path of gray_oracle.c with
 * every real in float -- camera (KS.cl:188-232 via driver.cl:36-67), the
 * geodesic right-hand side (KS.cl:263-378), getdt (phys.cl:48-64), RK4
 * (RK4.cl:37-47), the integer-tick loop (driver.cl:81-99) and the torus
 * transfer (rt.cl:185-198 form) -- so that the CPU baseline has a like-for-
 * like single-precision figure beside the FP64 one.  Its results are not a
 * parity reference; the FP64 restatement is.
 */
#include "gray_oracle.h"

#include <limits.h>
#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EPS0 1e-28f /* sim-org/preamble.cl:30 */
#define ND32 (8 + 2 * ORC_MAX_FREQ)

typedef struct {
	float a, rp, risco, eps_stop;
	float n0, kappa, hr;
	int   nf, flow;
	float nupow[ORC_MAX_FREQ], nuinv2[ORC_MAX_FREQ];
} c32;

/* KS.cl:48-61 */
static float
getrr32(float a, const float *q)
{
	float aa = a * a, zz = q[3] * q[3];
	float kk = 0.5f * (q[1] * q[1] + q[2] * q[2] + zz - aa);
	return sqrtf(kk * kk + aa * zz) + kk;
}

typedef struct {
	float r, f, lx, ly, lz, flu, iss;
} aux32;

/* KS.cl:263-378, the Chan et al. grouping in float */
static void
rhs32_ks(float a, const float *s, float *ds, aux32 *x)
{
	const float X = s[1], Y = s[2], Z = s[3];
	const float ut = s[4], ux = s[5], uy = s[6], uz = s[7];
	float aa = a * a, zz = Z * Z;
	float kk = 0.5f * (X * X + Y * Y + zz - aa);
	float dd = sqrtf(kk * kk + aa * zz);
	float rr = dd + kk, r = sqrtf(rr), ir = 1.0f / r;
	float ss = rr + aa, iss = 1.0f / ss;
	float tmp = 0.5f / (r * dd);
	float dz_r = tmp * ss * Z;
	tmp *= rr;
	float dy_r = tmp * Y, dx_r = tmp * X;
	tmp = 2.0f / (rr + aa * zz / rr);
	float tmp2 = 3.0f - 2.0f * rr * tmp;
	float f = tmp * r;
	float dx_f = tmp * dx_r * tmp2, dy_f = tmp * dy_r * tmp2;
	float dz_f = tmp * (dz_r * tmp2 - tmp * aa * Z * ir);

	float m2r = -2.0f * r, issr = iss * r, issa = iss * a;
	float lx = iss * (X * r + Y * a);
	tmp = iss * (X + m2r * lx);
	float dx_lx = tmp * dx_r + issr, dy_lx = tmp * dy_r + issa, dz_lx = tmp * dz_r;
	float ly = iss * (Y * r - X * a);
	tmp = iss * (Y + m2r * ly);
	float dx_ly = tmp * dx_r - issa, dy_ly = tmp * dy_r + issr, dz_ly = tmp * dz_r;
	float lz = Z * ir;
	tmp = -lz * ir;
	float dx_lz = tmp * dx_r, dy_lz = tmp * dy_r, dz_lz = tmp * dz_r + ir;

	float lu = ut + lx * ux + ly * uy + lz * uz, flu = f * lu;
	float Dx0 = dx_f * lu + f * (dx_lx * ux + dx_ly * uy + dx_lz * uz);
	float Dy0 = dy_f * lu + f * (dy_lx * ux + dy_ly * uy + dy_lz * uz);
	float Dz0 = dz_f * lu + f * (dz_lx * ux + dz_ly * uy + dz_lz * uz);
	float Dx1 = Dx0 * lx + flu * dx_lx, Dx2 = Dx0 * ly + flu * dx_ly, Dx3 = Dx0 * lz + flu * dx_lz;
	float Dy1 = Dy0 * lx + flu * dy_lx, Dy2 = Dy0 * ly + flu * dy_ly, Dy3 = Dy0 * lz + flu * dy_lz;
	float Dz1 = Dz0 * lx + flu * dz_lx, Dz2 = Dz0 * ly + flu * dz_ly, Dz3 = Dz0 * lz + flu * dz_lz;
	float hDxu = 0.5f * (Dx0 * ut + Dx1 * ux + Dx2 * uy + Dx3 * uz);
	float hDyu = 0.5f * (Dy0 * ut + Dy1 * ux + Dy2 * uy + Dy3 * uz);
	float hDzu = 0.5f * (Dz0 * ut + Dz1 * ux + Dz2 * uy + Dz3 * uz);
	float uD0 = ux * Dx0 + uy * Dy0 + uz * Dz0;
	float uD1 = ux * Dx1 + uy * Dy1 + uz * Dz1;
	float uD2 = ux * Dx2 + uy * Dy2 + uz * Dz2;
	float uD3 = ux * Dx3 + uy * Dy3 + uz * Dz3;
	tmp = f * (-uD0 + lx * (uD1 - hDxu) + ly * (uD2 - hDyu) + lz * (uD3 - hDzu));
	ds[0] = ut; ds[1] = ux; ds[2] = uy; ds[3] = uz;
	ds[4] = uD0 - tmp;
	ds[5] = hDxu - uD1 + lx * tmp;
	ds[6] = hDyu - uD2 + ly * tmp;
	ds[7] = hDzu - uD3 + lz * tmp;
	x->r = r; x->f = f; x->lx = lx; x->ly = ly; x->lz = lz; x->flu = flu; x->iss = iss;
}

/* the analytic torus of the FP64 restatement, in float */
static void
rhs32(const c32 *c, const float *s, float *ds)
{
	aux32 x;
	rhs32_ks(c->a, s, ds, &x);
	const int nf = c->nf;
	if(nf == 0)
		return;
	float n = 0.0f, shift = 1.0f;
	if(c->flow == ORC_FLOW_TORUS && x.r > c->risco) {
		float kt = x.flu - s[4], kx = x.flu * x.lx + s[5], ky = x.flu * x.ly + s[6];
		float R2 = s[1] * s[1] + s[2] * s[2];
		float Om = 1.0f / (x.r * sqrtf(x.r) + c->a);
		float vv = Om * Om * R2 - 1.0f;
		float lv = 1.0f - c->a * Om * R2 * x.iss;
		float D = -(x.f * lv * lv + vv);
		if(D > 0.0f) {
			shift = -(Om * (s[1] * ky - s[2] * kx) + kt) / sqrtf(D);
			if(shift > 0.0f) {
				float qr = c->rp / x.r, hz = c->hr * x.r;
				n = c->n0 * qr * sqrtf(qr) * expf(-(s[3] * s[3]) / (2.0f * hz * hz));
			}
		}
	}
	if(n == 0.0f) {
		for(int i = 0; i < 2 * nf; ++i)
			ds[8 + i] = 0.0f;
		return;
	}
	float jfac = n * powf(shift, -0.7f), tfac = c->kappa * n / shift;
	float is2 = 1.0f / (shift * shift + EPS0);
	for(int i = 0; i < nf; ++i) {
		ds[8 + i] = -(jfac * c->nupow[i] * expf(-s[8 + nf + i])) * is2;
		ds[8 + nf + i] = -(tfac * c->nuinv2[i]);
	}
}

/* phys.cl:48-64 */
static float
getdt32(const c32 *c, const float *q, float dt)
{
	float eps = sqrtf(getrr32(c->a, q)) - c->rp;
	if(eps < c->eps_stop)
		return 0.0f;
	float cap = 0.01f * eps * eps;
	return fabsf(dt) > cap ? copysignf(cap, dt) : dt;
}

/* RK4.cl:37-47 */
static void
rk4_32(const c32 *c, int nd, float *s, float dt)
{
	float k1[ND32], k2[ND32], k3[ND32], k4[ND32], t[ND32];
	int i;
	rhs32(c, s, k1);
	for(i = 0; i < nd; ++i) t[i] = s[i] + 0.5f * dt * k1[i];
	rhs32(c, t, k2);
	for(i = 0; i < nd; ++i) t[i] = s[i] + 0.5f * dt * k2[i];
	rhs32(c, t, k3);
	for(i = 0; i < nd; ++i) t[i] = s[i] + dt * k3[i];
	rhs32(c, t, k4);
	for(i = 0; i < nd; ++i)
		s[i] += dt * (k1[i] + 2.0f * (k2[i] + k3[i]) + k4[i]) / 6.0f;
}

/* driver.cl:81-99 in float: dh = getdt / dt * n, truncated */
static int64_t
ticks32(const c32 *c, int nd, float *s, float dt, int64_t n_sub)
{
	const int n = (int)((INT_MAX / n_sub) * n_sub);
	int64_t steps = 0;
	int h, dh;
	for(h = 0; h < n; h += dh) {
		dh = (int)(getdt32(c, s, dt / (float)n_sub) / dt * (float)n);
		if(dh <= 0)
			break;
		if(dh > n - h)
			dh = n - h;
		rk4_32(c, nd, s, (float)dh * dt / (float)n);
		++steps;
	}
	return steps;
}

int
orc32_trace(const orc_desc *d, const int64_t *rays, int64_t n, double *out, int64_t *steps,
            int nthreads)
{
	const int nd = 8 + 2 * d->n_freq;
	c32 c;
	if(d->n_freq < 0 || d->n_freq > ORC_MAX_FREQ || d->n_sub <= 0)
		return -1;
	memset(&c, 0, sizeof(c));
	c.a = (float)d->a_spin;
	c.rp = 1.0f + sqrtf(1.0f - c.a * c.a);
	c.risco = (float)orc_risco(d->a_spin);
	c.eps_stop = d->term == ORC_TERM_RPLUS ? 0.01f * c.rp : 0.01f;
	c.n0 = (float)d->torus_n0;
	c.kappa = (float)d->torus_kappa;
	c.hr = (float)d->torus_hr;
	c.nf = d->n_freq;
	c.flow = d->flow;
	for(int i = 0; i < d->n_freq; ++i) {
		c.nupow[i] = powf((float)d->nu[i], -0.7f);
		c.nuinv2[i] = 1.0f / ((float)d->nu[i] * (float)d->nu[i]);
	}
	const float deg = 3.14159265358979f / 180.0f;
	const float ci = cosf(deg * (float)d->i_obs), si = sinf(deg * (float)d->i_obs);
	const float cj = cosf(deg * (float)d->j_obs), sj = sinf(deg * (float)d->j_obs);
#ifdef _OPENMP
	if(nthreads <= 0)
		nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
	for(int64_t j = 0; j < n; ++j) {
		float s[ND32];
		/* driver.cl:47-57 pixel map, KS.cl:199-229 camera ray */
		const int64_t gi = rays[j] % d->w_rays, gj = rays[j] / d->w_rays;
		float alpha = (((float)gi + 0.5f) / (float)d->w_rays - 0.5f) * (float)d->w_img;
		float beta  = (((float)gj + 0.5f) / (float)d->h_rays - 0.5f) * (float)d->h_img;
		float r_obs = (float)d->r_obs;
		float R0 = r_obs * si - beta * ci, z = r_obs * ci + beta * si;
		s[0] = 0.0f; s[1] = R0 * cj - alpha * sj; s[2] = R0 * sj + alpha * cj; s[3] = z;
		float ux = si * cj, uy = si * sj, uz = ci;
		{
			aux32 x;
			float tmp[8] = {s[0], s[1], s[2], s[3], 1.0f, 0.0f, 0.0f, 0.0f}, dtmp[8];
			rhs32_ks(c.a, tmp, dtmp, &x);
			float flx = x.f * x.lx, fly = x.f * x.ly, flz = x.f * x.lz;
			float A = x.f - 1.0f;
			float B = 2.0f * (flx * ux + fly * uy + flz * uz);
			float Cx = (flx * x.lx + 1.0f) * ux + flx * x.ly * uy + flx * x.lz * uz;
			float Cy = fly * x.lx * ux + (fly * x.ly + 1.0f) * uy + fly * x.lz * uz;
			float Cz = flz * x.lx * ux + flz * x.ly * uy + (flz * x.lz + 1.0f) * uz;
			float C = Cx * ux + Cy * uy + Cz * uz;
			float den = -(B + sqrtf(B * B - 4.0f * A * C)) / (2.0f * A);
			s[4] = 1.0f; s[5] = ux / den; s[6] = uy / den; s[7] = uz / den;
		}
		for(int i = 0; i < 2 * d->n_freq; ++i)
			s[8 + i] = 0.0f;
		int64_t st = 0;
		for(int64_t i = 0; i < d->n_dump;) {
			float t0 = (float)(d->t_init + (double)i * d->dt_dump);
			float t1 = (float)(d->t_init + (double)(++i) * d->dt_dump);
			st += ticks32(&c, nd, s, t1 - t0, d->n_sub);
		}
		steps[j] = st;
		for(int i = 0; i < nd; ++i)
			out[j * nd + i] = (double)s[i];
	}
	(void)nthreads;
	return 0;
}
