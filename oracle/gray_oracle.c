/*
 * CPU oracle for the GRay2 geodesic hot path -- TEST INFRASTRUCTURE ONLY.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this file's library, and only as the checker.
 *
 * Plain-C FP64 restatement of luxsrc/gray the sim-org OpenCL kernels.  Each function cites
 * the reference lines it follows.  Compile with -ffp-contract=off: every
 * fused multiply-add below is an explicit fma(), mirrored one-for-one by the
 * FP64 CUDA kernel, so the two agree bit for bit on the geodesic.
 */
#include "gray_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EPSILON 1e-28 /* sim-org/preamble.cl:30 */

/* ------------------------------------------------------------------------ */
/* Kerr-Schild radius and metric functions                                   */
/* ------------------------------------------------------------------------ */

/* KS.cl:48-55 getrr(): r^2 = sqrt(kk^2 + a^2 z^2) + kk,
 * kk = (x^2 + y^2 + z^2 - a^2) / 2. */
double
orc_getrr(double a, const double q[4])
{
	double aa = a * a;
	double zz = q[3] * q[3];
	double kk = 0.5 * (fma(q[1], q[1], fma(q[2], q[2], zz)) - aa);
	return sqrt(fma(kk, kk, aa * zz)) + kk;
}

double
orc_rplus(double a)
{
	return 1.0 + sqrt(1.0 - a * a);
}

/* KS.cl:57-61 geteps(): eps = r - r_+ (M = 1). */
double
orc_geteps(double a, const double q[4])
{
	return sqrt(orc_getrr(a, q)) - orc_rplus(a);
}

/* KS.cl:63-153 output coordinates.  The Cartesian Kerr-Schild event of the
 * metric of down() (l = (1, (r x + a y)/(r^2 + a^2), (r y - a x)/(r^2 + a^2),
 * z/r)) is x + i y = (r + i a) e^(i phi) sin(theta), z = r cos(theta), so
 * phi = arg((x + i y)(r - i a)).  KS.cl:68-69 takes arg((x + i y)(r + i a))
 * (and KS.cl:130 the matching d phi), and KS.cl:148-151 multiply u^phi and
 * u^t where the coordinate change has u^r: as_written = 1 reproduces those
 * lines, 0 gives coordinates in which the metric is Kerr's in
 * Boyer-Lindquist form. */

/* KS.cl:63-71 getsphKS(): (t, r, theta, phi) */
void
orc_getsphKS(double a, const double q[4], int as_written, double out[4])
{
	double r = sqrt(orc_getrr(a, q));
	double sa = as_written ? a : -a;
	out[0] = q[0];
	out[1] = r;
	out[2] = acos(q[3] / r);
	out[3] = atan2(fma(q[2], r, q[1] * sa), fma(q[1], r, -(q[2] * sa)));
}

/* KS.cl:73-89 getBL(): t matched to t_KS at r_match (a free parameter:
 * the reference never defines it), phi matched at r = infinity */
void
orc_getBL(double a, double r_match, const double q[4], int as_written, double out[4])
{
	double s[4];
	orc_getsphKS(a, q, as_written, s);
	double h  = sqrt(1.0 - a * a);
	double rp = 1.0 + h, rm = 1.0 - h, r = s[1];
	out[0] = s[0] + (rm * log((r - rm) / (r_match - rm)) -
	                 rp * log((r - rp) / (r_match - rp))) / h;
	out[1] = s[1];
	out[2] = s[2];
	out[3] = s[3] + 0.5 * a * log((r - rm) / (r - rp)) / h;
}

/* KS.cl:116-133 getsphKSu(): the Jacobian rows dr, dtheta, dphi of the
 * Cartesian KS position applied to u */
void
orc_getsphKSu(double a, const double q[4], const double u[4], int as_written, double out[4])
{
	double aa = a * a;
	double RR = fma(q[1], q[1], q[2] * q[2]);
	double zz = q[3] * q[3];
	double kk = 0.5 * (RR + zz - aa);
	double dd = sqrt(fma(kk, kk, aa * zz));
	double rr = dd + kk;
	double r  = sqrt(rr);
	double den = 2.0 * r * dd;
	double J1[4] = {0.0, rr * q[1] / den, rr * q[2] / den, (rr + aa) * q[3] / den};
	double zr = q[3] / r, sq = sqrt(rr - zz);
	double J2[4] = {0.0, zr * J1[1] / sq, zr * J1[2] / sq, (zr * J1[3] - 1.0) / sq};
	double c = (as_written ? -a : a) / (rr + aa);
	double J3[4] = {0.0, fma(c, J1[1], -q[2] / RR), fma(c, J1[2], q[1] / RR), c * J1[3]};
	out[0] = u[0];
	out[1] = fma(J1[3], u[3], fma(J1[2], u[2], J1[1] * u[1]));
	out[2] = fma(J2[3], u[3], fma(J2[2], u[2], J2[1] * u[1]));
	out[3] = fma(J3[3], u[3], fma(J3[2], u[2], J3[1] * u[1]));
}

/* KS.cl:135-153 getBLu(): dt_BL = dt - 2r/Delta dr, dphi_BL = dphi -
 * a/Delta dr */
void
orc_getBLu(double a, const double q[4], const double u[4], int as_written, double out[4])
{
	double v[4];
	orc_getsphKSu(a, q, u, as_written, v);
	double aa = a * a;
	double zz = q[3] * q[3];
	double kk = 0.5 * (fma(q[1], q[1], fma(q[2], q[2], zz)) - aa);
	double rr = sqrt(fma(kk, kk, aa * zz)) + kk;
	double r  = sqrt(rr);
	double D  = rr - 2.0 * r + aa;
	double ut = as_written ? v[3] : v[1]; /* multiplies 2r / Delta */
	double up = as_written ? v[0] : v[1]; /* multiplies a / Delta  */
	out[0] = v[0] - ut * 2.0 * r / D;
	out[1] = v[1];
	out[2] = v[2];
	out[3] = v[3] - up * a / D;
}

/* The KS scalar f and null covector l_mu = (1, lx, ly, lz), computed with
 * the same operation sequence as the head of orc_ks_rhs() (KS.cl:282-333),
 * so the reuse inside the RHS and the stand-alone down() agree bitwise. */
static void
ks_fl(double a, const double q[4], double *r_, double *f_, double *lx_,
      double *ly_, double *lz_, double *iss_)
{
	double aa  = a * a;
	double zz  = q[3] * q[3];
	double kk  = 0.5 * (fma(q[1], q[1], fma(q[2], q[2], zz)) - aa);
	double dd  = sqrt(fma(kk, kk, aa * zz));
	double rr  = dd + kk;
	double r   = sqrt(rr);
	double ir  = 1.0 / r;
	double ss  = rr + aa;
	double iss = 1.0 / ss;
	double tmp = 2.0 / (rr + (aa * zz) / rr);
	*r_   = r;
	*f_   = tmp * r;
	*lx_  = iss * fma(q[1], r, q[2] * a);
	*ly_  = iss * fma(q[2], r, -(q[1] * a));
	*lz_  = q[3] * ir;
	*iss_ = iss;
}

/* KS.cl:91-114 down(): k_mu = g_mu_nu u^nu with g = eta + f l l, written as
 * k = eta u + (f l.u) l. */
void
orc_down(double a, const double q[4], const double u[4], double k[4])
{
	double r, f, lx, ly, lz, iss;
	ks_fl(a, q, &r, &f, &lx, &ly, &lz, &iss);
	double lu  = fma(lz, u[3], fma(ly, u[2], fma(lx, u[1], u[0])));
	double flu = f * lu;
	k[0] = flu - u[0];
	k[1] = fma(flu, lx, u[1]);
	k[2] = fma(flu, ly, u[2]);
	k[3] = fma(flu, lz, u[3]);
}

static inline double
dot4(const double a[4], const double b[4])
{
	return fma(a[3], b[3], fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0])));
}

/* KS.cl:164-168 getuu(): g(u,u), the null-constraint diagnostic. */
double
orc_getuu(double a, const double s[8])
{
	double k[4];
	orc_down(a, s, s + 4, k);
	return dot4(k, s + 4);
}

/* ------------------------------------------------------------------------ */
/* Geodesic right-hand side (KS.cl:263-378, Chan et al. form)                */
/* ------------------------------------------------------------------------ */

typedef struct {
	double r, f, lx, ly, lz, flu, iss;
} ks_aux;

static void
ks_rhs_aux(double a, const double *s, double *ds, ks_aux *aux)
{
	const double x = s[1], y = s[2], z = s[3];
	const double ut = s[4], ux = s[5], uy = s[6], uz = s[7];

	double f, dx_f, dy_f, dz_f;
	double lx, dx_lx, dy_lx, dz_lx;
	double ly, dx_ly, dy_ly, dz_ly;
	double lz, dx_lz, dy_lz, dz_lz;
	double dx_r, dy_r, dz_r, r, ir, iss, tmp;

	{ /* KS.cl:282-309 */
		double aa = a * a;
		double zz = z * z;
		double kk = 0.5 * (fma(x, x, fma(y, y, zz)) - aa);
		double dd = sqrt(fma(kk, kk, aa * zz));
		double rr = dd + kk;
		r   = sqrt(rr);
		ir  = 1.0 / r;
		double ss = rr + aa;
		iss  = 1.0 / ss;
		tmp  = 0.5 / (r * dd);
		dz_r = (tmp * ss) * z;
		tmp  = tmp * rr;
		dy_r = tmp * y;
		dx_r = tmp * x;
		tmp  = 2.0 / (rr + (aa * zz) / rr);
		double tmp2 = fma(-2.0 * rr, tmp, 3.0);
		f    = tmp * r;
		dx_f = (tmp * dx_r) * tmp2;
		dy_f = (tmp * dy_r) * tmp2;
		dz_f = tmp * fma(dz_r, tmp2, -(((tmp * aa) * z) * ir));
	}
	{ /* KS.cl:312-334 */
		double m2r  = -2.0 * r;
		double issr = iss * r;
		double issa = iss * a;

		lx    = iss * fma(x, r, y * a);
		tmp   = iss * fma(m2r, lx, x);
		dx_lx = fma(tmp, dx_r, issr);
		dy_lx = fma(tmp, dy_r, issa);
		dz_lx = tmp * dz_r;

		ly    = iss * fma(y, r, -(x * a));
		tmp   = iss * fma(m2r, ly, y);
		dx_ly = fma(tmp, dx_r, -issa);
		dy_ly = fma(tmp, dy_r, issr);
		dz_ly = tmp * dz_r;

		lz    = z * ir;
		tmp   = -lz * ir;
		dx_lz = tmp * dx_r;
		dy_lz = tmp * dy_r;
		dz_lz = fma(tmp, dz_r, ir);
	}

	double flu, lu;
	double Dx0, Dx1, Dx2, Dx3, Dy0, Dy1, Dy2, Dy3, Dz0, Dz1, Dz2, Dz3;
	double hDxu, hDyu, hDzu, uD0, uD1, uD2, uD3;
	{ /* KS.cl:337-366 */
		lu  = fma(lz, uz, fma(ly, uy, fma(lx, ux, ut)));
		flu = f * lu;
		Dx0 = fma(dx_f, lu, f * fma(dx_lz, uz, fma(dx_ly, uy, dx_lx * ux)));
		Dy0 = fma(dy_f, lu, f * fma(dy_lz, uz, fma(dy_ly, uy, dy_lx * ux)));
		Dz0 = fma(dz_f, lu, f * fma(dz_lz, uz, fma(dz_ly, uy, dz_lx * ux)));

		Dx1 = fma(Dx0, lx, flu * dx_lx);
		Dx2 = fma(Dx0, ly, flu * dx_ly);
		Dx3 = fma(Dx0, lz, flu * dx_lz);

		Dy1 = fma(Dy0, lx, flu * dy_lx);
		Dy2 = fma(Dy0, ly, flu * dy_ly);
		Dy3 = fma(Dy0, lz, flu * dy_lz);

		Dz1 = fma(Dz0, lx, flu * dz_lx);
		Dz2 = fma(Dz0, ly, flu * dz_ly);
		Dz3 = fma(Dz0, lz, flu * dz_lz);

		hDxu = 0.5 * fma(Dx3, uz, fma(Dx2, uy, fma(Dx1, ux, Dx0 * ut)));
		hDyu = 0.5 * fma(Dy3, uz, fma(Dy2, uy, fma(Dy1, ux, Dy0 * ut)));
		hDzu = 0.5 * fma(Dz3, uz, fma(Dz2, uy, fma(Dz1, ux, Dz0 * ut)));

		uD0 = fma(uz, Dz0, fma(uy, Dy0, ux * Dx0));
		uD1 = fma(uz, Dz1, fma(uy, Dy1, ux * Dx1));
		uD2 = fma(uz, Dz2, fma(uy, Dy2, ux * Dx2));
		uD3 = fma(uz, Dz3, fma(uy, Dy3, ux * Dx3));

		tmp = f * fma(lz, uD3 - hDzu, fma(ly, uD2 - hDyu, fma(lx, uD1 - hDxu, -uD0)));
	}
	/* KS.cl:368-377 */
	ds[0] = ut;
	ds[1] = ux;
	ds[2] = uy;
	ds[3] = uz;
	ds[4] = uD0 - tmp;
	ds[5] = fma(lx, tmp, hDxu - uD1);
	ds[6] = fma(ly, tmp, hDyu - uD2);
	ds[7] = fma(lz, tmp, hDzu - uD3);

	if(aux) {
		aux->r = r; aux->f = f; aux->lx = lx; aux->ly = ly; aux->lz = lz;
		aux->flu = flu; aux->iss = iss;
	}
}

void
orc_ks_rhs(double a, const double s[8], double ds[8])
{
	ks_rhs_aux(a, s, ds, NULL);
}

/* ------------------------------------------------------------------------ */
/* Camera initial conditions (driver.cl:36-67, KS.cl:188-232)               */
/* ------------------------------------------------------------------------ */

void
orc_camera(const orc_desc *d, double cam[4])
{
	/* KS.cl:195-197: the angles are converted once per render on the host,
	 * so the per-pixel part is rounding-identical on CPU and GPU. */
	const double deg2rad = 3.14159265358979323846264338327950288 / 180.0;
	cam[0] = cos(deg2rad * d->i_obs);
	cam[1] = sin(deg2rad * d->i_obs);
	cam[2] = cos(deg2rad * d->j_obs);
	cam[3] = sin(deg2rad * d->j_obs);
}

/* Pixel map of driver.cl:47-51,56-57 (gi column, fastest; gj row). */
static void
pixel(const orc_desc *d, int64_t ray, double *alpha, double *beta)
{
	int64_t gi = ray % d->w_rays;
	int64_t gj = ray / d->w_rays;
	*alpha = (((double)gi + 0.5) / (double)d->w_rays - 0.5) * d->w_img;
	*beta  = (((double)gj + 0.5) / (double)d->h_rays - 0.5) * d->h_img;
}

/* Camera position and direction, KS.cl:199-205 / dyst.cl:106-109. */
static void
camera_ray(const orc_desc *d, const double cam[4], int64_t ray, double s[8])
{
	double alpha, beta;
	const double ci = cam[0], si = cam[1], cj = cam[2], sj = cam[3];
	pixel(d, ray, &alpha, &beta);
	double R0 = fma(d->r_obs, si, -(beta * ci));
	double z  = fma(d->r_obs, ci, beta * si);
	double y  = fma(R0, sj, alpha * cj);
	double x  = fma(R0, cj, -(alpha * sj));
	s[0] = 0.0; s[1] = x; s[2] = y; s[3] = z;
	s[4] = 1.0; s[5] = si * cj; s[6] = si * sj; s[7] = ci;
}

void
orc_icond(const orc_desc *d, const double cam[4], int64_t ray, double *s)
{
	camera_ray(d, cam, ray, s);

	/* KS.cl:207-229: rescale the spatial direction so that g(u,u) = 0. */
	double r, f, lx, ly, lz, iss;
	ks_fl(d->a_spin, s, &r, &f, &lx, &ly, &lz, &iss);
	const double ux = s[5], uy = s[6], uz = s[7];
	double flx = f * lx, fly = f * ly, flz = f * lz;

	double A  = f - 1.0;
	double B  = 2.0 * fma(flz, uz, fma(fly, uy, flx * ux));
	double Cx = fma(flx * lz, uz, fma(flx * ly, uy, fma(flx, lx, 1.0) * ux));
	double Cy = fma(fly * lz, uz, fma(fma(fly, ly, 1.0), uy, (fly * lx) * ux));
	double Cz = fma(fma(flz, lz, 1.0), uz, fma(flz * ly, uy, (flz * lx) * ux));
	double C  = fma(Cz, uz, fma(Cy, uy, Cx * ux));
	double den = -(B + sqrt(fma(B, B, -((4.0 * A) * C)))) / (2.0 * A);
	s[5] = ux / den;
	s[6] = uy / den;
	s[7] = uz / den;

	/* rt.cl:179-183: I = tau = 0 */
	for(int i = 0; i < 2 * d->n_freq; ++i)
		s[8 + i] = 0.0;
}

/* ------------------------------------------------------------------------ */
/* Step control (phys.cl:48-64)                                             */
/* ------------------------------------------------------------------------ */

double
orc_getdt(const orc_desc *d, const double q[4], double dt)
{
	double rp  = orc_rplus(d->a_spin);
	double eps = sqrt(orc_getrr(d->a_spin, q)) - rp;
	double stop = d->term == ORC_TERM_RPLUS ? 0.01 * rp : 0.01;

	if(eps < stop) /* stop near horizon */
		return 0.0;
	/* phys.cl:57 (dot(q.s123, q.s123) < 0) can never hold: omitted */
	if(fabs(dt) > (0.01 * eps) * eps)
		return copysign((0.01 * eps) * eps, dt);
	return dt;
}

/* ------------------------------------------------------------------------ */
/* Radiative transfer with the analytic torus (rt.cl:174-198 form)          */
/* ------------------------------------------------------------------------ */

/* Bardeen-Press-Teukolsky prograde ISCO radius (M = 1). */
double
orc_risco(double a)
{
	double z1 = 1.0 + cbrt(1.0 - a * a) * (cbrt(1.0 + a) + cbrt(1.0 - a));
	double z2 = sqrt(3.0 * a * a + z1 * z1);
	return 3.0 + z2 - sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
}

/* Torus flow + transfer.  Density n = n0 (r/r_+)^-1.5 exp(-z^2/(2 (h r)^2))
 * for r > r_isco; Keplerian Omega = 1/(r^1.5 + a) on circles about z (so
 * u^x = -Omega y u^t, u^y = Omega x u^t in Cartesian KS); emissivity
 * j = n nu^-0.7 and absorption alpha = kappa n nu^-2 at the fluid-frame
 * frequency nu = nu_i shift, shift = -k_mu u^mu.  Transfer in the form of
 * rt.cl:193-194: dI = -j e^-tau / (shift^2 + eps0), dtau = -alpha shift. */
static void
torus_rt(const orc_desc *d, const double *s, const ks_aux *x, double rp,
         double risco, const double *nupow, const double *nuinv2, double *ds)
{
	const int nf = d->n_freq;
	const double a = d->a_spin;
	double n = 0.0, shift = 1.0;

	if(x->r > risco) {
		const double q1 = s[1], q2 = s[2], q3 = s[3];
		double kt = x->flu - s[4];
		double kx = fma(x->flu, x->lx, s[5]);
		double ky = fma(x->flu, x->ly, s[6]);
		double R2 = fma(q1, q1, q2 * q2);
		double Om = 1.0 / fma(x->r, sqrt(x->r), a);
		double vv = fma(Om * Om, R2, -1.0);
		double lv = fma(-((a * Om) * R2), x->iss, 1.0);
		double D  = -fma(x->f * lv, lv, vv);
		if(D > 0.0) {
			double utf = 1.0 / sqrt(D);
			shift = -utf * fma(Om, fma(q1, ky, -(q2 * kx)), kt);
			if(shift > 0.0) {
				double qr = rp / x->r;
				double hz = d->torus_hr * x->r;
				n = ((d->torus_n0 * qr) * sqrt(qr)) *
				    exp(-((q3 * q3) / ((2.0 * hz) * hz)));
			}
		}
	}
	if(n == 0.0) {
		for(int i = 0; i < 2 * nf; ++i)
			ds[8 + i] = 0.0;
		return;
	}
	double ish  = 1.0 / shift;
	double jfac = n * pow(shift, -0.7);
	double tfac = (d->torus_kappa * n) * ish;
	double is2  = 1.0 / fma(shift, shift, ORC_EPSILON);
	for(int i = 0; i < nf; ++i) {
		double j = jfac * nupow[i];
		ds[8 + i]      = -(j * exp(-s[8 + nf + i])) * is2;
		ds[8 + nf + i] = -(tfac * nuinv2[i]);
	}
}

typedef struct {
	double rp, risco;
	double nupow[ORC_MAX_FREQ], nuinv2[ORC_MAX_FREQ];
} rt_consts;

static void
rt_setup(const orc_desc *d, rt_consts *c)
{
	c->rp    = orc_rplus(d->a_spin);
	c->risco = orc_risco(d->a_spin);
	for(int i = 0; i < d->n_freq; ++i) {
		c->nupow[i]  = pow(d->nu[i], -0.7);
		c->nuinv2[i] = 1.0 / (d->nu[i] * d->nu[i]);
	}
}

/* phys.cl:66-74 rhs(): geodesic and transfer together. */
static void
rhs_c(const orc_desc *d, const rt_consts *c, const double *s, double *ds)
{
	ks_aux aux;
	ks_rhs_aux(d->a_spin, s, ds, &aux);
	if(d->n_freq > 0) {
		if(d->flow == ORC_FLOW_TORUS)
			torus_rt(d, s, &aux, c->rp, c->risco, c->nupow, c->nuinv2, ds);
		else
			for(int i = 0; i < 2 * d->n_freq; ++i)
				ds[8 + i] = 0.0;
	}
}

void
orc_rhs(const orc_desc *d, const double *s, double *ds)
{
	rt_consts c;
	rt_setup(d, &c);
	rhs_c(d, &c, s, ds);
}

/* ------------------------------------------------------------------------ */
/* RK4 (RK4.cl:37-47) and the integer-tick substep loop (driver.cl:69-108)   */
/* ------------------------------------------------------------------------ */

#define NDMAX (8 + 2 * ORC_MAX_FREQ)

typedef void (*rhs_fn)(const void *ctx, const double *s, double *ds);

static void
rk4(rhs_fn fn, const void *ctx, int nd, double *s, double dt)
{
	double k1[NDMAX], k2[NDMAX], k3[NDMAX], k4[NDMAX], t[NDMAX] = {0.0};
	double hdt = 0.5 * dt;
	int i;
	fn(ctx, s, k1);
	for(i = 0; i < nd; ++i) t[i] = fma(hdt, k1[i], s[i]);
	fn(ctx, t, k2);
	for(i = 0; i < nd; ++i) t[i] = fma(hdt, k2[i], s[i]);
	fn(ctx, t, k3);
	for(i = 0; i < nd; ++i) t[i] = fma(dt, k3[i], s[i]);
	fn(ctx, t, k4);
	double h6 = dt / 6.0;
	for(i = 0; i < nd; ++i)
		s[i] = fma(h6, fma(2.0, k2[i] + k3[i], k1[i]) + k4[i], s[i]);
}

typedef struct {
	const orc_desc *d;
	rt_consts c;
} ks_ctx;

static void
ks_fn(const void *ctx, const double *s, double *ds)
{
	const ks_ctx *k = (const ks_ctx *)ctx;
	rhs_c(k->d, &k->c, s, ds);
}

void
orc_integrate(const orc_desc *d, double *s, double dt)
{
	ks_ctx k; memset(&k, 0, sizeof(k)); k.d = d;
	rt_setup(d, &k.c);
	rk4(ks_fn, &k, 8 + 2 * d->n_freq, s, dt);
}

/* driver.cl:81,92-99: n = (INT_MAX / n_sub) * n_sub integer ticks per dump;
 * dh = (int)(getdt(dt / n_sub) / dt * n); stop if dh == 0; clamp to the
 * remaining ticks; step size dh * dt / n. */
static int64_t
tick_loop(const orc_desc *d, const ks_ctx *k, double *s, double dt, int64_t n_sub)
{
	const int n = (int)((INT_MAX / n_sub) * n_sub);
	const double dts = dt / (double)n_sub;
	const int nd = 8 + 2 * d->n_freq;
	int64_t steps = 0;
	int h, dh;
	for(h = 0; h < n; h += dh) {
		dh = (int)(orc_getdt(d, s, dts) / dt * (double)n);
		if(!dh)
			break;
		if(dh > n - h)
			dh = n - h;
		rk4(ks_fn, k, nd, s, ((double)dh * dt) / (double)n);
		++steps;
	}
	return steps;
}

int64_t
orc_evolve_ray(const orc_desc *d, double *s, double dt, int64_t n_sub)
{
	ks_ctx k; memset(&k, 0, sizeof(k)); k.d = d;
	rt_setup(d, &k.c);
	return tick_loop(d, &k, s, dt, n_sub);
}

/* sim-org/gray.c:248-257: dumps at t_init + i dt_dump; each evolve() covers
 * target - t.  The dump interval is recomputed exactly as the host loop
 * does it. */
static int64_t
all_dumps(const orc_desc *d, const ks_ctx *k, double *s)
{
	int64_t steps = 0;
	for(int64_t i = 0; i < d->n_dump; ) {
		double t      = d->t_init + (double)i * d->dt_dump;
		double target = d->t_init + (double)(++i) * d->dt_dump;
		steps += tick_loop(d, k, s, target - t, d->n_sub);
	}
	return steps;
}

int
orc_trace(const orc_desc *d, const int64_t *rays, int64_t n, double *out,
          double *info, int64_t *steps, int nthreads)
{
	const int nd = 8 + 2 * d->n_freq;
	double cam[4];
	ks_ctx k; memset(&k, 0, sizeof(k)); k.d = d;
	if(d->n_freq < 0 || d->n_freq > ORC_MAX_FREQ || d->n_sub <= 0)
		return -1;
	rt_setup(d, &k.c);
	orc_camera(d, cam);
#ifdef _OPENMP
	if(nthreads <= 0)
		nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
	for(int64_t j = 0; j < n; ++j) {
		double *s = out + j * nd;
		orc_icond(d, cam, rays[j], s);
		steps[j] = all_dumps(d, &k, s);
		info[j]  = orc_getuu(d->a_spin, s);
	}
	(void)nthreads;
	return 0;
}

int
orc_evolve_states(const orc_desc *d, double *states, int64_t n, double *info,
                  int64_t *steps, int nthreads)
{
	const int nd = 8 + 2 * d->n_freq;
	ks_ctx k; memset(&k, 0, sizeof(k)); k.d = d;
	if(d->n_freq < 0 || d->n_freq > ORC_MAX_FREQ || d->n_sub <= 0)
		return -1;
	rt_setup(d, &k.c);
#ifdef _OPENMP
	if(nthreads <= 0)
		nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
	for(int64_t j = 0; j < n; ++j) {
		double *s = states + j * nd;
		steps[j] = all_dumps(d, &k, s);
		info[j]  = orc_getuu(d->a_spin, s);
	}
	(void)nthreads;
	return 0;
}

/* ------------------------------------------------------------------------ */
/* Numerical spacetime: fisheye map + trilinear + time (interp.cl:53-205)   */
/* ------------------------------------------------------------------------ */

#define ORC_NCOMP 51

/* Node coordinate of logical index i along one axis: interp.cl:99-121,
 * x = sinh((A i + B)^3), A and B from the box (interp.cl:116-117). */
static double
node(double lo, double hi, int n, int i)
{
	double B = cbrt(asinh(lo));
	double A = (cbrt(asinh(hi)) - B) / (double)(n - 1);
	double f = fma(A, (double)i, B);
	return sinh((f * f) * f);
}

/* interp.cl:69-97 + 123-164 for one axis: the fractional logical
 * coordinate, clamped to [0, n-1]. */
static double
axis_uvw(double x, double lo, double hi, int n)
{
	double B  = cbrt(asinh(lo));
	double A  = (cbrt(asinh(hi)) - B) / (double)(n - 1);
	double xi = floor((cbrt(asinh(x)) - B) / A);
	int i; /* clamp before converting (NaN and overflow safe) */
	if(!(xi >= 0.0))
		i = 0;
	else if(xi > (double)(n - 1))
		i = n - 1;
	else
		i = (int)xi;
	double x0 = node(lo, hi, n, i);
	double x1 = node(lo, hi, n, i + 1);
	double u  = (double)i + (x - x0) / (x1 - x0);
	if(!(u >= 0.0)) u = 0.0; /* clamp (NaN-safe) */
	if(u > (double)(n - 1)) u = (double)(n - 1);
	return u;
}

/* OpenCL CLK_FILTER_LINEAR with CLAMP_TO_EDGE on unnormalised coords
 * (u + 0.5): i0 = floor(u), frac = u - i0, i1 = min(i0 + 1, n - 1). */
static double
trilinear(const orc_grid *g, const float *F, const double uvw[3], int comp)
{
	int i0[3], i1[3];
	double w[3];
	const int n[3] = {g->nx, g->ny, g->nz};
	for(int c = 0; c < 3; ++c) {
		double fl = floor(uvw[c]);
		i0[c] = (int)fl;
		w[c]  = uvw[c] - fl;
		i1[c] = i0[c] + 1 < n[c] ? i0[c] + 1 : n[c] - 1;
	}
#define T(ix, iy, iz) ((double)F[(((size_t)(iz) * g->ny + (iy)) * g->nx + (ix)) * ORC_NCOMP + comp])
	double ax = 1.0 - w[0], ay = 1.0 - w[1], az = 1.0 - w[2];
	double w000 = (ax * ay) * az, w100 = (w[0] * ay) * az;
	double w010 = (ax * w[1]) * az, w110 = (w[0] * w[1]) * az;
	double w001 = (ax * ay) * w[2], w101 = (w[0] * ay) * w[2];
	double w011 = (ax * w[1]) * w[2], w111 = (w[0] * w[1]) * w[2];
	double v = w000 * T(i0[0], i0[1], i0[2]);
	v = fma(w100, T(i1[0], i0[1], i0[2]), v);
	v = fma(w010, T(i0[0], i1[1], i0[2]), v);
	v = fma(w110, T(i1[0], i1[1], i0[2]), v);
	v = fma(w001, T(i0[0], i0[1], i1[2]), v);
	v = fma(w101, T(i1[0], i0[1], i1[2]), v);
	v = fma(w011, T(i0[0], i1[1], i1[2]), v);
	v = fma(w111, T(i1[0], i1[1], i1[2]), v);
#undef T
	return v;
}

static int
inside_box(const orc_grid *g, const double q[4])
{
	for(int c = 1; c <= 3; ++c)
		if(!(q[c] >= (double)g->box[c] && q[c] <= (double)g->box[c + 4]))
			return 0;
	return 1;
}

/* interp.cl:183-205: single level when t1 == t2, else linear in time
 * (unclamped in reference semantics; clamped to [0,1] in physics mode). */
static void
interp_all(const orc_grid *g, const double q[4], double out[ORC_NCOMP])
{
	double uvw[3];
	for(int c = 0; c < 3; ++c)
		uvw[c] = axis_uvw(q[c + 1], g->box[c + 1], g->box[c + 5],
		                  c == 0 ? g->nx : c == 1 ? g->ny : g->nz);
	double t1 = g->box[0], t2 = g->box[4];
	if(t1 == t2) {
		for(int m = 0; m < ORC_NCOMP; ++m)
			out[m] = trilinear(g, g->fields[0], uvw, m);
		return;
	}
	double ft = (q[0] - t1) / (t2 - t1);
	if(g->physics) {
		if(!(ft >= 0.0)) ft = 0.0;
		if(ft > 1.0) ft = 1.0;
	}
	for(int m = 0; m < ORC_NCOMP; ++m) {
		double y1 = trilinear(g, g->fields[0], uvw, m);
		double y2 = trilinear(g, g->fields[1], uvw, m);
		out[m] = fma(ft, y2 - y1, y1);
	}
}

double
orc_interp(const orc_grid *g, const double q[4], int comp)
{
	double v[ORC_NCOMP];
	interp_all(g, q, v);
	return v[comp];
}

/* Fill the 4x4 symmetric matrix from the 10 stored components in the order
 * tt,tx,ty,tz,xx,xy,xz,yy,yz,zz (dyst.cl:138-139 symmetrisation). */
static void
sym10(const double *c, double M[4][4])
{
	int k = 0;
	for(int i = 0; i < 4; ++i)
		for(int j = i; j < 4; ++j) {
			M[i][j] = c[k];
			M[j][i] = c[k];
			++k;
		}
}

/* Quadratic form sum_ab M_ab u^a u^b over the 10 stored components, with
 * off-diagonal products doubled. */
static double
quad10(const double *c, const double p[10])
{
	double v = c[0] * p[0];
	for(int k = 1; k < 10; ++k)
		v = fma(c[k], p[k], v);
	return v;
}

static void
pairs10(const double u[4], double p[10])
{
	int k = 0;
	for(int i = 0; i < 4; ++i)
		for(int j = i; j < 4; ++j) {
			double uu = u[i] * u[j];
			p[k++] = i == j ? uu : 2.0 * uu;
		}
}

/* ------------------------------------------------------------------------ */
/* Thermal emissivities (rt.cl:28-170) and the template flow (flow.cl)       */
/* ------------------------------------------------------------------------ */

/* CGS constants of rt.cl:28-36 */
#define C_c    2.99792458e+10
#define C_h    6.62606957e-27
#define C_G    6.67384800e-08
#define C_kB   1.38064881e-16
#define C_Ry   2.17987197e-11
#define C_e    4.80320425e-10
#define C_me   9.10938291e-28
#define C_mSun 1.98910000e+33
#define O_PI   3.14159265358979323846
#define O_SQRT2 1.41421356237309504880
#define T_MIN  1e-1
#define T_MAX  1e+2
#define T_GRID 60

#include "../gray_b200/csrc/logk2_table.h"
static const double LOGK2[GRAY_LOGK2_N] = {GRAY_LOGK2_VALUES};

/* Constants that need libm, evaluated at run time from volatile inputs
 * (no compile-time folding), exactly as the library's host code does. */
typedef struct {
	double g1, g2, g3, g4, g5, ff_f, lk_scale;
} th_consts;

static void
th_setup(th_consts *t)
{
	volatile double three = 3.0, four = 4.0, twelve = 12.0, pi = O_PI, e_gaunt = 1.78107241799;
	volatile double ff_in = C_G * C_mSun / (C_c * C_c) * 6.8e-38, mec2_kb = C_me * C_c * C_c / C_kB;
	volatile double tmax_tmin = T_MAX / T_MIN;
	t->g1 = sqrt(three / pi);
	t->g2 = sqrt(three) / pi;
	t->g3 = log(four / e_gaunt);
	t->g4 = log(four / pow(e_gaunt, 2.5));
	t->g5 = sqrt(twelve);
	t->ff_f = sqrt(ff_in / (4 * pi * sqrt(mec2_kb)));
	t->lk_scale = (double)T_GRID / log(tmax_tmin);
}

static th_consts TH;

/* set up once when the library loads, before any OpenMP region reads it */
__attribute__((constructor)) static void
th_init(void)
{
	th_setup(&TH);
}

static const th_consts *
th(void)
{
	return &TH;
}

/* rt.cl:70-78; the index is kept inside the table (te == T_MAX exactly
 * would read one entry past its end in the reference) */
double
orc_log_K2it(double te)
{
	const double h = log(te / T_MIN) * th()->lk_scale;
	int i = (int)h;
	if(i > T_GRID - 1)
		i = T_GRID - 1;
	const double d = h - i;
	return (1 - d) * LOGK2[i] + d * LOGK2[i + 1];
}

/* rt.cl:80-93 */
double
orc_B_Planck(double nu, double te)
{
	double f1 = 2 * C_h * C_c;
	double f2 = C_h / (C_me * C_c);
	nu /= C_c;
	f1 *= nu * nu;
	f2 *= nu / (te + ORC_EPSILON);
	return nu * (f2 > 1e-5 ? f1 / (exp(f2) - 1) : (f1 / f2) / (1 + f2 / 2 + f2 * f2 / 6));
}

/* rt.cl:95-120 */
double
orc_Gaunt(double x, double y)
{
	const th_consts *t = th();
	const double sx = sqrt(x);
	const double sy = sqrt(y);
	if(x > 1)
		return y > 1 ? t->g1 / sy : t->g2 * (t->g3 - log(y + ORC_EPSILON));
	else if(x * y > 1)
		return t->g5 / (sx * sy);
	else if(y > sx)
		return 1;
	else {
		const double g = t->g2 * (t->g4 + log(sx / (y + ORC_EPSILON)));
		return g > ORC_EPSILON ? g : ORC_EPSILON;
	}
}

/* rt.cl:122-143 (M_ADM passed in) */
double
orc_L_j_ff(double m_adm, double nu, double te, double ne)
{
	double x = C_me * C_c * C_c / C_Ry;
	double y = C_h / (C_me * C_c * C_c);
	double f = th()->ff_f;
	x *= te;
	y *= nu / te;
	f *= ne;
	return (m_adm * f * orc_Gaunt(x, y)) * (f / (sqrt(te) * exp(y) + ORC_EPSILON));
}

/* rt.cl:145-170 */
double
orc_L_j_syn(double m_adm, double nu, double te, double ne, double b, double cos_theta)
{
	if(te <= T_MIN || cos_theta <= -1 || cos_theta >= 1)
		return 0;
	const double nus = te * te * b * sqrt(1 - cos_theta * cos_theta) *
	                   (C_e / (9 * O_PI * C_me * C_c));
	const double x = nu / (nus + ORC_EPSILON);
	const double f = (C_G * C_mSun / (C_c * C_c)) * (O_SQRT2 * O_PI * C_e * C_e / (3 * C_c));
	const double cbrtx = cbrt(x);
	const double xx = sqrt(x) + 1.88774862536 * sqrt(cbrtx);
	const double log_K2 = (te > T_MAX) ? log(2 * te * te - 0.5) : orc_log_K2it(te);
	return (m_adm * xx * exp(-cbrtx)) * (xx * exp(-log_K2)) * (f * ne * nus);
}

/* rt.cl:185-198 with the template flow of flow.cl:36-58 generalised to a
 * field of magnitude b along z: shift = -k.u with u = (1,0,0,0),
 * cos = k.b / (shift |b|). */
static void
thermal_rt(const orc_desc *d, const double k[4], double ne, const double *s, double *ds)
{
	const int nf = d->n_freq;
	const double te = d->flow_te, b = d->flow_b;
	const double shift = -k[0];
	const double bkcos = (k[3] * b) / (shift * b + ORC_EPSILON);
	for(int i = 0; i < nf; ++i) {
		const double nu = d->nu[i] * shift;
		const double B_nu = orc_B_Planck(nu, te);
		const double L = orc_L_j_syn(d->m_adm, nu, te, ne, b, bkcos) +
		                 orc_L_j_ff(d->m_adm, nu, te, ne);
		ds[8 + i]      = -L * exp(-s[8 + nf + i]) / (shift * shift + ORC_EPSILON);
		ds[8 + nf + i] = -L * shift / (B_nu + ORC_EPSILON);
	}
}

/* dyst.cl:112-194: a^mu = -Gamma^mu_ab u^a u^b + (Gamma^t_ab u^a u^b) u^mu */
void
orc_dyst_rhs(const orc_grid *g, const double s[8], double ds[8])
{
	const double *u = s + 4;
	ds[0] = u[0]; ds[1] = u[1]; ds[2] = u[2]; ds[3] = u[3];
	if(g->physics && !inside_box(g, s)) {
		ds[4] = ds[5] = ds[6] = ds[7] = 0.0;
		return;
	}
	double v[ORC_NCOMP], p[10], G[4];
	interp_all(g, s, v);
	pairs10(u, p);
	for(int m = 0; m < 4; ++m)
		G[m] = quad10(v + 10 * m, p);
	for(int m = 0; m < 4; ++m)
		ds[4 + m] = fma(G[0], u[m], -G[m]);
}

/* dyst.cl:55-81 down(); bug_gzz reproduces dyst.cl:78 where g_zz is
 * read from the g_yz image. */
void
orc_dyst_down(const orc_grid *g, const double q[4], const double u[4], double k[4])
{
	double v[ORC_NCOMP], M[4][4], c[10];
	if(g->physics && !inside_box(g, q)) {
		k[0] = -u[0]; k[1] = u[1]; k[2] = u[2]; k[3] = u[3];
		return;
	}
	interp_all(g, q, v);
	for(int i = 0; i < 10; ++i)
		c[i] = v[40 + i];
	if(g->bug_gzz)
		c[9] = c[8];
	sym10(c, M);
	for(int i = 0; i < 4; ++i)
		k[i] = dot4(M[i], u);
}

/* dyst.cl:89-110: camera ray without null normalisation. */
void
orc_dyst_icond(const orc_desc *d, const double cam[4], int64_t ray, double s[8])
{
	camera_ray(d, cam, ray, s);
}

/* phys.cl:48-64 with dyst.cl:43-53 (getrr = geteps = 1). */
double
orc_dyst_getdt(double dt)
{
	const double eps = 1.0;
	if(fabs(dt) > (0.01 * eps) * eps)
		return copysign((0.01 * eps) * eps, dt);
	return dt;
}

/* phys.cl:66-74 on the numerical spacetime: the geodesic, and for the
 * thermal flow the transfer with k = down(q, u) (dyst.cl:55-81) and n_e the
 * interpolated rho (flow.cl:48).  One interpolation serves all fields
 * (the reference interpolates them field by field: same values).  In
 * physics mode outside the box the spacetime is flat and n_e = 0. */
void
orc_dyst_rhs_rt(const orc_desc *d, const orc_grid *g, const double *s, double *ds)
{
	const double *u = s + 4;
	const int nf = d->n_freq;
	if(nf == 0 || d->flow != ORC_FLOW_THERMAL) {
		orc_dyst_rhs(g, s, ds);
		for(int i = 0; i < 2 * nf; ++i)
			ds[8 + i] = 0.0;
		return;
	}
	double v[ORC_NCOMP], k[4], ne;
	ds[0] = u[0]; ds[1] = u[1]; ds[2] = u[2]; ds[3] = u[3];
	if(g->physics && !inside_box(g, s)) {
		ds[4] = ds[5] = ds[6] = ds[7] = 0.0;
		k[0] = -u[0]; k[1] = u[1]; k[2] = u[2]; k[3] = u[3];
		ne = 0.0;
	} else {
		double p[10], G[4], c[10], M[4][4];
		interp_all(g, s, v);
		pairs10(u, p);
		for(int m = 0; m < 4; ++m)
			G[m] = quad10(v + 10 * m, p);
		for(int m = 0; m < 4; ++m)
			ds[4 + m] = fma(G[0], u[m], -G[m]);
		for(int i = 0; i < 10; ++i)
			c[i] = v[40 + i];
		if(g->bug_gzz)
			c[9] = c[8];
		sym10(c, M);
		for(int i = 0; i < 4; ++i)
			k[i] = dot4(M[i], u);
		ne = v[50];
	}
	thermal_rt(d, k, ne, s, ds);
}

typedef struct {
	const orc_desc *d;
	const orc_grid *g;
} dyst_ctx;

static void
dyst_fn(const void *ctx, const double *s, double *ds)
{
	const dyst_ctx *c = (const dyst_ctx *)ctx;
	orc_dyst_rhs_rt(c->d, c->g, s, ds);
}

int64_t
orc_dyst_evolve_ray(const orc_desc *d, const orc_grid *g, double *s, double dt,
                    int64_t n_sub)
{
	const int n = (int)((INT_MAX / n_sub) * n_sub);
	const double dts = dt / (double)n_sub;
	dyst_ctx c = {d, g};
	int64_t steps = 0;
	int h, dh;
	for(h = 0; h < n; h += dh) {
		dh = (int)(orc_dyst_getdt(dts) / dt * (double)n);
		if(!dh)
			break;
		if(dh > n - h)
			dh = n - h;
		rk4(dyst_fn, &c, 8 + 2 * d->n_freq, s, ((double)dh * dt) / (double)n);
		++steps;
	}
	return steps;
}

int
orc_dyst_trace(const orc_desc *d, const orc_grid *g, const int64_t *rays,
               int64_t n, double *out, double *info, int64_t *steps, int nthreads)
{
	double cam[4];
	const int nd = 8 + 2 * d->n_freq;
	if(d->n_freq < 0 || d->n_freq > ORC_MAX_FREQ || d->n_sub <= 0)
		return -1;
	orc_camera(d, cam);
#ifdef _OPENMP
	if(nthreads <= 0)
		nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
	for(int64_t j = 0; j < n; ++j) {
		double *s = out + j * nd;
		int64_t st = 0;
		orc_dyst_icond(d, cam, rays[j], s);
		for(int i = 0; i < 2 * d->n_freq; ++i)
			s[8 + i] = 0.0; /* rt.cl:179-183 */
		for(int64_t i = 0; i < d->n_dump; ) {
			double t      = d->t_init + (double)i * d->dt_dump;
			double target = d->t_init + (double)(++i) * d->dt_dump;
			st += orc_dyst_evolve_ray(d, g, s, target - t, d->n_sub);
		}
		steps[j] = st;
		double k[4];
		orc_dyst_down(g, s, s + 4, k);
		info[j] = dot4(k, s + 4);
	}
	(void)nthreads;
	return 0;
}

/* ------------------------------------------------------------------------ */
/* Boosted Kerr-Schild sampler (tools/boosted_ks.py)                        */
/* ------------------------------------------------------------------------ */

/* Forward-mode dual numbers, as tools/boosted_ks.py:40-115 uses them. */
typedef struct { double f, s; } dual;
static inline dual dd_(double f, double s) { dual r = {f, s}; return r; }
static inline dual dadd(dual a, dual b) { return dd_(a.f + b.f, a.s + b.s); }
static inline dual dsub(dual a, dual b) { return dd_(a.f - b.f, a.s - b.s); }
static inline dual dmul(dual a, dual b) { return dd_(a.f * b.f, a.s * b.f + a.f * b.s); }
static inline dual dscale(dual a, double c) { return dd_(a.f * c, a.s * c); }
static inline dual ddiv(dual a, dual b)
{
	return dd_(a.f / b.f, (a.s * b.f - a.f * b.s) / (b.f * b.f));
}
static inline dual dsqrt(dual a)
{
	double r = sqrt(a.f);
	return dd_(r, a.s * 0.5 / r);
}

/* boosted_ks.py:120-186 metric(): Kerr-Schild with mass m and spin a,
 * boosted with speed v along `axis` (1=x, 2=y, 3=z; the reference tool
 * hard-wires z).  Returns h = m r/(r^2 + a^2 cos^2) and covariant l_mu. */
static void
bks_hl(double m, double a, double v, int axis, const dual X[4], dual *h, dual l[4])
{
	double gam = 1.0 / sqrt(1.0 - v * v);
	dual x0[4];
	for(int c = 0; c < 4; ++c)
		x0[c] = X[c];
	/* Lorentz boost mixing t and the boost axis */
	x0[0]    = dscale(dsub(X[0], dscale(X[axis], v)), gam);
	x0[axis] = dscale(dsub(X[axis], dscale(X[0], v)), gam);

	/* the spin axis stays along z of the rest frame */
	dual xx = x0[1], yy = x0[2], zz = x0[3];
	dual rho2 = dadd(dadd(dmul(xx, xx), dmul(yy, yy)), dmul(zz, zz));
	dual w = dsub(rho2, dd_(a * a, 0.0));
	dual r2 = dadd(dscale(w, 0.5),
	               dsqrt(dadd(dscale(dmul(w, w), 0.25), dscale(dmul(zz, zz), a * a))));
	dual r = dsqrt(r2);
	dual ct = ddiv(zz, r);
	*h = ddiv(dscale(r, m), dadd(r2, dscale(dmul(ct, ct), a * a)));

	dual ra2 = dadd(r2, dd_(a * a, 0.0));
	dual l0[4];
	l0[0] = dd_(1.0, 0.0);
	l0[1] = ddiv(dadd(dmul(r, xx), dscale(yy, a)), ra2);
	l0[2] = ddiv(dsub(dmul(r, yy), dscale(xx, a)), ra2);
	l0[3] = ddiv(zz, r);
	for(int c = 0; c < 4; ++c)
		l[c] = l0[c];
	/* covector boost, boosted_ks.py:147-148 */
	l[0]    = dscale(dsub(l0[0], dscale(l0[axis], v)), gam);
	l[axis] = dscale(dsub(l0[axis], dscale(l0[0], v)), gam);
}

static const double ETA[4] = {-1.0, 1.0, 1.0, 1.0};

/* Christoffel symbols from the dual-number metric derivatives,
 * boosted_ks.py:233-275: Gamma^i_kl = 1/2 g^im (d_l g_mk + d_k g_ml - d_m g_kl). */
void
orc_boosted_ks(double m, double a, double v, int axis, const double q[4], double out[50])
{
	double dg[4][4][4]; /* dg[w][i][j] = d_w g_ij */
	double gd[4][4], gu[4][4];
	for(int w = 0; w < 4; ++w) {
		dual X[4], h, l[4];
		for(int c = 0; c < 4; ++c)
			X[c] = dd_(q[c], c == w ? 1.0 : 0.0);
		bks_hl(m, a, v, axis, X, &h, l);
		for(int i = 0; i < 4; ++i)
			for(int j = 0; j < 4; ++j) {
				dual gij = dscale(dmul(h, dmul(l[i], l[j])), 2.0);
				dg[w][i][j] = gij.s;
				if(w == 0) {
					gd[i][j] = (i == j ? ETA[i] : 0.0) + gij.f;
					/* inverse: eta - 2 h l^i l^j with l^t = -l_t */
					double li = i == 0 ? -l[0].f : l[i].f;
					double lj = j == 0 ? -l[0].f : l[j].f;
					gu[i][j] = (i == j ? ETA[i] : 0.0) - 2.0 * h.f * li * lj;
				}
			}
	}
	int k = 0;
	for(int i = 0; i < 4; ++i)
		for(int b = 0; b < 4; ++b)
			for(int c = b; c < 4; ++c) {
				double t = 0.0;
				for(int mm = 0; mm < 4; ++mm)
					t += gu[i][mm] * (dg[c][mm][b] + dg[b][mm][c] - dg[mm][b][c]);
				out[k++] = 0.5 * t;
			}
	for(int i = 0; i < 4; ++i)
		for(int j = i; j < 4; ++j)
			out[k++] = gd[i][j];
}

/* ------------------------------------------------------------------------ */
/* Snapshot series ("slow light", sim-org/gray.c:147-294)                    */
/* ------------------------------------------------------------------------ */

/* sim-org/gray.c:41-57 */
static int64_t
series_find(const double *times, int64_t n, double t)
{
	for(int64_t k = 0; k + 1 < n; ++k)
		if(t >= times[k] && t <= times[k + 1])
			return k;
	return -1;
}

int
orc_series_schedule(const double *times, int64_t n, double t_init, double dt_dump,
                    int64_t n_dump, int fast_light, int64_t *first, int64_t *pairs)
{
	int64_t snap;
	int frozen = n == 1 || fast_light;
	if(n < 1)
		return -1;
	for(int64_t k = 1; k < n; ++k)
		if(!(times[k] > times[k - 1]))
			return -1;
	if(n == 1)
		snap = 0;                             /* gray.c:188-191 */
	else if(fast_light)
		snap = series_find(times, n, t_init); /* gray.c:214 */
	else {
		double t_final = t_init + (0 + 1) * dt_dump * n_dump; /* gray.c:200 */
		if(t_init < times[0] || t_init > times[n - 1] ||
		   t_final < times[0] || t_final > times[n - 1])
			return -1;
		snap = series_find(times, n, t_init); /* gray.c:232 */
	}
	if(snap < 0)
		return -1;
	*first = snap;
	for(int64_t i = 0; i < n_dump; ) {
		double target;
		pairs[i] = snap;
		target = t_init + (double)(++i) * dt_dump;
		if(!frozen && (target < times[snap] || target > times[snap + 1])) {
			snap = series_find(times, n, target); /* gray.c:267-270 */
			if(snap < 0)
				return -1;
		}
	}
	return 0;
}

static void
series_grid(const orc_grid *tmpl, const float *const *snaps, const double *times,
            int64_t k, int frozen, orc_grid *g)
{
	*g = *tmpl;
	g->fields[0] = snaps[k];
	g->fields[1] = frozen ? snaps[k] : snaps[k + 1];
	g->box[0] = frozen ? 0.0f : (float)times[k];     /* gray.c:225-226, 237-238 */
	g->box[4] = frozen ? 0.0f : (float)times[k + 1];
}

int
orc_dyst_series_trace(const orc_desc *d, const orc_grid *tmpl, const float *const *snaps,
                      const double *times, int64_t n_times, int fast_light,
                      const int64_t *rays, int64_t n, double *out, double *info,
                      int64_t *steps, int nthreads)
{
	double cam[4];
	const int nd = 8 + 2 * d->n_freq;
	const int frozen = n_times == 1 || fast_light;
	int64_t first, *pairs;
	if(d->n_freq < 0 || d->n_freq > ORC_MAX_FREQ || d->n_sub <= 0)
		return -1;
	pairs = (int64_t *)malloc(sizeof(int64_t) * (d->n_dump ? d->n_dump : 1));
	if(!pairs)
		return -1;
	if(orc_series_schedule(times, n_times, d->t_init, d->dt_dump, d->n_dump, fast_light,
	                       &first, pairs)) {
		free(pairs);
		return -1;
	}
	orc_camera(d, cam);
#ifdef _OPENMP
	if(nthreads <= 0)
		nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
	for(int64_t j = 0; j < n; ++j) {
		double *s = out + j * nd;
		int64_t st = 0, k = first;
		orc_grid g;
		orc_dyst_icond(d, cam, rays[j], s);
		for(int i = 0; i < 2 * d->n_freq; ++i)
			s[8 + i] = 0.0;
		for(int64_t i = 0; i < d->n_dump; ) {
			k = pairs[i];
			series_grid(tmpl, snaps, times, k, frozen, &g);
			double t      = d->t_init + (double)i * d->dt_dump;
			double target = d->t_init + (double)(++i) * d->dt_dump;
			st += orc_dyst_evolve_ray(d, &g, s, target - t, d->n_sub);
		}
		series_grid(tmpl, snaps, times, k, frozen, &g);
		steps[j] = st;
		double kd[4];
		orc_dyst_down(&g, s, s + 4, kd);
		info[j] = dot4(kd, s + 4);
	}
	(void)nthreads;
	free(pairs);
	return 0;
}
