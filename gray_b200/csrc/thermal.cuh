/*
 * Thermal radiative transfer in FP64 (rt.cl:28-198) with the template flow
 * of flow.cl:36-58: electrons at rest in the grid frame, u = (1, 0, 0, 0),
 * number density n_e from the grid's rho field, temperature te and a
 * magnetic field of strength b along z (the reference's template has
 * b = 0, the default here).
 *
 * Shared by the FP64 kernels (kernels_dyst64.cu, -fmad=false) and the
 * mixed kernel's FP64 transfer island (kernels_dyst.cu).  The emissivities
 * span tens of decades in CGS units (j_ff ~ 1e-36 for n_e ~ 1), below the
 * FP32 normal range, so the transfer is FP64 in both.
 */
#ifndef GRAY_THERMAL_CUH
#define GRAY_THERMAL_CUH

#include "gray_internal.h"
#include "logk2_table.h"

namespace thermal {

/* CGS constants of rt.cl:28-36 */
constexpr double C_c    = 2.99792458e+10;
constexpr double C_h    = 6.62606957e-27;
constexpr double C_G    = 6.67384800e-08;
constexpr double C_Ry   = 2.17987197e-11;
constexpr double C_e    = 4.80320425e-10;
constexpr double C_me   = 9.10938291e-28;
constexpr double C_mSun = 1.98910000e+33;
constexpr double PI     = 3.14159265358979323846;
constexpr double SQRT2  = 1.41421356237309504880;
constexpr double T_MIN  = 1e-1;
constexpr double T_MAX  = 1e+2;
constexpr int    T_GRID = 60;
constexpr double EPS    = GRAY_EPSILON;

/* log K_2(1/te) on the logarithmic grid of rt.cl:38-68 */
static __constant__ double c_logk2[GRAY_LOGK2_N] = {GRAY_LOGK2_VALUES};

/* rt.cl:70-78 (callers guarantee T_MIN < te <= T_MAX; the last cell is
 * reused at te == T_MAX so that the table is never read past its end) */
__device__ __forceinline__ double
log_K2it(const ThermalConsts &t, double te)
{
	const double h = log(te / T_MIN) * t.lk_scale;
	int i = (int)h;
	if(i > T_GRID - 1)
		i = T_GRID - 1;
	const double d = h - i;
	return (1 - d) * c_logk2[i] + d * c_logk2[i + 1];
}

/* rt.cl:80-93 */
__device__ __forceinline__ double
B_Planck(double nu, double te)
{
	double f1 = 2 * C_h * C_c;
	double f2 = C_h / (C_me * C_c);
	nu /= C_c;
	f1 *= nu * nu;
	f2 *= nu / (te + EPS);
	return nu * (f2 > 1e-5 ? f1 / (exp(f2) - 1) : (f1 / f2) / (1 + f2 / 2 + f2 * f2 / 6));
}

/* rt.cl:95-120 */
__device__ __forceinline__ double
Gaunt(const ThermalConsts &t, double x, double y)
{
	const double sx = sqrt(x);
	const double sy = sqrt(y);
	if(x > 1)
		return y > 1 ? t.g1 / sy : t.g2 * (t.g3 - log(y + EPS));
	else if(x * y > 1)
		return t.g5 / (sx * sy);
	else if(y > sx)
		return 1;
	const double g = t.g2 * (t.g4 + log(sx / (y + EPS)));
	return g > EPS ? g : EPS;
}

/* rt.cl:122-143 */
__device__ __forceinline__ double
L_j_ff(const ThermalConsts &t, double m_adm, double nu, double te, double ne)
{
	double x = C_me * C_c * C_c / C_Ry;
	double y = C_h / (C_me * C_c * C_c);
	double f = t.ff_f;
	x *= te;
	y *= nu / te;
	f *= ne;
	return (m_adm * f * Gaunt(t, x, y)) * (f / (sqrt(te) * exp(y) + EPS));
}

/* rt.cl:145-170 */
__device__ __forceinline__ double
L_j_syn(const ThermalConsts &t, double m_adm, double nu, double te, double ne, double b,
        double cos_theta)
{
	if(te <= T_MIN || cos_theta <= -1 || cos_theta >= 1)
		return 0;
	const double nus = te * te * b * sqrt(1 - cos_theta * cos_theta) *
	                   (C_e / (9 * PI * C_me * C_c));
	const double x = nu / (nus + EPS);
	const double f = (C_G * C_mSun / (C_c * C_c)) * (SQRT2 * PI * C_e * C_e / (3 * C_c));
	const double cbrtx = cbrt(x);
	const double xx = sqrt(x) + 1.88774862536 * sqrt(cbrtx);
	const double log_K2 = (te > T_MAX) ? log(2 * te * te - 0.5) : log_K2it(t, te);
	return (m_adm * xx * exp(-cbrtx)) * (xx * exp(-log_K2)) * (f * ne * nus);
}

/* Per-render inputs of the transfer. */
struct Flow {
	const double *nu;   /* observed frequencies [NF] (Hz)      */
	double m_adm, te, b;
	const ThermalConsts *th;
};

/* rt.cl:185-198 with getflow() of flow.cl:36-58: k is the covariant
 * photon momentum, tau[NF] the optical depths of the state; writes
 * dI[NF], dtau[NF]. */
template <int NF>
__device__ __forceinline__ void
rt_rhs(const Flow &f, const double k[4], double ne, const double *tau, double *dI,
       double *dtau)
{
	const double shift = -k[0];
	const double bkcos = (k[3] * f.b) / (shift * f.b + EPS);
#pragma unroll
	for(int i = 0; i < NF; ++i) {
		const double nu = f.nu[i] * shift;
		const double B_nu = B_Planck(nu, f.te);
		const double L = L_j_syn(*f.th, f.m_adm, nu, f.te, ne, f.b, bkcos) +
		                 L_j_ff(*f.th, f.m_adm, nu, f.te, ne);
		dI[i]   = -L * exp(-tau[i]) / (shift * shift + EPS);
		dtau[i] = -L * shift / (B_nu + EPS);
	}
}

} /* namespace thermal */

#endif /* GRAY_THERMAL_CUH */
