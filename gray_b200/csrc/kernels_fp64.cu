/*
 * Plain FP64 kernels: one ray per thread, SoA state, one launch per dump
 * interval -- the structure of the reference's evolve_drv (driver.cl:69-108)
 * on B200.  This is the FP64 baseline the mixed-precision path is measured
 * against, and the kernel that must agree with the CPU oracle to 1e-10.
 *
 * Rounding contract: this translation unit is compiled with -fmad=false,
 * so the only fused multiply-adds are the explicit fma() calls below; they
 * sit exactly where the oracle (oracle/gray_oracle.c) places its fma()
 * calls.  FP64 '/' and sqrt() are IEEE round-to-nearest on sm_100, as in
 * the oracle, so the geodesic agrees bit for bit.
 */
#include <climits>

#include "gray_internal.h"

namespace {

/* KS.cl:48-55 getrr() */
__device__ __forceinline__ double
getrr64(const RenderParams &p, double x, double y, double z)
{
	double zz = z * z;
	double kk = 0.5 * (fma(x, x, fma(y, y, zz)) - p.aa);
	return sqrt(fma(kk, kk, p.aa * zz)) + kk;
}

struct Aux64 {
	double r, f, lx, ly, lz, flu, iss;
};

/* KS.cl:263-378 gr_rhs(), Chan et al. form; returns f, l and f l.u for the
 * transfer step (phys.cl:70 down() reuses them). */
__device__ __forceinline__ void
ks_rhs64(const RenderParams &p, const double *s, double *ds, Aux64 &aux)
{
	const double a = p.a;
	const double x = s[1], y = s[2], z = s[3];
	const double ut = s[4], ux = s[5], uy = s[6], uz = s[7];

	double f, dx_f, dy_f, dz_f;
	double lx, dx_lx, dy_lx, dz_lx;
	double ly, dx_ly, dy_ly, dz_ly;
	double lz, dx_lz, dy_lz, dz_lz;
	double dx_r, dy_r, dz_r, r, ir, iss, tmp;
	{
		double aa = p.aa;
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
	{
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
	double lu  = fma(lz, uz, fma(ly, uy, fma(lx, ux, ut)));
	double flu = f * lu;
	double Dx0 = fma(dx_f, lu, f * fma(dx_lz, uz, fma(dx_ly, uy, dx_lx * ux)));
	double Dy0 = fma(dy_f, lu, f * fma(dy_lz, uz, fma(dy_ly, uy, dy_lx * ux)));
	double Dz0 = fma(dz_f, lu, f * fma(dz_lz, uz, fma(dz_ly, uy, dz_lx * ux)));

	double Dx1 = fma(Dx0, lx, flu * dx_lx);
	double Dx2 = fma(Dx0, ly, flu * dx_ly);
	double Dx3 = fma(Dx0, lz, flu * dx_lz);

	double Dy1 = fma(Dy0, lx, flu * dy_lx);
	double Dy2 = fma(Dy0, ly, flu * dy_ly);
	double Dy3 = fma(Dy0, lz, flu * dy_lz);

	double Dz1 = fma(Dz0, lx, flu * dz_lx);
	double Dz2 = fma(Dz0, ly, flu * dz_ly);
	double Dz3 = fma(Dz0, lz, flu * dz_lz);

	double hDxu = 0.5 * fma(Dx3, uz, fma(Dx2, uy, fma(Dx1, ux, Dx0 * ut)));
	double hDyu = 0.5 * fma(Dy3, uz, fma(Dy2, uy, fma(Dy1, ux, Dy0 * ut)));
	double hDzu = 0.5 * fma(Dz3, uz, fma(Dz2, uy, fma(Dz1, ux, Dz0 * ut)));

	double uD0 = fma(uz, Dz0, fma(uy, Dy0, ux * Dx0));
	double uD1 = fma(uz, Dz1, fma(uy, Dy1, ux * Dx1));
	double uD2 = fma(uz, Dz2, fma(uy, Dy2, ux * Dx2));
	double uD3 = fma(uz, Dz3, fma(uy, Dy3, ux * Dx3));

	tmp = f * fma(lz, uD3 - hDzu, fma(ly, uD2 - hDyu, fma(lx, uD1 - hDxu, -uD0)));

	ds[0] = ut;
	ds[1] = ux;
	ds[2] = uy;
	ds[3] = uz;
	ds[4] = uD0 - tmp;
	ds[5] = fma(lx, tmp, hDxu - uD1);
	ds[6] = fma(ly, tmp, hDyu - uD2);
	ds[7] = fma(lz, tmp, hDzu - uD3);

	aux.r = r; aux.f = f; aux.lx = lx; aux.ly = ly; aux.lz = lz;
	aux.flu = flu; aux.iss = iss;
}

/* Torus flow + transfer in the rt.cl:185-198 form (see the oracle's
 * torus_rt() for the model). */
template <int NF>
__device__ __forceinline__ void
torus_rt64(const RenderParams &p, const double *s, const Aux64 &x, double *ds)
{
	double n = 0.0, shift = 1.0;
	if(x.r > p.risco) {
		const double q1 = s[1], q2 = s[2], q3 = s[3];
		double kt = x.flu - s[4];
		double kx = fma(x.flu, x.lx, s[5]);
		double ky = fma(x.flu, x.ly, s[6]);
		double R2 = fma(q1, q1, q2 * q2);
		double Om = 1.0 / fma(x.r, sqrt(x.r), p.a);
		double vv = fma(Om * Om, R2, -1.0);
		double lv = fma(-((p.a * Om) * R2), x.iss, 1.0);
		double D  = -fma(x.f * lv, lv, vv);
		if(D > 0.0) {
			double utf = 1.0 / sqrt(D);
			shift = -utf * fma(Om, fma(q1, ky, -(q2 * kx)), kt);
			if(shift > 0.0) {
				double qr = p.rp / x.r;
				double hz = p.torus_hr * x.r;
				n = ((p.torus_n0 * qr) * sqrt(qr)) *
				    exp(-((q3 * q3) / ((2.0 * hz) * hz)));
			}
		}
	}
	if(n == 0.0) {
#pragma unroll
		for(int i = 0; i < 2 * NF; ++i)
			ds[8 + i] = 0.0;
		return;
	}
	double ish  = 1.0 / shift;
	double jfac = n * pow(shift, -0.7);
	double tfac = (p.torus_kappa * n) * ish;
	double is2  = 1.0 / fma(shift, shift, GRAY_EPSILON);
#pragma unroll
	for(int i = 0; i < NF; ++i) {
		double j = jfac * p.nupow[i];
		ds[8 + i]      = -(j * exp(-s[8 + NF + i])) * is2;
		ds[8 + NF + i] = -(tfac * p.nuinv2[i]);
	}
}

/* phys.cl:66-74 rhs() */
template <int NF>
__device__ __forceinline__ void
rhs64(const RenderParams &p, const double *s, double *ds)
{
	Aux64 aux;
	ks_rhs64(p, s, ds, aux);
	if(NF > 0) {
		if(p.flow == GRAY_FLOW_TORUS) {
			torus_rt64<NF>(p, s, aux, ds);
		} else {
#pragma unroll
			for(int i = 0; i < 2 * NF; ++i)
				ds[8 + i] = 0.0;
		}
	}
}

/* RK4.cl:37-47 integrate() */
template <int NF>
__device__ __forceinline__ void
rk4_64(const RenderParams &p, double *s, double dt)
{
	constexpr int ND = 8 + 2 * NF;
	double k1[ND], k2[ND], k3[ND], k4[ND], t[ND];
	double hdt = 0.5 * dt;
	rhs64<NF>(p, s, k1);
#pragma unroll
	for(int i = 0; i < ND; ++i) t[i] = fma(hdt, k1[i], s[i]);
	rhs64<NF>(p, t, k2);
#pragma unroll
	for(int i = 0; i < ND; ++i) t[i] = fma(hdt, k2[i], s[i]);
	rhs64<NF>(p, t, k3);
#pragma unroll
	for(int i = 0; i < ND; ++i) t[i] = fma(dt, k3[i], s[i]);
	rhs64<NF>(p, t, k4);
	double h6 = dt / 6.0;
#pragma unroll
	for(int i = 0; i < ND; ++i)
		s[i] = fma(h6, fma(2.0, k2[i] + k3[i], k1[i]) + k4[i], s[i]);
}

/* phys.cl:48-64 getdt() */
__device__ __forceinline__ double
getdt64(const RenderParams &p, const double *q, double dt)
{
	double eps = sqrt(getrr64(p, q[1], q[2], q[3])) - p.rp;
	if(eps < p.eps_stop)
		return 0.0;
	if(fabs(dt) > (0.01 * eps) * eps)
		return copysign((0.01 * eps) * eps, dt);
	return dt;
}

/* f and l_mu at q with the operation sequence of ks_rhs64() */
__device__ __forceinline__ void
ks_fl64(const RenderParams &p, const double *q, double &r_, double &f_,
        double &lx_, double &ly_, double &lz_)
{
	double aa  = p.aa;
	double zz  = q[3] * q[3];
	double kk  = 0.5 * (fma(q[1], q[1], fma(q[2], q[2], zz)) - aa);
	double dd  = sqrt(fma(kk, kk, aa * zz));
	double rr  = dd + kk;
	double r   = sqrt(rr);
	double ir  = 1.0 / r;
	double ss  = rr + aa;
	double iss = 1.0 / ss;
	double tmp = 2.0 / (rr + (aa * zz) / rr);
	r_  = r;
	f_  = tmp * r;
	lx_ = iss * fma(q[1], r, q[2] * p.a);
	ly_ = iss * fma(q[2], r, -(q[1] * p.a));
	lz_ = q[3] * ir;
}

/* KS.cl:91-114 down() */
__device__ __forceinline__ void
down64(const RenderParams &p, const double *q, const double *u, double *k)
{
	double r, f, lx, ly, lz;
	ks_fl64(p, q, r, f, lx, ly, lz);
	double lu  = fma(lz, u[3], fma(ly, u[2], fma(lx, u[1], u[0])));
	double flu = f * lu;
	k[0] = flu - u[0];
	k[1] = fma(flu, lx, u[1]);
	k[2] = fma(flu, ly, u[2]);
	k[3] = fma(flu, lz, u[3]);
}

/* KS.cl:164-168 getuu() */
__device__ __forceinline__ double
getuu64(const RenderParams &p, const double *s)
{
	double k[4];
	down64(p, s, s + 4, k);
	return fma(k[3], s[7], fma(k[2], s[6], fma(k[1], s[5], k[0] * s[4])));
}

__device__ __forceinline__ void
warp_add_steps(unsigned long long *steps, unsigned long long v)
{
#pragma unroll
	for(int o = 16; o > 0; o >>= 1)
		v += __shfl_xor_sync(0xffffffffu, v, o);
	if((threadIdx.x & 31) == 0 && v)
		atomicAdd(steps, v);
}

/* driver.cl:36-67 icond_drv(), KS.cl:188-232 gr_icond(), rt.cl:179-183 */
__global__ void __launch_bounds__(128)
icond64_kernel(const RenderParams p, double *__restrict__ data,
               double *__restrict__ info)
{
	const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if(g >= p.n_rays)
		return;
	const long long gi = g % p.w_rays;
	const long long gj = p.row0 + g / p.w_rays;
	double alpha = (((double)gi + 0.5) / (double)p.w_rays - 0.5) * p.w_img;
	double beta  = (((double)gj + 0.5) / (double)p.h_rays - 0.5) * p.h_img;

	double R0 = fma(p.r_obs, p.si, -(beta * p.ci));
	double z  = fma(p.r_obs, p.ci, beta * p.si);
	double y  = fma(R0, p.sj, alpha * p.cj);
	double x  = fma(R0, p.cj, -(alpha * p.sj));
	double s[8] = {0.0, x, y, z, 1.0, p.si * p.cj, p.si * p.sj, p.ci};

	double r, f, lx, ly, lz;
	ks_fl64(p, s, r, f, lx, ly, lz);
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

	const long long n = p.n_rays;
#pragma unroll
	for(int c = 0; c < 8; ++c)
		data[c * n + g] = s[c];
	for(int c = 8; c < p.n_data; ++c)
		data[c * n + g] = 0.0;
	info[g] = getuu64(p, s);
}

/* driver.cl:69-108 evolve_drv(): integer-tick substepping over one dump
 * interval of affine length dt with n_sub substeps. */
template <int NF>
__global__ void __launch_bounds__(128)
evolve64_kernel(const RenderParams p, double *__restrict__ data,
                double *__restrict__ info, const double dt, const long long n_sub,
                unsigned long long *__restrict__ steps)
{
	constexpr int ND = 8 + 2 * NF;
	const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	const long long nr = p.n_rays;
	unsigned long long cnt = 0;
	if(g < nr) {
		double s[ND];
#pragma unroll
		for(int c = 0; c < ND; ++c)
			s[c] = data[c * nr + g];

		const int n = (int)((INT_MAX / n_sub) * n_sub);
		const double dts = dt / (double)n_sub;
		int h, dh;
		for(h = 0; h < n; h += dh) {
			dh = (int)(getdt64(p, s, dts) / dt * (double)n);
			if(!dh)
				break;
			if(dh > n - h)
				dh = n - h;
			rk4_64<NF>(p, s, ((double)dh * dt) / (double)n);
			++cnt;
		}
#pragma unroll
		for(int c = 0; c < ND; ++c)
			data[c * nr + g] = s[c];
		info[g] = getuu64(p, s);
	}
	warp_add_steps(steps, cnt);
}

__global__ void
kdown64_kernel(const RenderParams p, const double *__restrict__ data,
               double *__restrict__ k)
{
	const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	const long long n = p.n_rays;
	if(g >= n)
		return;
	double s[8], kk[4];
#pragma unroll
	for(int c = 0; c < 8; ++c)
		s[c] = data[c * n + g];
	down64(p, s, s + 4, kk);
#pragma unroll
	for(int c = 0; c < 4; ++c)
		k[c * n + g] = kk[c];
}

/* KS.cl:63-153 output coordinates, in the oracle's operation order.  The
 * event of down()'s metric is x + i y = (r + i a) e^(i phi) sin(theta);
 * KS.cl:68-69 and 130 use (r - i a), and KS.cl:148-151 put u^phi and u^t
 * where u^r belongs: as_written reproduces both. */
__device__ __forceinline__ void
sph_ks64(const RenderParams &p, const double *q, int as_written, double *out)
{
	double r = sqrt(getrr64(p, q[1], q[2], q[3]));
	double sa = as_written ? p.a : -p.a;
	out[0] = q[0];
	out[1] = r;
	out[2] = acos(q[3] / r);
	out[3] = atan2(fma(q[2], r, q[1] * sa), fma(q[1], r, -(q[2] * sa)));
}

__device__ __forceinline__ void
sph_ks_u64(const RenderParams &p, const double *q, const double *u, int as_written,
           double *out)
{
	const double aa = p.aa;
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
	double c = (as_written ? -p.a : p.a) / (rr + aa);
	double J3[4] = {0.0, fma(c, J1[1], -q[2] / RR), fma(c, J1[2], q[1] / RR), c * J1[3]};
	out[0] = u[0];
	out[1] = fma(J1[3], u[3], fma(J1[2], u[2], J1[1] * u[1]));
	out[2] = fma(J2[3], u[3], fma(J2[2], u[2], J2[1] * u[1]));
	out[3] = fma(J3[3], u[3], fma(J3[2], u[2], J3[1] * u[1]));
}

/* system 0: spherical KS; 1: Boyer-Lindquist with t matched at r_match */
__global__ void
coords64_kernel(const RenderParams p, const double *__restrict__ data,
                double *__restrict__ out, int system, double r_match, int as_written)
{
	const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	const long long n = p.n_rays;
	if(g >= n)
		return;
	double s[8], x[4], v[4];
#pragma unroll
	for(int c = 0; c < 8; ++c)
		s[c] = data[c * n + g];
	const double *q = s, *u = s + 4;
	sph_ks64(p, q, as_written, x);
	sph_ks_u64(p, q, u, as_written, v);
	if(system == 1) {
		double h  = sqrt(1.0 - p.aa);
		double rp = 1.0 + h, rm = 1.0 - h, r = x[1];
		x[0] = x[0] + (rm * log((r - rm) / (r_match - rm)) -
		               rp * log((r - rp) / (r_match - rp))) / h;
		x[3] = x[3] + 0.5 * p.a * log((r - rm) / (r - rp)) / h;
		double rr = getrr64(p, q[1], q[2], q[3]);
		double rq = sqrt(rr);
		double D  = rr - 2.0 * rq + p.aa;
		double ut = as_written ? v[3] : v[1];
		double up = as_written ? v[0] : v[1];
		v[0] = v[0] - ut * 2.0 * rq / D;
		v[3] = v[3] - up * p.a / D;
	}
#pragma unroll
	for(int c = 0; c < 4; ++c) {
		out[c * n + g] = x[c];
		out[(4 + c) * n + g] = v[c];
	}
}

__global__ void
getuu64_kernel(const RenderParams p, const double *__restrict__ data,
               double *__restrict__ info)
{
	const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	const long long n = p.n_rays;
	if(g >= n)
		return;
	double s[8];
#pragma unroll
	for(int c = 0; c < 8; ++c)
		s[c] = data[c * n + g];
	info[g] = getuu64(p, s);
}

/* SoA <-> AoS (sim-org/SoA.cl:29 vs AoS.cl:29) through a tile in shared
 * memory so both sides stay coalesced. */
__global__ void
transpose_kernel(const double *__restrict__ src, double *__restrict__ dst,
                 long long n_rays, int n_data, int to_aos)
{
	extern __shared__ double tile[]; /* [n_data][64] */
	const long long base = (long long)blockIdx.x * 64;
	const int tid = threadIdx.x;
	const int total = 64 * n_data;
	for(int e = tid; e < total; e += blockDim.x) {
		if(to_aos) {
			int c = e / 64, r = e % 64;
			long long g = base + r;
			if(g < n_rays)
				tile[c * 64 + r] = src[(long long)c * n_rays + g];
		} else {
			int r = e / n_data, c = e % n_data;
			long long g = base + r;
			if(g < n_rays)
				tile[c * 64 + r] = src[g * n_data + c];
		}
	}
	__syncthreads();
	for(int e = tid; e < total; e += blockDim.x) {
		if(to_aos) {
			int r = e / n_data, c = e % n_data;
			long long g = base + r;
			if(g < n_rays)
				dst[g * n_data + c] = tile[c * 64 + r];
		} else {
			int c = e / 64, r = e % 64;
			long long g = base + r;
			if(g < n_rays)
				dst[(long long)c * n_rays + g] = tile[c * 64 + r];
		}
	}
}

inline unsigned
blocks_for(long long n, int block)
{
	return (unsigned)((n + block - 1) / block);
}

} /* namespace */

cudaError_t
launch_icond64(const RenderParams &p, double *data, double *info, cudaStream_t st)
{
	icond64_kernel<<<blocks_for(p.n_rays, 128), 128, 0, st>>>(p, data, info);
	return cudaGetLastError();
}

cudaError_t
launch_evolve64(const RenderParams &p, double *data, double *info, double dt,
                long long n_sub, unsigned long long *steps, cudaStream_t st, int block)
{
	if(block <= 0 || block > 128 || block % 32)
		block = 128;
	const unsigned grid = blocks_for(p.n_rays, block);
	switch(p.n_freq) {
#define CASE(NF) case NF: evolve64_kernel<NF><<<grid, block, 0, st>>>(p, data, info, dt, n_sub, steps); break;
	CASE(0) CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
#undef CASE
	default:
		return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

cudaError_t
launch_kdown64(const RenderParams &p, const double *data, double *k, cudaStream_t st)
{
	kdown64_kernel<<<blocks_for(p.n_rays, 128), 128, 0, st>>>(p, data, k);
	return cudaGetLastError();
}

cudaError_t
launch_coords64(const RenderParams &p, const double *data, double *out, int system,
                double r_match, int as_written, cudaStream_t st)
{
	coords64_kernel<<<blocks_for(p.n_rays, 128), 128, 0, st>>>(p, data, out, system, r_match,
	                                                           as_written);
	return cudaGetLastError();
}

cudaError_t
launch_getuu64(const RenderParams &p, const double *data, double *info, cudaStream_t st)
{
	getuu64_kernel<<<blocks_for(p.n_rays, 128), 128, 0, st>>>(p, data, info);
	return cudaGetLastError();
}

cudaError_t
launch_transpose(const double *src, double *dst, long long n_rays, int n_data,
                 int to_aos, cudaStream_t st)
{
	size_t smem = sizeof(double) * 64 * (size_t)n_data;
	transpose_kernel<<<blocks_for(n_rays, 64), 256, smem, st>>>(src, dst, n_rays,
	                                                            n_data, to_aos);
	return cudaGetLastError();
}
