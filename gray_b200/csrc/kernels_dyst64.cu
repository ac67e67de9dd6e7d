/*
 * FP64 numerical-spacetime kernels and the boosted Kerr-Schild grid
 * generator.  Compiled with -fmad=false: the only fused multiply-adds are
 * the explicit fma() calls that mirror the CPU oracle.
 *
 *  - dyst_icond_kernel, dyst_evolve64_kernel: dyst.cl:89-110 camera rays
 *    and driver.cl:69-108 substepping on the interpolated spacetime, one
 *    ray per thread, one launch per dump (the reference structure).
 *  - boosted_ks_kernel: samples boosted Kerr-Schild on the grid (the
 *    generator of tools/generate_data.py:87-160 with tools/boosted_ks.py's
 *    dual-number derivatives), one grid point per thread.
 */
#include <climits>

#include "dyst64.cuh"

namespace {

using namespace dyst64;

/* dyst.cl:89-110: camera ray, not null-normalised */
__global__ void __launch_bounds__(128)
dyst_icond_kernel(const RenderParams p, const GridParams g, double *__restrict__ data,
                  double *__restrict__ info)
{
	const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if(r >= p.n_rays)
		return;
	const long long gi = r % p.w_rays;
	const long long gj = p.row0 + r / p.w_rays;
	double alpha = (((double)gi + 0.5) / (double)p.w_rays - 0.5) * p.w_img;
	double beta  = (((double)gj + 0.5) / (double)p.h_rays - 0.5) * p.h_img;
	double R0 = fma(p.r_obs, p.si, -(beta * p.ci));
	double z  = fma(p.r_obs, p.ci, beta * p.si);
	double y  = fma(R0, p.sj, alpha * p.cj);
	double x  = fma(R0, p.cj, -(alpha * p.sj));
	double s[8] = {0.0, x, y, z, 1.0, p.si * p.cj, p.si * p.sj, p.ci};
	const long long n = p.n_rays;
#pragma unroll
	for(int c = 0; c < 8; ++c)
		data[c * n + r] = s[c];
	for(int c = 8; c < p.n_data; ++c)
		data[c * n + r] = 0.0; /* rt_icond(), rt.cl:179-183 */
	info[r] = dyst_getuu64(g, s);
}

/* driver.cl:69-108 on the numerical spacetime, with NF transfer pairs */
template <int NF>
__global__ void __launch_bounds__(128)
dyst_evolve64_kernel(const __grid_constant__ RenderParams p, const GridParams g,
                     double *__restrict__ data, double *__restrict__ info, const double dt,
                     const long long n_sub, unsigned long long *__restrict__ steps)
{
	constexpr int ND = 8 + 2 * NF;
	const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	const long long nr = p.n_rays;
	const thermal::Flow f = {p.nu, p.m_adm, p.flow_te, p.flow_b, &p.th};
	unsigned long long cnt = 0;
	if(r < nr) {
		double s[ND];
#pragma unroll
		for(int c = 0; c < ND; ++c)
			s[c] = data[c * nr + r];
		const int n = (int)((INT_MAX / n_sub) * n_sub);
		const double dts = dt / (double)n_sub;
		int h, dh;
		for(h = 0; h < n; h += dh) {
			dh = (int)(dyst_getdt64(dts) / dt * (double)n);
			if(!dh)
				break;
			if(dh > n - h)
				dh = n - h;
			if(NF == 0)
				rk4_dyst64(g, s, ((double)dh * dt) / (double)n);
			else
				rk4_dyst_rt64<NF>(f, g, s, ((double)dh * dt) / (double)n);
			++cnt;
		}
#pragma unroll
		for(int c = 0; c < ND; ++c)
			data[c * nr + r] = s[c];
		info[r] = dyst_getuu64(g, s);
	}
#pragma unroll
	for(int o = 16; o > 0; o >>= 1)
		cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
	if((threadIdx.x & 31) == 0 && cnt)
		atomicAdd(steps, cnt);
}

/* ------------------------------------------------------- boosted KS grid */

struct Dual {
	double f, s;
};
__device__ __forceinline__ Dual D(double f, double s) { Dual r = {f, s}; return r; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return D(a.f + b.f, a.s + b.s); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return D(a.f - b.f, a.s - b.s); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return D(a.f * b.f, a.s * b.f + a.f * b.s); }
__device__ __forceinline__ Dual operator*(Dual a, double c) { return D(a.f * c, a.s * c); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
	return D(a.f / b.f, (a.s * b.f - a.f * b.s) / (b.f * b.f));
}
__device__ __forceinline__ Dual dsqrt(Dual a)
{
	double r = sqrt(a.f);
	return D(r, a.s * 0.5 / r);
}

/* boosted_ks.py:120-186: h and covariant l_mu at X (dual numbers) */
__device__ void
bks_hl(double m, double a, double v, int axis, const Dual *X, Dual &h, Dual *l)
{
	double gam = 1.0 / sqrt(1.0 - v * v);
	Dual x0[4] = {X[0], X[1], X[2], X[3]};
	x0[0]    = (X[0] - X[axis] * v) * gam;
	x0[axis] = (X[axis] - X[0] * v) * gam;
	Dual xx = x0[1], yy = x0[2], zz = x0[3];
	Dual rho2 = xx * xx + yy * yy + zz * zz;
	Dual w = rho2 - D(a * a, 0.0);
	Dual r2 = w * 0.5 + dsqrt(w * w * 0.25 + zz * zz * (a * a));
	Dual r = dsqrt(r2);
	Dual ct = zz / r;
	h = (r * m) / (r2 + ct * ct * (a * a));
	Dual ra2 = r2 + D(a * a, 0.0);
	Dual l0[4] = {D(1.0, 0.0), (r * xx + yy * a) / ra2, (r * yy - xx * a) / ra2, zz / r};
	for(int c = 0; c < 4; ++c)
		l[c] = l0[c];
	l[0]    = (l0[0] - l0[axis] * v) * gam;
	l[axis] = (l0[axis] - l0[0] * v) * gam;
}

/* numpy.nan_to_num then float32 (tools/generate_data.py:143-144) */
__device__ __forceinline__ float
to_f32(double x)
{
	if(x != x)
		return 0.0f;
	return (float)x;
}

__global__ void __launch_bounds__(128)
boosted_ks_kernel(const GridParams g, float *__restrict__ lvl, double m, double a,
                  double v, int axis, double t)
{
	const long long npts = (long long)g.nx * g.ny * g.nz;
	const long long pt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if(pt >= npts)
		return;
	const int ix = (int)(pt % g.nx);
	const int iy = (int)((pt / g.nx) % g.ny);
	const int iz = (int)(pt / ((long long)g.nx * g.ny));
	const double q[4] = {t, g.nodes[0][ix], g.nodes[1][iy], g.nodes[2][iz]};
	const double ETA[4] = {-1.0, 1.0, 1.0, 1.0};
	double dg[4][4][4], gd[4][4], gu[4][4];
	for(int w = 0; w < 4; ++w) {
		Dual X[4], h, l[4];
		for(int c = 0; c < 4; ++c)
			X[c] = D(q[c], c == w ? 1.0 : 0.0);
		bks_hl(m, a, v, axis, X, h, l);
		for(int i = 0; i < 4; ++i)
			for(int j = 0; j < 4; ++j) {
				Dual gij = h * (l[i] * l[j]) * 2.0;
				dg[w][i][j] = gij.s;
				if(w == 0) {
					gd[i][j] = (i == j ? ETA[i] : 0.0) + gij.f;
					double li = i == 0 ? -l[0].f : l[i].f;
					double lj = j == 0 ? -l[0].f : l[j].f;
					gu[i][j] = (i == j ? ETA[i] : 0.0) - 2.0 * h.f * li * lj;
				}
			}
	}
	float *out = lvl + pt * GRAY_NSTRIDE;
	int k = 0;
	for(int i = 0; i < 4; ++i)
		for(int b = 0; b < 4; ++b)
			for(int c = b; c < 4; ++c) {
				double s = 0.0;
				for(int mm = 0; mm < 4; ++mm)
					s += gu[i][mm] * (dg[c][mm][b] + dg[b][mm][c] - dg[mm][b][c]);
				out[k++] = to_f32(0.5 * s);
			}
	for(int i = 0; i < 4; ++i)
		for(int j = i; j < 4; ++j)
			out[k++] = to_f32(gd[i][j]);
	/* generate_data.py:124-128: rho = 1 / r */
	out[50] = to_f32(1.0 / sqrt(q[1] * q[1] + q[2] * q[2] + q[3] * q[3]));
	for(int pad = GRAY_NCOMP; pad < GRAY_NSTRIDE; ++pad)
		out[pad] = 0.0f;
}

inline unsigned
blocks_for(long long n, int block)
{
	return (unsigned)((n + block - 1) / block);
}

} /* namespace */

cudaError_t
launch_dyst_icond(const RenderParams &p, const GridParams &g, double *data, double *info,
                  cudaStream_t st)
{
	dyst_icond_kernel<<<blocks_for(p.n_rays, 128), 128, 0, st>>>(p, g, data, info);
	return cudaGetLastError();
}

cudaError_t
launch_dyst_evolve64(const RenderParams &p, const GridParams &g, double *data, double *info,
                     double dt, long long n_sub, unsigned long long *steps, cudaStream_t st)
{
	const unsigned nb = blocks_for(p.n_rays, 128);
	switch(p.n_freq) {
#define GRAY_DYST64_CASE(NF)                                                             \
	case NF:                                                                         \
		dyst_evolve64_kernel<NF><<<nb, 128, 0, st>>>(p, g, data, info, dt, n_sub, steps); \
		break;
	GRAY_DYST64_CASE(0) GRAY_DYST64_CASE(1) GRAY_DYST64_CASE(2) GRAY_DYST64_CASE(3)
	GRAY_DYST64_CASE(4) GRAY_DYST64_CASE(5) GRAY_DYST64_CASE(6) GRAY_DYST64_CASE(7)
	GRAY_DYST64_CASE(8)
#undef GRAY_DYST64_CASE
	default:
		return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

cudaError_t
launch_boosted_ks(const GridParams &g, float *lvl, double a, double v, int axis, double t,
                  cudaStream_t st)
{
	const long long npts = (long long)g.nx * g.ny * g.nz;
	boosted_ks_kernel<<<blocks_for(npts, 128), 128, 0, st>>>(g, lvl, 1.0, a, v, axis, t);
	return cudaGetLastError();
}
