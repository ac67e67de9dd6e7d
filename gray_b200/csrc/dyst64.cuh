/*
 * FP64 numerical-spacetime device functions (interp.cl:53-205, dyst.cl:14-194),
 * shared by the FP64 kernels (kernels_dyst64.cu, compiled with -fmad=false so
 * that they round like the CPU oracle) and by the mixed kernel's FP64 island
 * (the final null-constraint check).
 */
#ifndef GRAY_DYST64_CUH
#define GRAY_DYST64_CUH

#include "gray_internal.h"
#include "thermal.cuh"

namespace dyst64 {


/* interp.cl:69-97 + 123-164 for one axis (fractional logical coordinate) */
__device__ __forceinline__ double
axis_uvw64(const GridParams &g, int a, double x)
{
	const int n = a == 0 ? g.nx : a == 1 ? g.ny : g.nz;
	double xi = floor((cbrt(asinh(x)) - g.B[a]) / g.A[a]);
	int i;
	if(!(xi >= 0.0))
		i = 0;
	else if(xi > (double)(n - 1))
		i = n - 1;
	else
		i = (int)xi;
	double x0 = g.nodes[a][i];
	double x1 = g.nodes[a][i + 1];
	double u  = (double)i + (x - x0) / (x1 - x0);
	if(!(u >= 0.0))
		u = 0.0;
	if(u > (double)(n - 1))
		u = (double)(n - 1);
	return u;
}

struct Cell64 {
	long long idx[8]; /* corner row offsets (in floats) */
	double w[8];
};

/* CLK_FILTER_LINEAR + CLAMP_TO_EDGE weights, corner order 000, 100, 010,
 * 110, 001, 101, 011, 111 (as the oracle's trilinear()) */
__device__ __forceinline__ void
cell64(const GridParams &g, const double *q, Cell64 &c)
{
	int i0[3], i1[3];
	double w[3];
	const int n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
	for(int a = 0; a < 3; ++a) {
		double u  = axis_uvw64(g, a, q[a + 1]);
		double fl = floor(u);
		i0[a] = (int)fl;
		w[a]  = u - fl;
		i1[a] = i0[a] + 1 < n[a] ? i0[a] + 1 : n[a] - 1;
	}
	double ax = 1.0 - w[0], ay = 1.0 - w[1], az = 1.0 - w[2];
	c.w[0] = (ax * ay) * az;     c.w[1] = (w[0] * ay) * az;
	c.w[2] = (ax * w[1]) * az;   c.w[3] = (w[0] * w[1]) * az;
	c.w[4] = (ax * ay) * w[2];   c.w[5] = (w[0] * ay) * w[2];
	c.w[6] = (ax * w[1]) * w[2]; c.w[7] = (w[0] * w[1]) * w[2];
#pragma unroll
	for(int k = 0; k < 8; ++k) {
		int ix = (k & 1) ? i1[0] : i0[0];
		int iy = (k & 2) ? i1[1] : i0[1];
		int iz = (k & 4) ? i1[2] : i0[2];
		c.idx[k] = (((long long)iz * g.ny + iy) * g.nx + ix) * GRAY_NSTRIDE;
	}
}

__device__ __forceinline__ double
trilin64(const float *F, const Cell64 &c, int comp)
{
	double v = c.w[0] * (double)F[c.idx[0] + comp];
#pragma unroll
	for(int k = 1; k < 8; ++k)
		v = fma(c.w[k], (double)F[c.idx[k] + comp], v);
	return v;
}

__device__ __forceinline__ bool
inside64(const GridParams &g, const double *q)
{
#pragma unroll
	for(int a = 1; a <= 3; ++a)
		if(!(q[a] >= (double)g.box[a] && q[a] <= (double)g.box[a + 4]))
			return false;
	return true;
}

/* interp.cl:183-205 for components [c0, c0 + nc) */
__device__ __forceinline__ void
interp64(const GridParams &g, const double *q, int c0, int nc, double *out)
{
	Cell64 c;
	cell64(g, q, c);
	if(g.single) {
		for(int m = 0; m < nc; ++m)
			out[m] = trilin64(g.lvl[0], c, c0 + m);
		return;
	}
	double t1 = g.box[0], t2 = g.box[4];
	double ft = (q[0] - t1) / (t2 - t1);
	if(g.physics) {
		if(!(ft >= 0.0))
			ft = 0.0;
		if(ft > 1.0)
			ft = 1.0;
	}
	for(int m = 0; m < nc; ++m) {
		double y1 = trilin64(g.lvl[0], c, c0 + m);
		double y2 = trilin64(g.lvl[1], c, c0 + m);
		out[m] = fma(ft, y2 - y1, y1);
	}
}

/* dyst.cl:112-194 gr_rhs */
__device__ __forceinline__ void
dyst_rhs64(const GridParams &g, const double *s, double *ds)
{
	const double *u = s + 4;
	ds[0] = u[0]; ds[1] = u[1]; ds[2] = u[2]; ds[3] = u[3];
	if(g.physics && !inside64(g, s)) {
		ds[4] = ds[5] = ds[6] = ds[7] = 0.0;
		return;
	}
	double v[40], p[10], G[4];
	interp64(g, s, 0, 40, v);
	int k = 0;
#pragma unroll
	for(int i = 0; i < 4; ++i)
#pragma unroll
		for(int j = i; j < 4; ++j) {
			double uu = u[i] * u[j];
			p[k++] = i == j ? uu : 2.0 * uu;
		}
#pragma unroll
	for(int m = 0; m < 4; ++m) {
		double acc = v[10 * m] * p[0];
#pragma unroll
		for(int kk = 1; kk < 10; ++kk)
			acc = fma(v[10 * m + kk], p[kk], acc);
		G[m] = acc;
	}
#pragma unroll
	for(int m = 0; m < 4; ++m)
		ds[4 + m] = fma(G[0], u[m], -G[m]);
}

/* dyst.cl:55-81 down() with the optional g_zz bug of dyst.cl:78 */
__device__ __forceinline__ void
dyst_down64(const GridParams &g, const double *q, const double *u, double *k)
{
	if(g.physics && !inside64(g, q)) {
		k[0] = -u[0]; k[1] = u[1]; k[2] = u[2]; k[3] = u[3];
		return;
	}
	double c[10], M[4][4];
	interp64(g, q, 40, 10, c);
	if(g.bug_gzz)
		c[9] = c[8];
	int n = 0;
	for(int i = 0; i < 4; ++i)
		for(int j = i; j < 4; ++j) {
			M[i][j] = c[n];
			M[j][i] = c[n];
			++n;
		}
	for(int i = 0; i < 4; ++i)
		k[i] = fma(M[i][3], u[3], fma(M[i][2], u[2], fma(M[i][1], u[1], M[i][0] * u[0])));
}

__device__ __forceinline__ double
dyst_getuu64(const GridParams &g, const double *s)
{
	double k[4];
	dyst_down64(g, s, s + 4, k);
	return fma(k[3], s[7], fma(k[2], s[6], fma(k[1], s[5], k[0] * s[4])));
}

__device__ __forceinline__ void
rk4_dyst64(const GridParams &g, double *s, double dt)
{
	double k1[8], k2[8], k3[8], k4[8], t[8];
	double hdt = 0.5 * dt;
	dyst_rhs64(g, s, k1);
#pragma unroll
	for(int i = 0; i < 8; ++i) t[i] = fma(hdt, k1[i], s[i]);
	dyst_rhs64(g, t, k2);
#pragma unroll
	for(int i = 0; i < 8; ++i) t[i] = fma(hdt, k2[i], s[i]);
	dyst_rhs64(g, t, k3);
#pragma unroll
	for(int i = 0; i < 8; ++i) t[i] = fma(dt, k3[i], s[i]);
	dyst_rhs64(g, t, k4);
	double h6 = dt / 6.0;
#pragma unroll
	for(int i = 0; i < 8; ++i)
		s[i] = fma(h6, fma(2.0, k2[i] + k3[i], k1[i]) + k4[i], s[i]);
}

/* phys.cl:66-74 on the numerical spacetime with the thermal transfer of
 * NF frequencies: the geodesic of dyst_rhs64, k = down(q, u) of
 * dyst_down64 and n_e = rho from one cell search for all 51 fields (the
 * reference interpolates field by field: same values).  In physics mode
 * outside the box the spacetime is flat and n_e = 0. */
template <int NF>
__device__ __forceinline__ void
dyst_rhs_rt64(const thermal::Flow &f, const GridParams &g, const double *s, double *ds)
{
	const double *u = s + 4;
	double k[4], ne;
	ds[0] = u[0]; ds[1] = u[1]; ds[2] = u[2]; ds[3] = u[3];
	if(g.physics && !inside64(g, s)) {
		ds[4] = ds[5] = ds[6] = ds[7] = 0.0;
		k[0] = -u[0]; k[1] = u[1]; k[2] = u[2]; k[3] = u[3];
		ne = 0.0;
	} else {
		double v[GRAY_NCOMP], p[10], G[4], M[4][4];
		interp64(g, s, 0, GRAY_NCOMP, v);
		int n = 0;
#pragma unroll
		for(int i = 0; i < 4; ++i)
#pragma unroll
			for(int j = i; j < 4; ++j) {
				double uu = u[i] * u[j];
				p[n++] = i == j ? uu : 2.0 * uu;
			}
#pragma unroll
		for(int m = 0; m < 4; ++m) {
			double acc = v[10 * m] * p[0];
#pragma unroll
			for(int kk = 1; kk < 10; ++kk)
				acc = fma(v[10 * m + kk], p[kk], acc);
			G[m] = acc;
		}
#pragma unroll
		for(int m = 0; m < 4; ++m)
			ds[4 + m] = fma(G[0], u[m], -G[m]);
		if(g.bug_gzz)
			v[49] = v[48];
		n = 40;
#pragma unroll
		for(int i = 0; i < 4; ++i)
#pragma unroll
			for(int j = i; j < 4; ++j) {
				M[i][j] = v[n];
				M[j][i] = v[n];
				++n;
			}
#pragma unroll
		for(int i = 0; i < 4; ++i)
			k[i] = fma(M[i][3], u[3], fma(M[i][2], u[2], fma(M[i][1], u[1], M[i][0] * u[0])));
		ne = v[50];
	}
	thermal::rt_rhs<NF>(f, k, ne, s + 8 + NF, ds + 8, ds + 8 + NF);
}

/* RK4 of the geodesic and NF transfer pairs (I, tau) */
template <int NF>
__device__ __forceinline__ void
rk4_dyst_rt64(const thermal::Flow &f, const GridParams &g, double *s, double dt)
{
	constexpr int ND = 8 + 2 * NF;
	double k1[ND], k2[ND], k3[ND], k4[ND], t[ND];
	double hdt = 0.5 * dt;
	dyst_rhs_rt64<NF>(f, g, s, k1);
#pragma unroll
	for(int i = 0; i < ND; ++i) t[i] = fma(hdt, k1[i], s[i]);
	dyst_rhs_rt64<NF>(f, g, t, k2);
#pragma unroll
	for(int i = 0; i < ND; ++i) t[i] = fma(hdt, k2[i], s[i]);
	dyst_rhs_rt64<NF>(f, g, t, k3);
#pragma unroll
	for(int i = 0; i < ND; ++i) t[i] = fma(dt, k3[i], s[i]);
	dyst_rhs_rt64<NF>(f, g, t, k4);
	double h6 = dt / 6.0;
#pragma unroll
	for(int i = 0; i < ND; ++i)
		s[i] = fma(h6, fma(2.0, k2[i] + k3[i], k1[i]) + k4[i], s[i]);
}

/* phys.cl:48-64 with dyst.cl:43-53 (getrr = geteps = 1) */
__device__ __forceinline__ double
dyst_getdt64(double dt)
{
	const double eps = 1.0;
	if(fabs(dt) > (0.01 * eps) * eps)
		return copysign((0.01 * eps) * eps, dt);
	return dt;
}

} /* namespace dyst64 */

#endif /* GRAY_DYST64_CUH */
