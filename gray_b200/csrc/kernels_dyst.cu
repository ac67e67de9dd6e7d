/*
 * Mixed-precision persistent kernel for numerical spacetimes (interp.cl +
 * dyst.cl): warp-refilled rays, FP32 gathers of the 40 Christoffel symbols
 * accumulated with packed f32x2 FMA over component pairs, compensated
 * (hi, lo) state update, FP64 null-constraint check at the end.
 *
 * Grid layout: per time level float [nz][ny][nx][GRAY_NSTRIDE] with the
 * fields of one grid point contiguous (Gamma 0..39, g 40..49, rho 50, pad),
 * so the 8 corners of a cell are 8 rows of 224 bytes and the 40 Gamma of a
 * corner are 5 aligned 32-byte loads (sm_100 ld.global.v8.f32).  The fisheye node coordinates come
 * from a per-axis table (n + 1 entries) instead of sinh((A i + B)^3) per
 * field and call (interp.cl:99-121), and the cell search runs once per RHS
 * for all fields instead of once per field (102 times in the reference).
 */
#include <cfloat>
#include <climits>

#include "dyst64.cuh"
#include "mixed_table.h"

#ifndef GRAY_DYST_PREFETCH
#define GRAY_DYST_PREFETCH 0
#endif

namespace {

using dyst64::dyst_getuu64;
using dyst64::dyst_getdt64;

/* ---------------------------------------------------------------- mixed */

__device__ __forceinline__ float
rcp_a(float x)
{
	float r;
	asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
	return r;
}

__device__ __forceinline__ float
ex2_a(float x)
{
	float r;
	asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
	return r;
}

__device__ __forceinline__ float
lg2_a(float x)
{
	float r;
	asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
	return r;
}

__device__ __forceinline__ float
sqrt_a(float x)
{
	float r;
	asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
	return r;
}

struct DystConst {
	float B[3], iA[3];
};

/* threads per block at most (the kernels' launch bound): the stride of the
 * per-thread cell cache in shared memory */
constexpr int CELL_STRIDE = 256;

/* Fractional logical coordinate on a fisheye axis, with the cell found
 * exactly against the node table: the FP32 map only gives the first guess,
 * node comparisons settle it (the answer depends on x and the table alone).
 * The last interior cell of each thread is kept in `cache` (x0, x1,
 * 1/(x1 - x0), i): a ray moves about 0.01 M per stage through cells 0.2-2 M
 * wide, so nearly every call skips the map (three MUFU in a chain) and the
 * two node loads, with the same result the search would give. */
__device__ __forceinline__ float
axis_uvw32c(const GridParams &g, int a, float x, float Bf, float iAf, float4 &cache)
{
	if(x >= cache.x && x < cache.y)
		return cache.w + (x - cache.x) * cache.z;
	const int n = a == 0 ? g.nx : a == 1 ? g.ny : g.nz;
	const float *nd = g.nodes_f[a];
	if(!(x >= __ldg(nd)))
		return 0.0f;              /* before the first node (or NaN): clamp-to-edge */
	if(x >= __ldg(nd + n - 1))
		return (float)(n - 1);    /* at or past the last node */
	float ax = fabsf(x);
	float as = 0.69314718f * lg2_a(ax + sqrt_a(fmaf(ax, ax, 1.0f)));   /* asinh|x| */
	float cb = as > 0.0f ? ex2_a(0.33333334f * lg2_a(as)) : 0.0f;       /* cbrt     */
	cb = copysignf(cb, x);
	float xi = floorf((cb - Bf) * iAf);
	int i = xi >= 0.0f ? (xi <= (float)(n - 2) ? (int)xi : n - 2) : 0;
	float x0 = __ldg(nd + i), x1 = __ldg(nd + i + 1);
	/* nd[0] <= x < nd[n-1] keeps both walks inside [0, n-2] */
	for(int it = 0; it < 2 && x < x0; ++it) {
		--i;
		x1 = x0;
		x0 = __ldg(nd + i);
	}
	for(int it = 0; it < 2 && x >= x1; ++it) {
		++i;
		x0 = x1;
		x1 = __ldg(nd + i + 1);
	}
	const float inv = rcp_a(x1 - x0);
	cache = make_float4(x0, x1, inv, (float)i);
	return (float)i + (x - x0) * inv;
}

/* eight consecutive floats from a 32-byte aligned address, through the
 * read-only path */
struct F8 {
	float v[8];
};

__device__ __forceinline__ F8
ldg8(const float *p)
{
	F8 r;
	asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
	    : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]), "=f"(r.v[5]),
	      "=f"(r.v[6]), "=f"(r.v[7])
	    : "l"(p));
	return r;
}

/* ------------------------------------------------ thermal transfer island */

/* 1/b to ~1e-14 relative: the FP32 approximate reciprocal refined by one
 * FP64 Newton step (b within the FP32 normal range) */
__device__ __forceinline__ double
rcp64(double b)
{
	const double r = (double)rcp_a((float)b);
	return fma(r, fma(-b, r, 1.0), r);
}

/* e^x for |x| within the FP32 range, ~1e-7 relative */
__device__ __forceinline__ float
exp_f(float x)
{
	return ex2_a(x * 1.4426950408889634f);
}

/* rt.cl:80-198 for the mixed kernel: the magnitudes (1e-47 .. 1e+39 in CGS)
 * stay FP64, the special functions of O(1) arguments (exp, log, cbrt,
 * sqrt) take the FP32 approximate instructions, and everything that
 * depends only on the render is a ThermalFast constant.  Same formulas and
 * branches as the FP64 kernels; agreement to ~1e-6 relative. */
template <int NF>
__device__ __forceinline__ void
rt_rhs_fast(const ThermalFast &t, const double *nu_hz, const double *k, double ne,
            const double *tau, double *dI, double *dtau)
{
	const double EPS = GRAY_EPSILON;
	const double shift = -k[0];
	const float bkcos = (float)(k[3] * t.b) * rcp_a((float)(shift * t.b + EPS));
	const double ish2 = rcp64(fma(shift, shift, EPS));
	/* synchrotron frequency: nu_s = knus sin(theta), zero along the field */
	double nus = 0.0, inus = 0.0;
	const bool syn = t.syn && bkcos > -1.0f && bkcos < 1.0f;
	if(syn) {
		nus = t.knus * (double)sqrt_a(fmaf(-bkcos, bkcos, 1.0f));
		inus = rcp64(nus + EPS);
	}
	const double ne2 = ne * ne;
#pragma unroll
	for(int i = 0; i < NF; ++i) {
		const double nu = nu_hz[i] * shift;
		/* rt.cl:80-93 */
		const double f2 = nu * t.kf2;
		double B;
		if(f2 > 1e-5) {
			double em1;
			if(f2 < 0.3) /* e^f2 - 1 by its series: no cancellation */
				em1 = f2 * fma(f2, fma(f2, fma(f2, fma(f2, fma(f2, fma(f2,
				      1.0 / 5040, 1.0 / 720), 1.0 / 120), 1.0 / 24), 1.0 / 6), 0.5), 1.0);
			else if(f2 < 80.0)
				em1 = (double)exp_f((float)f2) - 1.0;
			else
				em1 = exp(f2);
			B = t.kB * (nu * nu) * nu / em1;
		} else {
			B = t.kB2 * (nu * nu) * rcp64(fma(f2, fma(f2, 1.0 / 6, 0.5), 1.0));
		}
		/* rt.cl:95-143 bremsstrahlung */
		const double y = nu * t.ky;
		double Lff = 0.0;
		if(y < 80.0) {
			const float yf = (float)(y + EPS);
			const float sy = sqrt_a((float)y);
			double G;
			if(t.xg > 1.0)
				G = y > 1.0 ? t.g1 / (double)sy
				            : t.g2 * (t.g3 - 0.6931471805599453 * (double)lg2_a(yf));
			else if(t.xg * y > 1.0)
				G = t.g5 * rcp64(t.sxg * (double)sy);
			else if(y > t.sxg)
				G = 1.0;
			else {
				G = t.g2 * (t.g4 + 0.6931471805599453 *
				                      (double)(lg2_a((float)t.sxg) - lg2_a(yf)));
				G = G > EPS ? G : EPS;
			}
			Lff = (t.kff * ne2) * G * rcp64(fma(t.sqte, (double)exp_f((float)y), EPS));
		}
		/* rt.cl:145-170 synchrotron */
		double Lsyn = 0.0;
		if(syn) {
			double x = nu * inus;
			x = x < 1e30 ? x : 1e30; /* e^-cbrt(x) is 0 long before */
			const float xf = (float)x;
			const float cx = ex2_a(0.33333334f * lg2_a(xf));
			const double xx = (double)sqrt_a(xf) + 1.88774862536 * (double)sqrt_a(cx);
			Lsyn = t.ksyn * (xx * xx) * (double)exp_f(-cx) * (ne * nus);
		}
		const double L = Lsyn + Lff;
		dI[i]   = -L * (double)exp_f(-(float)tau[i]) * ish2;
		dtau[i] = -L * shift * rcp64(B + EPS);
	}
}

__device__ __forceinline__ bool
inside32(const GridParams &g, const float *q)
{
#pragma unroll
	for(int a = 1; a <= 3; ++a)
		if(!(q[a] >= g.box[a] && q[a] <= g.box[a + 4]))
			return false;
	return true;
}

/* Gamma^mu_ab u^a u^b for mu = t,x,y,z from the 40 interpolated Gamma:
 * each corner's row is gathered with 32-byte loads and contracted with
 * u^a u^b before the trilinear weight is applied.
 * With RT, also the covariant momentum k_mu = g_mu,nu u^nu (dyst.cl:55-81,
 * with the g_zz flag of dyst.cl:78) and n_e = rho (flow.cl:48) into
 * kn[0..3] and kn[4], contracted per corner like Gamma. */
template <bool RT = false>
__device__ __forceinline__ void
dyst_rhs32(const GridParams &g, const DystConst &dc, float4 *cells, const float *s, float *ds,
           float *kn = nullptr)
{
	const float *u = s + 4;
	ds[0] = u[0]; ds[1] = u[1]; ds[2] = u[2]; ds[3] = u[3];
	if(g.physics && !inside32(g, s)) {
		ds[4] = ds[5] = ds[6] = ds[7] = 0.0f;
		if(RT) {
			kn[0] = -u[0]; kn[1] = u[1]; kn[2] = u[2]; kn[3] = u[3];
			kn[4] = 0.0f;
		}
		return;
	}
	int i0[3], i1[3];
	float w[3];
	const int n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
	for(int a = 0; a < 3; ++a) {
		float uu = axis_uvw32c(g, a, s[a + 1], dc.B[a], dc.iA[a], cells[a * CELL_STRIDE]);
		float fl = floorf(uu);
		i0[a] = (int)fl;
		w[a] = uu - fl;
		i1[a] = min(i0[a] + 1, n[a] - 1);
	}
	float ft = 0.0f;
	if(!g.single) {
		ft = (s[0] - g.box[0]) * rcp_a(g.box[4] - g.box[0]);
		if(g.physics)
			ft = fminf(fmaxf(ft, 0.0f), 1.0f);
	}
	/* u^a u^b over the 10 stored (a <= b) components, off-diagonal doubled */
	float p[10];
	{
		int k = 0;
#pragma unroll
		for(int i = 0; i < 4; ++i)
#pragma unroll
			for(int j = i; j < 4; ++j) {
				float uu = u[i] * u[j];
				p[k++] = i == j ? uu : 2.0f * uu;
			}
	}
	/* Interpolation and the contraction with u u are both linear, so each
	 * corner's 40 Gamma are contracted first (4 sums) and only the sums are
	 * weighted: 4 accumulators instead of 40 keeps registers for warps. */
	float Gm[4] = {0.0f, 0.0f, 0.0f, 0.0f};
	float Km[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
	const float ax = 1.0f - w[0], ay = 1.0f - w[1], az = 1.0f - w[2];
	/* a time level whose weight is zero (t outside [t1, t2] in physics
	 * mode, where the factor is clamped) is not fetched at all */
	const bool use0 = g.single || ft < 1.0f;
	const bool use1 = !g.single && ft > 0.0f;
#if GRAY_DYST_PREFETCH
	if constexpr(!RT) {
		/* the (corner, level) rows double-buffered in registers: the next
		 * row's five loads are in flight while the current row is
		 * contracted.  Built only with GRAY_DYST_PREFETCH=1: on
		 * numerical_128 it measured 1.6x slower under the 128-register
		 * cap (the second buffer spills) and 1.17x slower at 250 registers
		 * (half the warps per SM) */
		const int nl = (use0 ? 1 : 0) + (use1 ? 1 : 0), l0 = use0 ? 0 : 1, items = 8 * nl;
		auto src_of = [&](int it) {
			const int c = it / nl, l = l0 + it % nl;
			const int ix = (c & 1) ? i1[0] : i0[0];
			const int iy = (c & 2) ? i1[1] : i0[1];
			const int iz = (c & 4) ? i1[2] : i0[2];
			return g.lvl[l] + (((long long)iz * g.ny + iy) * g.nx + ix) * GRAY_NSTRIDE;
		};
		auto contract = [&](const F8 *v, int it) {
			const int c = it / nl, l = l0 + it % nl;
			float wl = ((c & 1) ? w[0] : ax) * ((c & 2) ? w[1] : ay) * ((c & 4) ? w[2] : az);
			if(!g.single)
				wl *= l ? ft : 1.0f - ft;
			float sm[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
			for(int k = 0; k < 5; ++k)
#pragma unroll
				for(int q = 0; q < 8; ++q) {
					const int idx = 8 * k + q;
					sm[idx / 10] = fmaf(v[k].v[q], p[idx % 10], sm[idx / 10]);
				}
#pragma unroll
			for(int m = 0; m < 4; ++m)
				Gm[m] = fmaf(wl, sm[m], Gm[m]);
		};
		F8 A[5], B[5];
		{
			const float *s0 = src_of(0);
#pragma unroll
			for(int k = 0; k < 5; ++k)
				A[k] = ldg8(s0 + 8 * k);
		}
#pragma unroll 1
		for(int it = 0; it < items; it += 2) { /* items is 8 or 16 */
			const float *sb = src_of(it + 1);
#pragma unroll
			for(int k = 0; k < 5; ++k)
				B[k] = ldg8(sb + 8 * k);
			contract(A, it);
			if(it + 2 < items) {
				const float *sa = src_of(it + 2);
#pragma unroll
				for(int k = 0; k < 5; ++k)
					A[k] = ldg8(sa + 8 * k);
			}
			contract(B, it + 1);
		}
#pragma unroll
		for(int m = 0; m < 4; ++m)
			ds[4 + m] = fmaf(Gm[0], u[m], -Gm[m]);
		return;
	}
#endif
	/* one corner at a time: unrolling the eight corners buys no load
	 * parallelism the 16 resident warps do not already give, and its
	 * register pressure spills (measured 13% slower) */
#pragma unroll 1
	for(int c = 0; c < 8; ++c) {
		float wc = ((c & 1) ? w[0] : ax) * ((c & 2) ? w[1] : ay) * ((c & 4) ? w[2] : az);
		int ix = (c & 1) ? i1[0] : i0[0];
		int iy = (c & 2) ? i1[1] : i0[1];
		int iz = (c & 4) ? i1[2] : i0[2];
		long long row = (((long long)iz * g.ny + iy) * g.nx + ix) * GRAY_NSTRIDE;
		for(int l = 0; l < 2; ++l) {
			if(!(l ? use1 : use0))
				continue;
			float wl = g.single ? wc : wc * (l ? ft : 1.0f - ft);
			const float *src = g.lvl[l] + row;
			float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
			for(int k = 0; k < 5; ++k) {
				const F8 v = ldg8(src + 8 * k);
#pragma unroll
				for(int q = 0; q < 8; ++q) {
					const int idx = 8 * k + q; /* Gamma^(idx/10)_(idx%10) */
					s[idx / 10] = fmaf(v.v[q], p[idx % 10], s[idx / 10]);
				}
			}
#pragma unroll
			for(int m = 0; m < 4; ++m)
				Gm[m] = fmaf(wl, s[m], Gm[m]);
			if(RT) {
				/* g_tt g_tx g_ty g_tz g_xx g_xy g_xz g_yy | g_yz g_zz rho pad */
				const F8 ab = ldg8(src + 40), de = ldg8(src + 48);
				const float4 a = make_float4(ab.v[0], ab.v[1], ab.v[2], ab.v[3]);
				const float4 b = make_float4(ab.v[4], ab.v[5], ab.v[6], ab.v[7]);
				const float4 d = make_float4(de.v[0], de.v[1], de.v[2], de.v[3]);
				const float gzz = g.bug_gzz ? d.x : d.y;
				const float k0 = fmaf(a.w, u[3], fmaf(a.z, u[2], fmaf(a.y, u[1], a.x * u[0])));
				const float k1 = fmaf(b.z, u[3], fmaf(b.y, u[2], fmaf(b.x, u[1], a.y * u[0])));
				const float k2 = fmaf(d.x, u[3], fmaf(b.w, u[2], fmaf(b.y, u[1], a.z * u[0])));
				const float k3 = fmaf(gzz, u[3], fmaf(d.x, u[2], fmaf(b.z, u[1], a.w * u[0])));
				Km[0] = fmaf(wl, k0, Km[0]);
				Km[1] = fmaf(wl, k1, Km[1]);
				Km[2] = fmaf(wl, k2, Km[2]);
				Km[3] = fmaf(wl, k3, Km[3]);
				Km[4] = fmaf(wl, d.z, Km[4]);
			}
		}
	}
#pragma unroll
	for(int m = 0; m < 4; ++m)
		ds[4 + m] = fmaf(Gm[0], u[m], -Gm[m]);
	if(RT) {
#pragma unroll
		for(int m = 0; m < 5; ++m)
			kn[m] = Km[m];
	}
}

/* ------------------------------------------ gathers staged in shared memory */

/* The same geodesic RHS with the corner rows staged through shared memory:
 * each (corner, level) row of 40 Gamma is copied global -> shared with ten
 * 16-byte cp.async (through L1, .ca) into a per-thread double buffer, and
 * the copy of the next row is in flight while the current one is
 * contracted.  The loads then hold no registers while they wait, so more of
 * them overlap than the register-resident form allows at 16 warps per SM.
 * Buffer layout [stage][chunk][thread] of float4: a warp's LDS.128 of one
 * chunk touches 32 consecutive float4, without bank conflicts.
 *
 * Built only with GRAY_DYST_STAGED=1: on numerical_128 it measured 5.2x
 * slower than the register gathers.  Its 80 KiB of shared memory per block
 * come out of the same on-chip storage as L1, and the rows that hit L1 95%
 * of the time in the register form then come from L2. */
constexpr int STAGE_CHUNKS = 10; /* 40 floats = 10 x 16 bytes */

__device__ __forceinline__ void
cp_async16(float4 *dst, const float *src)
{
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void
cp_async_commit()
{
	asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int N>
__device__ __forceinline__ void
cp_async_wait()
{
	asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void
dyst_rhs32_staged(const GridParams &g, const DystConst &dc, float4 *cells, float4 *stage,
                  const float *s, float *ds)
{
	const float *u = s + 4;
	ds[0] = u[0]; ds[1] = u[1]; ds[2] = u[2]; ds[3] = u[3];
	if(g.physics && !inside32(g, s)) {
		ds[4] = ds[5] = ds[6] = ds[7] = 0.0f;
		return;
	}
	int i0[3], i1[3];
	float w[3];
	const int n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
	for(int a = 0; a < 3; ++a) {
		float uu = axis_uvw32c(g, a, s[a + 1], dc.B[a], dc.iA[a], cells[a * CELL_STRIDE]);
		float fl = floorf(uu);
		i0[a] = (int)fl;
		w[a] = uu - fl;
		i1[a] = min(i0[a] + 1, n[a] - 1);
	}
	float ft = 0.0f;
	if(!g.single) {
		ft = (s[0] - g.box[0]) * rcp_a(g.box[4] - g.box[0]);
		if(g.physics)
			ft = fminf(fmaxf(ft, 0.0f), 1.0f);
	}
	float p[10];
	{
		int k = 0;
#pragma unroll
		for(int i = 0; i < 4; ++i)
#pragma unroll
			for(int j = i; j < 4; ++j) {
				float uu = u[i] * u[j];
				p[k++] = i == j ? uu : 2.0f * uu;
			}
	}
	float Gm[4] = {0.0f, 0.0f, 0.0f, 0.0f};
	const float ax = 1.0f - w[0], ay = 1.0f - w[1], az = 1.0f - w[2];
	const bool use0 = g.single || ft < 1.0f;
	const bool use1 = !g.single && ft > 0.0f;
	/* the (corner, level) rows to gather: corner-major, levels in order */
	const int nl = (use0 ? 1 : 0) + (use1 ? 1 : 0);
	const int l0 = use0 ? 0 : 1;
	const int items = 8 * nl;
	auto row_of = [&](int it) {
		const int c = it / nl, l = l0 + it % nl;
		const int ix = (c & 1) ? i1[0] : i0[0];
		const int iy = (c & 2) ? i1[1] : i0[1];
		const int iz = (c & 4) ? i1[2] : i0[2];
		return g.lvl[l] + (((long long)iz * g.ny + iy) * g.nx + ix) * GRAY_NSTRIDE;
	};
	auto issue = [&](int it) {
		const float *src = row_of(it);
		float4 *dst = stage + (it & 1) * STAGE_CHUNKS * CELL_STRIDE;
#pragma unroll
		for(int k = 0; k < STAGE_CHUNKS; ++k)
			cp_async16(dst + k * CELL_STRIDE, src + 4 * k);
		cp_async_commit();
	};
	issue(0);
#pragma unroll 1
	for(int it = 0; it < items; ++it) {
		if(it + 1 < items) {
			issue(it + 1);
			cp_async_wait<1>(); /* row it has landed, row it + 1 in flight */
		} else {
			cp_async_wait<0>();
		}
		const int c = it / nl, l = l0 + it % nl;
		float wl = ((c & 1) ? w[0] : ax) * ((c & 2) ? w[1] : ay) * ((c & 4) ? w[2] : az);
		if(!g.single)
			wl *= l ? ft : 1.0f - ft;
		const float4 *src = stage + (it & 1) * STAGE_CHUNKS * CELL_STRIDE;
		float sm[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
		for(int k = 0; k < STAGE_CHUNKS; ++k) {
			const float4 v = src[k * CELL_STRIDE];
			const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
			for(int q = 0; q < 4; ++q) {
				const int idx = 4 * k + q; /* Gamma^(idx/10)_(idx%10) */
				sm[idx / 10] = fmaf(vv[q], p[idx % 10], sm[idx / 10]);
			}
		}
#pragma unroll
		for(int m = 0; m < 4; ++m)
			Gm[m] = fmaf(wl, sm[m], Gm[m]);
	}
#pragma unroll
	for(int m = 0; m < 4; ++m)
		ds[4 + m] = fmaf(Gm[0], u[m], -Gm[m]);
}

/* NF > 0: the thermal transfer pairs (I, tau) ride along in FP64 (rt[],
 * first the NF intensities, then the NF optical depths), integrated by the
 * same RK4 stages with the FP64 emissivities of thermal.cuh on the FP32
 * momentum and density; the stages run as a rolled loop so that the FP64
 * transfer is instantiated once. */
template <int NF, bool STAGED>
__global__ void __launch_bounds__(256, NF == 0 ? 2 : 1)
dyst_mixed_kernel(const MixedTable T, const GridParams g, const DystConst dc,
                  unsigned int *__restrict__ queue, unsigned long long *__restrict__ steps,
                  unsigned long long *__restrict__ inbox)
{
	static_assert(!STAGED || NF == 0, "staged gathers: geodesic-only renders");
	extern __shared__ float4 s_stage[]; /* STAGED: 2 x STAGE_CHUNKS x CELL_STRIDE */
	float4 *stage = s_stage + threadIdx.x;
	constexpr int ND = 8;            /* FP32 geodesic state           */
	constexpr int NR = 2 * NF;       /* FP64 transfer state           */
	const unsigned FULL = 0xffffffffu;
	const int lane = threadIdx.x & 31;
	/* each thread's last cell per axis (axis_uvw32c); empty to start */
	__shared__ float4 s_cells[3 * CELL_STRIDE];
	float4 *cells = s_cells + threadIdx.x;
#pragma unroll
	for(int a = 0; a < 3; ++a)
		cells[a * CELL_STRIDE] = make_float4(INFINITY, -INFINITY, 0.0f, 0.0f);
	float hi[ND], lo[ND];
	double rt[NR > 0 ? NR : 1];
	long long ray = 0;
	int dump = 0, h = 0, dh_step = 0, n = 0;
	float dtn = 0.0f;
	double dtnd = 0.0; /* the FP64 substep unit of the transfer */
	bool active = false, exhausted = false;
	unsigned long long cnt = 0, cnt_in = 0; /* all steps; steps that interpolate */
	const MixedRender *c = nullptr;

	for(;;) {
		bool need = !active && !exhausted;
		unsigned mask = __ballot_sync(FULL, need);
		if(mask) {
			int leader = __ffs(mask) - 1;
			unsigned base = 0;
			if(lane == leader)
				base = atomicAdd(queue, (unsigned)__popc(mask));
			base = __shfl_sync(FULL, base, leader);
			if(need) {
				unsigned long long gidx = (unsigned long long)base +
				                          __popc(mask & ((1u << lane) - 1));
				if(gidx < T.total) {
					int rr = 0;
					while(rr + 1 < T.n_renders && T.prefix[rr + 1] <= gidx)
						++rr;
					c = &T.renders[rr];
					ray = (long long)(gidx - T.prefix[rr]);
					n = (int)((INT_MAX / c->n_sub) * c->n_sub);
#pragma unroll
					for(int k = 0; k < ND; ++k) {
						double v = c->data[k * c->n_rays + ray];
						hi[k] = (float)v;
						lo[k] = (float)((double)hi[k] - v);
					}
#pragma unroll
					for(int k = 0; k < NR; ++k)
						rt[k] = c->data[(ND + k) * c->n_rays + ray];
					dump = c->dump_begin - 1;
					h = n; /* forces the first dump set-up below */
					active = true;
				} else {
					exhausted = true;
				}
			}
		}
		if(!__any_sync(FULL, active))
			break;
		if(!active)
			continue;
		if(h >= n) { /* next dump interval: constants of driver.cl:93 */
			if(++dump >= c->dump_end) {
				double s[ND];
#pragma unroll
				for(int k = 0; k < ND; ++k) {
					s[k] = (double)hi[k] - (double)lo[k];
					c->data[k * c->n_rays + ray] = s[k];
				}
#pragma unroll
				for(int k = 0; k < NR; ++k)
					c->data[(ND + k) * c->n_rays + ray] = rt[k];
				c->info[ray] = dyst_getuu64(g, s);
				active = false;
				continue;
			}
			double t0 = c->t_init + (double)dump * c->dt_dump;
			double t1 = c->t_init + (double)(dump + 1) * c->dt_dump;
			double dt = t1 - t0;
			dh_step = (int)(dyst_getdt64(dt / (double)c->n_sub) / dt * (double)n);
			dtnd = dt / (double)n;
			dtn = (float)dtnd;
			h = 0;
			if(dh_step <= 0) { /* zero-length interval: nothing to integrate */
				h = n;
				continue;
			}
		}
		int dh = dh_step < n - h ? dh_step : n - h;
		const float hs = (float)dh * dtn, hh = 0.5f * hs;
		float k[ND], t[ND], sum[ND];
		cnt_in += (!g.physics || inside32(g, hi)) ? 1 : 0;
		if constexpr(NF > 0) {
			const double hsd = (double)dh * dtnd;
			double trt[NR], srt[NR], krt[NR];
#pragma unroll
			for(int i = 0; i < ND; ++i)
				t[i] = hi[i];
#pragma unroll
			for(int i = 0; i < NR; ++i)
				trt[i] = rt[i];
#pragma unroll 1
			for(int st = 0; st < 4; ++st) {
				float kn[5];
				dyst_rhs32<true>(g, dc, cells, t, k, kn);
				const double kd[4] = {kn[0], kn[1], kn[2], kn[3]};
				rt_rhs_fast<NF>(c->tf, c->nu_hz, kd, (double)kn[4], trt + NF, krt, krt + NF);
				const float wg = (st == 1 || st == 2) ? 2.0f : 1.0f;
				const float cg = st < 2 ? hh : hs;
				const double wd = wg, cd = st < 2 ? 0.5 * hsd : hsd;
#pragma unroll
				for(int i = 0; i < ND; ++i) { /* k4 stays in k for the update */
					if(st < 3)
						sum[i] = st == 0 ? k[i] : fmaf(wg, k[i], sum[i]);
					t[i] = fmaf(cg, k[i], hi[i]);
				}
#pragma unroll
				for(int i = 0; i < NR; ++i) {
					srt[i] = st == 0 ? krt[i] : fma(wd, krt[i], srt[i]);
					trt[i] = fma(cd, krt[i], rt[i]);
				}
			}
#pragma unroll
			for(int i = 0; i < NR; ++i)
				rt[i] = fma(hsd / 6.0, srt[i], rt[i]);
		} else {
		auto geo = [&](const float *sv, float *kv) {
			if constexpr(STAGED)
				dyst_rhs32_staged(g, dc, cells, stage, sv, kv);
			else
				dyst_rhs32(g, dc, cells, sv, kv);
		};
		geo(hi, k);
#pragma unroll
		for(int i = 0; i < ND; ++i) {
			sum[i] = k[i];
			t[i] = fmaf(hh, k[i], hi[i]);
		}
		geo(t, k);
#pragma unroll
		for(int i = 0; i < ND; ++i) {
			sum[i] = fmaf(2.0f, k[i], sum[i]);
			t[i] = fmaf(hh, k[i], hi[i]);
		}
		geo(t, k);
#pragma unroll
		for(int i = 0; i < ND; ++i) {
			sum[i] = fmaf(2.0f, k[i], sum[i]);
			t[i] = fmaf(hs, k[i], hi[i]);
		}
		geo(t, k);
		}
		const float h6 = hs * (1.0f / 6.0f);
		bool bad = false;
#pragma unroll
		for(int i = 0; i < ND; ++i) {
			float inc = h6 * (sum[i] + k[i]);
			float yv = inc - lo[i];
			float tv = hi[i] + yv;
			lo[i] = (tv - hi[i]) - yv;
			hi[i] = tv;
			bad |= !(fabsf(tv) <= FLT_MAX);
		}
		++cnt;
		h += dh;
		if(bad) { /* NaN/Inf (inside the singular region): ray done */
			double s[ND];
#pragma unroll
			for(int kk = 0; kk < ND; ++kk) {
				s[kk] = (double)hi[kk] - (double)lo[kk];
				c->data[kk * c->n_rays + ray] = s[kk];
			}
#pragma unroll
			for(int kk = 0; kk < NR; ++kk)
				c->data[(ND + kk) * c->n_rays + ray] = rt[kk];
			c->info[ray] = s[0] - s[0]; /* NaN marks the ray */
			active = false;
		}
	}
#pragma unroll
	for(int o = 16; o > 0; o >>= 1) {
		cnt += __shfl_xor_sync(FULL, cnt, o);
		cnt_in += __shfl_xor_sync(FULL, cnt_in, o);
	}
	if(lane == 0 && cnt)
		atomicAdd(steps, cnt);
	if(lane == 0 && cnt_in && inbox)
		atomicAdd(inbox, cnt_in);
}

template <int NF, bool STAGED>
cudaError_t
launch_dyst_nfs(const MixedTable &T, const GridParams &g, const DystConst &dc,
                unsigned int *queue, unsigned long long *steps, cudaStream_t st,
                const MixedLaunch &cfg, unsigned long long *inbox)
{
	int block = cfg.block > 0 ? cfg.block : 256;
	if(block > 256)
		return cudaErrorInvalidValue; /* __launch_bounds__(256) */
	/* the stage is indexed with the CELL_STRIDE of the launch bound */
	const size_t smem = STAGED ? 2 * STAGE_CHUNKS * CELL_STRIDE * sizeof(float4) : 0;
	cudaError_t e = cudaSuccess;
	if(STAGED)
		e = cudaFuncSetAttribute(dyst_mixed_kernel<NF, STAGED>,
		                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	if(e != cudaSuccess)
		return e;
	int per_sm = cfg.blocks_per_sm;
	if(per_sm <= 0) {
		e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dyst_mixed_kernel<NF, STAGED>,
		                                                  block, smem);
		if(e != cudaSuccess)
			return e;
		if(per_sm <= 0)
			per_sm = 1;
	}
	long long want = (long long)per_sm * (cfg.sms > 0 ? cfg.sms : 148);
	long long need = (long long)((T.total + block - 1) / block);
	unsigned grid = (unsigned)(want < need ? want : need);
	if(grid == 0)
		grid = 1;
	dyst_mixed_kernel<NF, STAGED><<<grid, block, smem, st>>>(T, g, dc, queue, steps, inbox);
	return cudaGetLastError();
}

#ifndef GRAY_DYST_STAGED
#define GRAY_DYST_STAGED 0
#endif

template <int NF>
cudaError_t
launch_dyst_nf(const MixedTable &T, const GridParams &g, const DystConst &dc,
               unsigned int *queue, unsigned long long *steps, cudaStream_t st,
               const MixedLaunch &cfg, unsigned long long *inbox)
{
	if constexpr(NF == 0)
		if(GRAY_DYST_STAGED)
			return launch_dyst_nfs<0, true>(T, g, dc, queue, steps, st, cfg, inbox);
	return launch_dyst_nfs<NF, false>(T, g, dc, queue, steps, st, cfg, inbox);
}

} /* namespace */

cudaError_t
launch_dyst_mixed_table(const MixedTable &T, const GridParams &g, int n_freq,
                        unsigned int *queue, unsigned long long *steps, cudaStream_t st,
                        const MixedLaunch &cfg, unsigned long long *inbox)
{
	static_assert(GRAY_MAX_FREQ == 8, "one instantiation per frequency count");
	DystConst dc;
	for(int a = 0; a < 3; ++a) {
		dc.B[a] = (float)g.B[a];
		dc.iA[a] = (float)(1.0 / g.A[a]);
	}
	if(n_freq < 0 || n_freq > GRAY_MAX_FREQ)
		return cudaErrorInvalidValue;
	cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned int), st);
	if(e != cudaSuccess)
		return e;
	switch(n_freq) {
	case 0: return launch_dyst_nf<0>(T, g, dc, queue, steps, st, cfg, inbox);
	case 1: return launch_dyst_nf<1>(T, g, dc, queue, steps, st, cfg, inbox);
	case 2: return launch_dyst_nf<2>(T, g, dc, queue, steps, st, cfg, inbox);
	case 3: return launch_dyst_nf<3>(T, g, dc, queue, steps, st, cfg, inbox);
	case 4: return launch_dyst_nf<4>(T, g, dc, queue, steps, st, cfg, inbox);
	case 5: return launch_dyst_nf<5>(T, g, dc, queue, steps, st, cfg, inbox);
	case 6: return launch_dyst_nf<6>(T, g, dc, queue, steps, st, cfg, inbox);
	case 7: return launch_dyst_nf<7>(T, g, dc, queue, steps, st, cfg, inbox);
	default: return launch_dyst_nf<8>(T, g, dc, queue, steps, st, cfg, inbox);
	}
}

