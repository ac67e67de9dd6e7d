/*
 * Mixed-precision persistent geodesic kernel (analytic Kerr-Schild + torus
 * transfer).  One launch integrates every dump interval of every ray of
 * one or many renders:
 *
 *  - persistent warps pull rays from a global queue; a warp ballot finds the
 *    lanes whose ray terminated (horizon capture, or all dumps done) and
 *    refills exactly those lanes, so captured rays do not idle SIMD lanes
 *    while their neighbours keep integrating;
 *  - the RHS (KS.cl:263-378), RK4 stages (RK4.cl:37-47) and transfer
 *    (rt.cl:185-198 form with the analytic torus) run in FP32, using the
 *    approximate rcp/rsqrt/ex2/lg2 instructions instead of IEEE divide and
 *    square-root sequences;
 *  - FP64 is kept where it matters: the state update is compensated (Kahan:
 *    hi + lo pairs of FP32), the Kerr-Schild radius root (KS.cl:48-55) is
 *    evaluated in FP64 near the horizon where the stop rule and step-size
 *    rule (phys.cl:48-64) read it, and the null-constraint diagnostic
 *    (KS.cl:164-168) is computed in FP64 from the final state;
 *  - the integer-tick substep loop of driver.cl:81-99 is kept, so dump
 *    boundaries are hit exactly as in the FP64 kernel.
 */
#include <climits>

#include "gray_internal.h"
#include "mixed_table.h"

namespace {

__device__ __forceinline__ float
rcp_a(float x)
{
	float r;
	asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
	return r;
}

__device__ __forceinline__ float
rsqrt_a(float x)
{
	float r;
	asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
	return r;
}

__device__ __forceinline__ float
sqrt_a(float x)
{
	float r;
	asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
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

struct Aux32 {
	float r, ir, f, lx, ly, lz, flu, iss;
};

/* KS.cl:263-378 in FP32: the same Chan et al. grouping, with the five
 * divides and two square roots folded into 2 rsqrt + 2 rcp. */
__device__ __forceinline__ void
ks_rhs32(const MixedRender &c, const float *s, float *ds, Aux32 &aux)
{
	const float a = c.a, aa = c.aa;
	const float x = s[1], y = s[2], z = s[3];
	const float ut = s[4], ux = s[5], uy = s[6], uz = s[7];

	float f, dx_f, dy_f, dz_f;
	float lx, dx_lx, dy_lx, dz_lx;
	float ly, dx_ly, dy_ly, dz_ly;
	float lz, dx_lz, dy_lz, dz_lz;
	float dx_r, dy_r, dz_r, r, ir, iss, tmp;
	{
		float zz  = z * z;
		float kk  = 0.5f * (fmaf(x, x, fmaf(y, y, zz)) - aa);
		float d2  = fmaf(kk, kk, aa * zz);
		float idd = rsqrt_a(d2);
		float dd  = d2 * idd;
		float rr  = dd + kk;
		ir  = rsqrt_a(rr);
		r   = rr * ir;
		float ss = rr + aa;
		iss  = rcp_a(ss);
		tmp  = 0.5f * ir * idd;
		dz_r = tmp * ss * z;
		tmp  = tmp * rr;
		dy_r = tmp * y;
		dx_r = tmp * x;
		tmp  = 2.0f * rr * rcp_a(fmaf(rr, rr, aa * zz));
		float tmp2 = fmaf(-2.0f * rr, tmp, 3.0f);
		f    = tmp * r;
		dx_f = tmp * dx_r * tmp2;
		dy_f = tmp * dy_r * tmp2;
		dz_f = tmp * fmaf(dz_r, tmp2, -(tmp * aa * z * ir));
	}
	{
		float m2r  = -2.0f * r;
		float issr = iss * r;
		float issa = iss * a;

		lx    = iss * fmaf(x, r, y * a);
		tmp   = iss * fmaf(m2r, lx, x);
		dx_lx = fmaf(tmp, dx_r, issr);
		dy_lx = fmaf(tmp, dy_r, issa);
		dz_lx = tmp * dz_r;

		ly    = iss * fmaf(y, r, -(x * a));
		tmp   = iss * fmaf(m2r, ly, y);
		dx_ly = fmaf(tmp, dx_r, -issa);
		dy_ly = fmaf(tmp, dy_r, issr);
		dz_ly = tmp * dz_r;

		lz    = z * ir;
		tmp   = -lz * ir;
		dx_lz = tmp * dx_r;
		dy_lz = tmp * dy_r;
		dz_lz = fmaf(tmp, dz_r, ir);
	}
	float lu  = fmaf(lz, uz, fmaf(ly, uy, fmaf(lx, ux, ut)));
	float flu = f * lu;
	float Dx0 = fmaf(dx_f, lu, f * fmaf(dx_lz, uz, fmaf(dx_ly, uy, dx_lx * ux)));
	float Dy0 = fmaf(dy_f, lu, f * fmaf(dy_lz, uz, fmaf(dy_ly, uy, dy_lx * ux)));
	float Dz0 = fmaf(dz_f, lu, f * fmaf(dz_lz, uz, fmaf(dz_ly, uy, dz_lx * ux)));

	float Dx1 = fmaf(Dx0, lx, flu * dx_lx);
	float Dx2 = fmaf(Dx0, ly, flu * dx_ly);
	float Dx3 = fmaf(Dx0, lz, flu * dx_lz);
	float Dy1 = fmaf(Dy0, lx, flu * dy_lx);
	float Dy2 = fmaf(Dy0, ly, flu * dy_ly);
	float Dy3 = fmaf(Dy0, lz, flu * dy_lz);
	float Dz1 = fmaf(Dz0, lx, flu * dz_lx);
	float Dz2 = fmaf(Dz0, ly, flu * dz_ly);
	float Dz3 = fmaf(Dz0, lz, flu * dz_lz);

	float hDxu = 0.5f * fmaf(Dx3, uz, fmaf(Dx2, uy, fmaf(Dx1, ux, Dx0 * ut)));
	float hDyu = 0.5f * fmaf(Dy3, uz, fmaf(Dy2, uy, fmaf(Dy1, ux, Dy0 * ut)));
	float hDzu = 0.5f * fmaf(Dz3, uz, fmaf(Dz2, uy, fmaf(Dz1, ux, Dz0 * ut)));

	float uD0 = fmaf(uz, Dz0, fmaf(uy, Dy0, ux * Dx0));
	float uD1 = fmaf(uz, Dz1, fmaf(uy, Dy1, ux * Dx1));
	float uD2 = fmaf(uz, Dz2, fmaf(uy, Dy2, ux * Dx2));
	float uD3 = fmaf(uz, Dz3, fmaf(uy, Dy3, ux * Dx3));

	tmp = f * fmaf(lz, uD3 - hDzu, fmaf(ly, uD2 - hDyu, fmaf(lx, uD1 - hDxu, -uD0)));

	ds[0] = ut;
	ds[1] = ux;
	ds[2] = uy;
	ds[3] = uz;
	ds[4] = uD0 - tmp;
	ds[5] = fmaf(lx, tmp, hDxu - uD1);
	ds[6] = fmaf(ly, tmp, hDyu - uD2);
	ds[7] = fmaf(lz, tmp, hDzu - uD3);

	aux.r = r; aux.ir = ir; aux.f = f; aux.lx = lx; aux.ly = ly; aux.lz = lz;
	aux.flu = flu; aux.iss = iss;
}

/* Torus flow + transfer in FP32 (same model as the FP64 kernel). */
template <int NF>
__device__ __forceinline__ void
torus_rt32(const MixedRender &c, const float *s, const Aux32 &x, float *ds)
{
	constexpr float LOG2E = 1.4426950408889634f;
	float n = 0.0f, shift = 1.0f;
	if(x.r > c.risco) {
		const float q1 = s[1], q2 = s[2], q3 = s[3];
		float kt = x.flu - s[4];
		float kx = fmaf(x.flu, x.lx, s[5]);
		float ky = fmaf(x.flu, x.ly, s[6]);
		float R2 = fmaf(q1, q1, q2 * q2);
		float irs = rsqrt_a(x.r);           /* r^-1/2 */
		float sr  = x.r * irs;              /* r^1/2  */
		float Om  = rcp_a(fmaf(x.r, sr, c.a));
		float vv  = fmaf(Om * Om, R2, -1.0f);
		float lv  = fmaf(-(c.a * Om * R2), x.iss, 1.0f);
		float D   = -fmaf(x.f * lv, lv, vv);
		if(D > 0.0f) {
			float utf = rsqrt_a(D);
			shift = -utf * fmaf(Om, fmaf(q1, ky, -(q2 * kx)), kt);
			if(shift > 0.0f) {
				/* n0 (r_+/r)^1.5 exp(-z^2 / (2 (h r)^2)) */
				float e = ex2_a(-(q3 * q3) * (x.ir * x.ir) * c.ihr2_log2e);
				n = c.n0_rp15 * (x.ir * irs) * e;
			}
		}
	}
	if(n == 0.0f) {
#pragma unroll
		for(int i = 0; i < 2 * NF; ++i)
			ds[8 + i] = 0.0f;
		return;
	}
	float ish  = rcp_a(shift);
	float jfac = n * ex2_a(-0.7f * lg2_a(shift));
	float tfac = c.kappa * n * ish;
	float is2  = ish * ish;
#pragma unroll
	for(int i = 0; i < NF; ++i) {
		float j = jfac * c.nupow[i];
		ds[8 + i]      = -(j * ex2_a(-s[8 + NF + i] * LOG2E)) * is2;
		ds[8 + NF + i] = -(tfac * c.nuinv2[i]);
	}
}

template <int NF>
__device__ __forceinline__ void
rhs32(const MixedRender &c, const float *s, float *ds)
{
	Aux32 aux;
	ks_rhs32(c, s, ds, aux);
	if(NF > 0) {
		if(c.flow == GRAY_FLOW_TORUS) {
			torus_rt32<NF>(c, s, aux, ds);
		} else {
#pragma unroll
			for(int i = 0; i < 2 * NF; ++i)
				ds[8 + i] = 0.0f;
		}
	}
}

/* FP64 radius root (KS.cl:48-55) for the near-horizon island */
__device__ __forceinline__ double
getrr_d(double aa, double x, double y, double z)
{
	double zz = z * z;
	double kk = 0.5 * (fma(x, x, fma(y, y, zz)) - aa);
	return sqrt(fma(kk, kk, aa * zz)) + kk;
}

/* FP64 null-constraint check from the final state (KS.cl:164-168) */
__device__ __forceinline__ double
getuu_d(double a, const double *s)
{
	double aa = a * a;
	double zz = s[3] * s[3];
	double kk = 0.5 * (fma(s[1], s[1], fma(s[2], s[2], zz)) - aa);
	double rr = sqrt(fma(kk, kk, aa * zz)) + kk;
	double r  = sqrt(rr);
	double f  = 2.0 * rr * r / fma(rr, rr, aa * zz);
	double iss = 1.0 / (rr + aa);
	double lx = iss * fma(s[1], r, s[2] * a);
	double ly = iss * fma(s[2], r, -(s[1] * a));
	double lz = s[3] / r;
	double lu = fma(lz, s[7], fma(ly, s[6], fma(lx, s[5], s[4])));
	double flu = f * lu;
	double k0 = flu - s[4];
	double k1 = fma(flu, lx, s[5]);
	double k2 = fma(flu, ly, s[6]);
	double k3 = fma(flu, lz, s[7]);
	return fma(k3, s[7], fma(k2, s[6], fma(k1, s[5], k0 * s[4])));
}

/* Per-lane state of the ray being integrated. */
template <int ND>
struct Lane {
	float hi[ND], lo[ND]; /* compensated state: value = hi - lo          */
	int   render;         /* index into the render table                 */
	long long ray;        /* ray index within its render                 */
	int   dump;           /* current dump interval                       */
	int   h;              /* ticks done in this interval                 */
	int   dh_cap;         /* ticks of a capped step (|dt| / n_sub)       */
	float cdt;            /* n / |dt|: ticks per unit affine length      */
	float dtn;            /* dt / n: affine length of one tick (signed)  */
};

/* Per-dump constants, computed in FP64 exactly like the host loop of
 * sim-org/gray.c:251-252 and driver.cl:93. */
template <int ND>
__device__ __forceinline__ void
start_dump(const MixedRender &c, Lane<ND> &L, int n)
{
	double t      = c.t_init + (double)L.dump * c.dt_dump;
	double target = c.t_init + (double)(L.dump + 1) * c.dt_dump;
	double dt     = target - t;
	double dts    = dt / (double)c.n_sub;
	L.dh_cap = (int)(dts / dt * (double)n);
	L.cdt    = (float)((double)n / fabs(dt));
	L.dtn    = (float)(dt / (double)n);
	L.h      = 0;
}

template <int ND>
__device__ __forceinline__ void
load_ray(const MixedRender &c, Lane<ND> &L, int n)
{
	const long long nr = c.n_rays;
#pragma unroll
	for(int k = 0; k < ND; ++k) {
		double v = c.data[k * nr + L.ray];
		float hi = (float)v;
		L.hi[k] = hi;
		L.lo[k] = (float)((double)hi - v);
	}
	L.dump = 0;
	start_dump(c, L, n);
}

template <int ND>
__device__ __forceinline__ void
store_ray(const MixedRender &c, const Lane<ND> &L)
{
	const long long nr = c.n_rays;
	double s[ND];
#pragma unroll
	for(int k = 0; k < ND; ++k) {
		s[k] = (double)L.hi[k] - (double)L.lo[k];
		c.data[k * nr + L.ray] = s[k];
	}
	c.info[L.ray] = getuu_d(c.a_d, s);
}

/* Map a global queue index to (render, ray) by binary search over the
 * prefix sums of the render sizes. */
__device__ __forceinline__ int
find_render(const MixedTable &T, unsigned long long g)
{
	int lo = 0, hi = T.n_renders - 1;
	while(lo < hi) {
		int mid = (lo + hi + 1) >> 1;
		if(T.prefix[mid] <= g)
			lo = mid;
		else
			hi = mid - 1;
	}
	return lo;
}

template <int NF>
__global__ void __launch_bounds__(256)
mixed_kernel(const MixedTable T, unsigned int *__restrict__ queue,
             unsigned long long *__restrict__ steps)
{
	constexpr int ND = 8 + 2 * NF;
	const unsigned FULL = 0xffffffffu;
	const int lane = threadIdx.x & 31;

	Lane<ND> L;
	bool active = false, exhausted = false;
	unsigned long long cnt = 0;
	const MixedRender *c = nullptr;
	int n = 0;

	for(;;) {
		/* refill the lanes whose ray finished (warp-ballot compaction) */
		bool need = !active && !exhausted;
		unsigned mask = __ballot_sync(FULL, need);
		if(mask) {
			int leader = __ffs(mask) - 1;
			unsigned base = 0;
			if(lane == leader)
				base = atomicAdd(queue, (unsigned)__popc(mask));
			base = __shfl_sync(FULL, base, leader);
			if(need) {
				unsigned long long g = (unsigned long long)base +
				                       __popc(mask & ((1u << lane) - 1));
				if(g < T.total) {
					L.render = find_render(T, g);
					c = &T.renders[L.render];
					L.ray = (long long)(g - T.prefix[L.render]);
					n = (int)((INT_MAX / c->n_sub) * c->n_sub);
					load_ray(*c, L, n);
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

		/* step control: phys.cl:48-64 with the FP64 island near r_+ */
		float rr32 = 0.0f;
		{
			float zz = L.hi[3] * L.hi[3];
			float kk = 0.5f * (fmaf(L.hi[1], L.hi[1], fmaf(L.hi[2], L.hi[2], zz)) - c->aa);
			rr32 = sqrt_a(fmaf(kk, kk, c->aa * zz)) + kk;
		}
		float eps = sqrt_a(rr32) - c->rp;
		if(eps < 1.0f) {
			double x = (double)L.hi[1] - (double)L.lo[1];
			double y = (double)L.hi[2] - (double)L.lo[2];
			double z = (double)L.hi[3] - (double)L.lo[3];
			eps = (float)(sqrt(getrr_d(c->aa_d, x, y, z)) - c->rp_d);
		}
		int dh;
		if(!(eps >= c->eps_stop)) { /* captured (or NaN): ray done */
			dh = 0;
		} else {
			float want = c->cdt_scale * eps * eps * L.cdt; /* 0.01 eps^2 n / |dt| */
			dh = want < (float)L.dh_cap ? (int)want : L.dh_cap;
		}
		if(dh == 0) {
			store_ray(*c, L);
			active = false;
			continue;
		}
		if(dh > n - L.h)
			dh = n - L.h;

		/* RK4.cl:37-47 with the compensated update */
		{
			const float hs  = (float)dh * L.dtn;
			const float hh  = 0.5f * hs;
			float k[ND], t[ND], sum[ND];
			rhs32<NF>(*c, L.hi, k);
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				sum[i] = k[i];
				t[i] = fmaf(hh, k[i], L.hi[i]);
			}
			rhs32<NF>(*c, t, k);
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				sum[i] = fmaf(2.0f, k[i], sum[i]);
				t[i] = fmaf(hh, k[i], L.hi[i]);
			}
			rhs32<NF>(*c, t, k);
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				sum[i] = fmaf(2.0f, k[i], sum[i]);
				t[i] = fmaf(hs, k[i], L.hi[i]);
			}
			rhs32<NF>(*c, t, k);
			const float h6 = hs * (1.0f / 6.0f);
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				float inc = h6 * (sum[i] + k[i]);
				/* Kahan: value = hi - lo */
				float yv = inc - L.lo[i];
				float tv = L.hi[i] + yv;
				L.lo[i] = (tv - L.hi[i]) - yv;
				L.hi[i] = tv;
			}
		}
		++cnt;
		L.h += dh;
		if(L.h >= n) {
			if(++L.dump >= c->n_dump) {
				store_ray(*c, L);
				active = false;
			} else {
				start_dump(*c, L, n);
			}
		}
	}

#pragma unroll
	for(int o = 16; o > 0; o >>= 1)
		cnt += __shfl_xor_sync(FULL, cnt, o);
	if(lane == 0 && cnt)
		atomicAdd(steps, cnt);
}

template <int NF>
cudaError_t
launch_nf(const MixedTable &T, unsigned int *queue, unsigned long long *steps,
          cudaStream_t st, const MixedLaunch &cfg)
{
	int block = cfg.block > 0 ? cfg.block : 256;
	int per_sm = cfg.blocks_per_sm;
	if(per_sm <= 0) {
		cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
			&per_sm, mixed_kernel<NF>, block, 0);
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
	mixed_kernel<NF><<<grid, block, 0, st>>>(T, queue, steps);
	return cudaGetLastError();
}

} /* namespace */

cudaError_t
launch_mixed_table(const MixedTable &T, int n_freq, unsigned int *queue,
                   unsigned long long *steps, cudaStream_t st, const MixedLaunch &cfg)
{
	cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned int), st);
	if(e != cudaSuccess)
		return e;
	switch(n_freq) {
	case 0: return launch_nf<0>(T, queue, steps, st, cfg);
	case 1: return launch_nf<1>(T, queue, steps, st, cfg);
	case 2: return launch_nf<2>(T, queue, steps, st, cfg);
	case 3: return launch_nf<3>(T, queue, steps, st, cfg);
	case 4: return launch_nf<4>(T, queue, steps, st, cfg);
	case 5: return launch_nf<5>(T, queue, steps, st, cfg);
	case 6: return launch_nf<6>(T, queue, steps, st, cfg);
	case 7: return launch_nf<7>(T, queue, steps, st, cfg);
	case 8: return launch_nf<8>(T, queue, steps, st, cfg);
	default: return cudaErrorInvalidValue;
	}
}

void
fill_mixed_render(const RenderParams &p, double *data, double *info, double t_init,
                  double dt_dump, long long n_dump, long long n_sub, MixedRender *m)
{
	m->a = (float)p.a;
	m->aa = (float)p.aa;
	m->rp = (float)p.rp;
	m->risco = (float)p.risco;
	m->eps_stop = (float)p.eps_stop;
	m->cdt_scale = 0.01f;
	m->kappa = (float)p.torus_kappa;
	/* n0 r_+^1.5 and log2(e) / (2 h^2) */
	m->n0_rp15 = (float)(p.torus_n0 * p.rp * sqrt(p.rp));
	m->ihr2_log2e = (float)(1.4426950408889634 / (2.0 * p.torus_hr * p.torus_hr));
	for(int i = 0; i < GRAY_MAX_FREQ; ++i) {
		m->nupow[i] = p.nupow_f[i];
		m->nuinv2[i] = p.nuinv2_f[i];
	}
	m->flow = p.flow;
	m->a_d = p.a;
	m->aa_d = p.aa;
	m->rp_d = p.rp;
	m->data = data;
	m->info = info;
	m->n_rays = p.n_rays;
	m->t_init = t_init;
	m->dt_dump = dt_dump;
	m->n_dump = (int)n_dump;
	m->n_sub = n_sub;
}
