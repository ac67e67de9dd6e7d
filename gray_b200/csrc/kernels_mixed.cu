/*
 * Mixed-precision persistent geodesic kernel (analytic Kerr-Schild + torus
 * transfer).  One launch integrates a window of dump intervals of every ray
 * of one or many renders:
 *
 *  - persistent warps pull rays from a global queue; a warp ballot finds the
 *    lanes whose ray terminated (horizon capture, or its dump window done)
 *    and refills exactly those lanes, so captured rays do not idle SIMD
 *    lanes while their neighbours keep integrating;
 *  - the RHS (KS.cl:263-378), RK4 stages (RK4.cl:37-47) and transfer
 *    (rt.cl:185-198 form with the analytic torus) run in FP32 with the
 *    approximate rcp/rsqrt/ex2/lg2 instructions in place of IEEE divide and
 *    square-root sequences; with two rays per thread the whole step runs in
 *    sm_100 packed f32x2 arithmetic (one FFMA2/FMUL2/FADD2 issue slot serves
 *    both rays), and with one ray per thread the RK4 stage sums, stage
 *    states and compensated update run on pairs of state components in
 *    the same packed arithmetic;
 *  - FP64 is kept where it matters: the state update is compensated (Kahan
 *    hi + lo pairs of FP32), the Kerr-Schild radius root (KS.cl:48-55) is
 *    evaluated in FP64 near the horizon where the stop rule and step-size
 *    rule (phys.cl:48-64) read it, and the null-constraint diagnostic
 *    (KS.cl:164-168) is computed in FP64 from the final state;
 *  - the integer-tick substep loop of driver.cl:81-99 is kept, so dump
 *    boundaries are hit exactly as in the FP64 kernel;
 *  - each ray's render constants live in registers (loaded when the ray is
 *    loaded), not re-read from the table every RHS.
 */
#include <climits>

#include "gray_internal.h"
#include "logk2_table.h"
#include "mixed_table.h"

namespace {

/* ---------------------------------------------------------- scalar MUFU */

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

/* ------------------------------------------- lane types: float and f32x2 */

struct F2 {
	float2 v;
};
struct M2 {
	bool x, y;
};

__device__ __forceinline__ F2 mk2(float a, float b) { F2 r; r.v = make_float2(a, b); return r; }

template <typename V> __device__ __forceinline__ V bc(float c);
template <> __device__ __forceinline__ float bc<float>(float c) { return c; }
template <> __device__ __forceinline__ F2 bc<F2>(float c) { return mk2(c, c); }

__device__ __forceinline__ F2 operator+(F2 a, F2 b) { F2 r; r.v = __fadd2_rn(a.v, b.v); return r; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { F2 r; r.v = __fmul2_rn(a.v, b.v); return r; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b)
{
	F2 r;
	r.v = __ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v);
	return r;
}
__device__ __forceinline__ F2 operator-(F2 a) { F2 r; r.v = __fmul2_rn(a.v, make_float2(-1.0f, -1.0f)); return r; }

/* a - b in one packed instruction (there is no __fsub2_rn intrinsic) */
__device__ __forceinline__ float2
sub2(float2 a, float2 b)
{
	float2 r;
	asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
	    "mov.b64 ra, {%2, %3};\n\t"
	    "mov.b64 rb, {%4, %5};\n\t"
	    "sub.rn.f32x2 rd, ra, rb;\n\t"
	    "mov.b64 {%0, %1}, rd;\n\t}"
	    : "=f"(r.x), "=f"(r.y)
	    : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
	return r;
}

__device__ __forceinline__ float fmav(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ F2 fmav(F2 a, F2 b, F2 c) { F2 r; r.v = __ffma2_rn(a.v, b.v, c.v); return r; }

#define LANEWISE(name, f)                                                       \
	__device__ __forceinline__ float name(float a) { return f(a); }             \
	__device__ __forceinline__ F2 name(F2 a) { return mk2(f(a.v.x), f(a.v.y)); }
LANEWISE(rcpv, rcp_a)
LANEWISE(rsqv, rsqrt_a)
LANEWISE(ex2v, ex2_a)
LANEWISE(lg2v, lg2_a)
#undef LANEWISE

__device__ __forceinline__ bool gtv(float a, float b) { return a > b; }
__device__ __forceinline__ M2 gtv(F2 a, F2 b) { M2 m = {a.v.x > b.v.x, a.v.y > b.v.y}; return m; }
__device__ __forceinline__ bool andv(bool a, bool b) { return a && b; }
__device__ __forceinline__ M2 andv(M2 a, M2 b) { M2 m = {a.x && b.x, a.y && b.y}; return m; }
__device__ __forceinline__ float selv(bool m, float a, float b) { return m ? a : b; }
__device__ __forceinline__ F2 selv(M2 m, F2 a, F2 b) { return mk2(m.x ? a.v.x : b.v.x, m.y ? a.v.y : b.v.y); }

template <typename V> struct MaskOf;
template <> struct MaskOf<float> { typedef bool T; };
template <> struct MaskOf<F2> { typedef M2 T; };

/* lane k of a V (k is a compile-time constant after unrolling) */
__device__ __forceinline__ float getl(float a, int) { return a; }
__device__ __forceinline__ float getl(F2 a, int k) { return k ? a.v.y : a.v.x; }
__device__ __forceinline__ void setl(float &a, int, float x) { a = x; }
__device__ __forceinline__ void setl(F2 &a, int k, float x)
{
	if(k)
		a.v.y = x;
	else
		a.v.x = x;
}

template <typename V> struct Lanes;
template <> struct Lanes<float> { static constexpr int N = 1; };
template <> struct Lanes<F2> { static constexpr int N = 2; };

/* ------------------------------------------------ per-ray render constants */

template <typename V, int NF>
struct RC {
	V a, aa, risco, kappa, n0t, ihr2;
	V lgnupow[NF > 0 ? NF : 1], nuinv2[NF > 0 ? NF : 1];
};

template <typename V, int NF>
__device__ __forceinline__ void
load_rc(RC<V, NF> &rc, int k, const MixedRender &c)
{
	setl(rc.a, k, c.a);
	setl(rc.aa, k, c.aa);
	setl(rc.risco, k, c.risco);
	setl(rc.kappa, k, c.kappa);
	/* the density scale, zero without the torus flow */
	setl(rc.n0t, k, c.flow == GRAY_FLOW_TORUS ? c.n0_rp15 : 0.0f);
	setl(rc.ihr2, k, c.ihr2_log2e);
#pragma unroll
	for(int i = 0; i < NF; ++i) {
		setl(rc.lgnupow[i], k, log2f(c.nupow[i])); /* nu_i^-0.7 as a power of 2 */
		setl(rc.nuinv2[i], k, c.nuinv2[i]);
	}
}

/* -------------------------------------------------------------- the RHS */

template <typename V>
struct Aux {
	V r, ir, f, lx, ly, lz, flu, iss, R2;
};

/* KS.cl:263-378 in FP32: the Chan et al. grouping, with the five divides
 * and two square roots folded into 2 rsqrt + 2 rcp. */
template <typename V, int NF>
__device__ __forceinline__ void
ks_rhs(const RC<V, NF> &c, const V *s, V *ds, Aux<V> &aux)
{
	const V a = c.a, aa = c.aa;
	const V x = s[1], y = s[2], z = s[3];
	const V ut = s[4], ux = s[5], uy = s[6], uz = s[7];
	const V half = bc<V>(0.5f), one = bc<V>(1.0f), two = bc<V>(2.0f);

	V f, dx_f, dy_f, dz_f;
	V lx, dx_lx, dy_lx, dz_lx;
	V ly, dx_ly, dy_ly, dz_ly;
	V lz, dx_lz, dy_lz, dz_lz;
	V dx_r, dy_r, dz_r, r, ir, iss, tmp, R2;
	{
		V zz  = z * z;
		V azz = aa * zz;
		R2       = fmav(x, x, y * y); /* also the torus's cylindrical radius */
		V kk  = half * ((R2 + zz) - aa);
		V d2  = fmav(kk, kk, azz);
		V idd = rsqv(d2);
		V rr  = fmav(d2, idd, kk);    /* sqrt(d2) + kk */
		ir  = rsqv(rr);
		r   = rr * ir;
		V ss = rr + aa;
		iss  = rcpv(ss);
		tmp  = half * (ir * idd);
		dz_r = (tmp * ss) * z;
		tmp  = tmp * rr;
		dy_r = tmp * y;
		dx_r = tmp * x;
		tmp  = (two * rr) * rcpv(fmav(rr, rr, azz));
		V tmp2 = fmav(-(two * rr), tmp, bc<V>(3.0f));
		f    = tmp * r;
		V tt2 = tmp * tmp2;
		dx_f = tt2 * dx_r;
		dy_f = tt2 * dy_r;
		dz_f = fmav(tt2, dz_r, -((tmp * tmp) * (aa * (z * ir))));
	}
	{
		V m2r  = -(two * r);
		V issr = iss * r;
		V issa = iss * a;

		lx    = iss * fmav(x, r, y * a);
		tmp   = iss * fmav(m2r, lx, x);
		dx_lx = fmav(tmp, dx_r, issr);
		dy_lx = fmav(tmp, dy_r, issa);
		dz_lx = tmp * dz_r;

		ly    = iss * fmav(y, r, -(x * a));
		tmp   = iss * fmav(m2r, ly, y);
		dx_ly = fmav(tmp, dx_r, -issa);
		dy_ly = fmav(tmp, dy_r, issr);
		dz_ly = tmp * dz_r;

		lz    = z * ir;
		tmp   = -(lz * ir);
		dx_lz = tmp * dx_r;
		dy_lz = tmp * dy_r;
		dz_lz = fmav(tmp, dz_r, ir);
	}
	V lu  = fmav(lz, uz, fmav(ly, uy, fmav(lx, ux, ut)));
	V flu = f * lu;
	/* KS.cl:340-363 form the covector derivatives D_a = d_a(f l.u l) (a =
	 * x, y, z) component by component and contract them twice.  With
	 * D_a^0 = d_a f (l.u) + f (d_a l . u) and D_a^i = D_a^0 l^i + f l.u d_a l^i
	 * the two contractions are, exactly,
	 *   hD_a u = (D_a^0 l.u + f l.u (d_a l . u)) / 2
	 *   uD^i   = uD^0 l^i + f l.u (u . grad) l^i,
	 * which skips the nine D_a^i (same mathematics, fewer operations). */
	V Lx = fmav(dx_lz, uz, fmav(dx_ly, uy, dx_lx * ux)); /* d_x l . u */
	V Ly = fmav(dy_lz, uz, fmav(dy_ly, uy, dy_lx * ux));
	V Lz = fmav(dz_lz, uz, fmav(dz_ly, uy, dz_lx * ux));
	V Dx0 = fmav(dx_f, lu, f * Lx);
	V Dy0 = fmav(dy_f, lu, f * Ly);
	V Dz0 = fmav(dz_f, lu, f * Lz);
	V hlu = half * lu, hflu = half * flu;
	V hDxu = fmav(Dx0, hlu, hflu * Lx);
	V hDyu = fmav(Dy0, hlu, hflu * Ly);
	V hDzu = fmav(Dz0, hlu, hflu * Lz);
	V uD0 = fmav(uz, Dz0, fmav(uy, Dy0, ux * Dx0));
	V Mx  = fmav(uz, dz_lx, fmav(uy, dy_lx, ux * dx_lx)); /* (u . grad) l */
	V My  = fmav(uz, dz_ly, fmav(uy, dy_ly, ux * dx_ly));
	V Mz  = fmav(uz, dz_lz, fmav(uy, dy_lz, ux * dx_lz));
	V uD1 = fmav(uD0, lx, flu * Mx);
	V uD2 = fmav(uD0, ly, flu * My);
	V uD3 = fmav(uD0, lz, flu * Mz);

	tmp = f * fmav(lz, uD3 - hDzu, fmav(ly, uD2 - hDyu, fmav(lx, uD1 - hDxu, -uD0)));

	ds[0] = ut;
	ds[1] = ux;
	ds[2] = uy;
	ds[3] = uz;
	ds[4] = uD0 - tmp;
	ds[5] = fmav(lx, tmp, hDxu - uD1);
	ds[6] = fmav(ly, tmp, hDyu - uD2);
	ds[7] = fmav(lz, tmp, hDzu - uD3);

	aux.r = r; aux.ir = ir; aux.f = f; aux.lx = lx; aux.ly = ly; aux.lz = lz; aux.R2 = R2;
	aux.flu = flu; aux.iss = iss;
	(void)one;
}

/* Torus flow + transfer (same model as the FP64 kernel), branch-free: the
 * emission is masked to zero outside r_isco, where the Keplerian flow is not
 * timelike, or where the shift is not positive. */
template <typename V, int NF>
__device__ __forceinline__ void
torus_rt(const RC<V, NF> &c, const V *s, const Aux<V> &x, V *ds)
{
	typedef typename MaskOf<V>::T M;
	const V one = bc<V>(1.0f), zero = bc<V>(0.0f);
	const V q1 = s[1], q2 = s[2], q3 = s[3];
	V kt  = x.flu - s[4];
	V kx  = fmav(x.flu, x.lx, s[5]);
	V ky  = fmav(x.flu, x.ly, s[6]);
	const V R2 = x.R2;
	V irs = rsqv(x.r);                 /* r^-1/2 */
	V sr  = x.r * irs;                 /* r^1/2  */
	V Om  = rcpv(fmav(x.r, sr, c.a));
	V vv  = fmav(Om * Om, R2, -one);
	V lv  = fmav(-((c.a * Om) * R2), x.iss, one);
	V D   = -fmav(x.f * lv, lv, vv);
	M ok  = andv(gtv(x.r, c.risco), gtv(D, zero));
	V utf = rsqv(selv(ok, D, one));
	V shift = -(utf * fmav(Om, fmav(q1, ky, -(q2 * kx)), kt));
	ok = andv(ok, gtv(shift, zero));
	V sh = selv(ok, shift, one);
	/* n0 (r_+/r)^1.5 exp(-z^2 / (2 (h r)^2)) */
	V e = ex2v(-((q3 * q3) * ((x.ir * x.ir) * c.ihr2)));
	V n = selv(ok, c.n0t * ((x.ir * irs) * e), zero);
	/* -j(nu) / shift^2 = -n nu_i^-0.7 shift^-2.7: one power of the shift
	 * for all frequencies, nu_i^-0.7 e^-tau_i as one power of 2 each */
	V mjis2 = -(n * ex2v(bc<V>(-2.7f) * lg2v(sh)));
	V mtfac = -((c.kappa * n) * rcpv(sh));
	const V mlog2e = bc<V>(-1.4426950408889634f);
#pragma unroll
	for(int i = 0; i < NF; ++i) {
		ds[8 + i]      = mjis2 * ex2v(fmav(s[8 + NF + i], mlog2e, c.lgnupow[i]));
		ds[8 + NF + i] = mtfac * c.nuinv2[i];
	}
}

template <typename V, int NF>
__device__ __forceinline__ void
rhs(const RC<V, NF> &c, const V *s, V *ds)
{
	Aux<V> aux;
	ks_rhs<V, NF>(c, s, ds, aux);
	if(NF > 0)
		torus_rt<V, NF>(c, s, aux, ds);
}

/* ---------------------------------------------------------- FP64 islands */

/* KS.cl:48-55 radius root */
__device__ __forceinline__ double
getrr_d(double aa, double x, double y, double z)
{
	double zz = z * z;
	double kk = 0.5 * (fma(x, x, fma(y, y, zz)) - aa);
	return sqrt(fma(kk, kk, aa * zz)) + kk;
}

/* KS.cl:164-168 null constraint from the final state */
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

/* ------------------------------------------------------ slot bookkeeping */

/* Scalar state of one ray slot (a thread has Lanes<V>::N slots). */
struct Slot {
	const MixedRender *c;
	long long ray;
	int dump, dump_end, h, n, dh_cap;
	float cdt;   /* n / |dt| */
	float dtn;   /* dt / n   */
	float rp, eps_stop, cdt_scale;
	double aa_d, rp_d;
	bool active;
};

/* Per-dump constants, computed in FP64 exactly like the host loop of
 * sim-org/gray.c:251-252 and driver.cl:93. */
__device__ __forceinline__ void
start_dump(Slot &S)
{
	const MixedRender &c = *S.c;
	double t      = c.t_init + (double)S.dump * c.dt_dump;
	double target = c.t_init + (double)(S.dump + 1) * c.dt_dump;
	double dt     = target - t;
	double dts    = dt / (double)c.n_sub;
	S.dh_cap = (int)(dts / dt * (double)S.n);
	S.cdt    = (float)((double)S.n / fabs(dt));
	S.dtn    = (float)(dt / (double)S.n);
	S.h      = 0;
}

template <typename V, int ND>
__device__ __forceinline__ void
store_slot(const Slot &S, int k, const V *hi, const V *lo)
{
	const MixedRender &c = *S.c;
	const long long nr = c.n_rays;
	double s[ND];
#pragma unroll
	for(int i = 0; i < ND; ++i) {
		s[i] = (double)getl(hi[i], k) - (double)getl(lo[i], k);
		c.data[i * nr + S.ray] = s[i];
	}
	c.info[S.ray] = getuu_d(c.a_d, s);
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

/* Step size of slot k in ticks (phys.cl:48-64 via driver.cl:93), with the
 * FP64 island near r_+; 0 means the ray stops (captured or NaN). */
template <typename V>
__device__ __forceinline__ int
ticks(const Slot &S, int k, const V *hi, const V *lo)
{
	float x = getl(hi[1], k), y = getl(hi[2], k), z = getl(hi[3], k);
	float aa = (float)S.aa_d;
	float zz = z * z;
	float kk = 0.5f * (fmaf(x, x, fmaf(y, y, zz)) - aa);
	float rr = sqrt_a(fmaf(kk, kk, aa * zz)) + kk;
	float eps = sqrt_a(rr) - S.rp;
	if(eps < 1.0f) {
		double xd = (double)x - (double)getl(lo[1], k);
		double yd = (double)y - (double)getl(lo[2], k);
		double zd = (double)z - (double)getl(lo[3], k);
		eps = (float)(sqrt(getrr_d(S.aa_d, xd, yd, zd)) - S.rp_d);
	}
	if(!(eps >= S.eps_stop))
		return 0;
	float want = S.cdt_scale * eps * eps * S.cdt; /* 0.01 eps^2 n / |dt| */
	int dh = want < (float)S.dh_cap ? (int)want : S.dh_cap;
	return dh < S.n - S.h ? dh : S.n - S.h;
}

template <int NF, typename V, bool ROLLED>
__global__ void __launch_bounds__(Lanes<V>::N == 1 ? 256 : 128)
mixed_kernel(const MixedTable T, unsigned int *__restrict__ queue,
             unsigned long long *__restrict__ steps)
{
	constexpr int ND = 8 + 2 * NF;
	constexpr int L = Lanes<V>::N;
	const unsigned FULL = 0xffffffffu;
	const int lane = threadIdx.x & 31;

	V hi[ND], lo[ND];
	RC<V, NF> rc;
	Slot S[L];
	bool exhausted = false;
	unsigned long long cnt = 0;
#pragma unroll
	for(int k = 0; k < L; ++k)
		S[k].active = false;
#pragma unroll
	for(int i = 0; i < ND; ++i) {
		hi[i] = bc<V>(0.0f);
		lo[i] = bc<V>(0.0f);
	}
	rc = RC<V, NF>();

	for(;;) {
		/* refill the slots whose ray finished (warp-ballot compaction) */
#pragma unroll
		for(int k = 0; k < L; ++k) {
			bool need = !S[k].active && !exhausted;
			unsigned mask = __ballot_sync(FULL, need);
			if(!mask)
				continue;
			int leader = __ffs(mask) - 1;
			unsigned base = 0;
			if(lane == leader)
				base = atomicAdd(queue, (unsigned)__popc(mask));
			base = __shfl_sync(FULL, base, leader);
			if(!need)
				continue;
			unsigned long long g = (unsigned long long)base + __popc(mask & ((1u << lane) - 1));
			if(g >= T.total) {
				exhausted = true;
				continue;
			}
			int rdx = find_render(T, g);
			const MixedRender &c = T.renders[rdx];
			Slot &s = S[k];
			s.c = &c;
			s.ray = (long long)(g - T.prefix[rdx]);
			s.n = (int)((INT_MAX / c.n_sub) * c.n_sub);
			s.dump = c.dump_begin;
			s.dump_end = c.dump_end;
			s.rp = c.rp;
			s.eps_stop = c.eps_stop;
			s.cdt_scale = c.cdt_scale;
			s.aa_d = c.aa_d;
			s.rp_d = c.rp_d;
			load_rc<V, NF>(rc, k, c);
			const long long nr = c.n_rays;
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				double v = c.data[i * nr + s.ray];
				float h = (float)v;
				setl(hi[i], k, h);
				setl(lo[i], k, (float)((double)h - v));
			}
			if(s.dump >= s.dump_end) { /* empty window: state unchanged */
				store_slot<V, ND>(s, k, hi, lo);
				continue;
			}
			start_dump(s);
			s.active = true;
		}
		bool any = false;
#pragma unroll
		for(int k = 0; k < L; ++k)
			any |= S[k].active;
		if(!__any_sync(FULL, any))
			break;

		/* step control per slot; finished slots store and free */
		int dh[L];
		bool step = false;
#pragma unroll
		for(int k = 0; k < L; ++k) {
			dh[k] = 0;
			if(!S[k].active)
				continue;
			dh[k] = ticks<V>(S[k], k, hi, lo);
			if(dh[k] == 0) {
				store_slot<V, ND>(S[k], k, hi, lo);
				S[k].active = false;
			} else {
				step = true;
			}
		}
		if(!step)
			continue;

		/* RK4.cl:37-47 with the compensated update */
		V hs;
#pragma unroll
		for(int k = 0; k < L; ++k)
			setl(hs, k, (float)dh[k] * S[k].dtn);
		const V hh = bc<V>(0.5f) * hs;
		if constexpr(ROLLED) {
			/* one RHS body, looped over the stages (less code, same
			 * arithmetic) */
			V kk[ND], t[ND], sum[ND];
#pragma unroll
			for(int i = 0; i < ND; ++i)
				t[i] = hi[i];
#pragma unroll 1
			for(int st = 0; st < 4; ++st) {
				rhs<V, NF>(rc, t, kk);
				const V wg = bc<V>((st == 1 || st == 2) ? 2.0f : 1.0f);
				const V cg = st < 2 ? hh : hs;
#pragma unroll
				for(int i = 0; i < ND; ++i) {
					if(st < 3)
						sum[i] = st == 0 ? kk[i] : fmav(wg, kk[i], sum[i]);
					t[i] = fmav(cg, kk[i], hi[i]);
				}
			}
			const V h6 = hs * bc<V>(1.0f / 6.0f);
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				V inc = h6 * (sum[i] + kk[i]);
				V yv = inc - lo[i];
				V tv = hi[i] + yv;
				lo[i] = (tv - hi[i]) - yv;
				hi[i] = tv;
			}
		} else if constexpr(L == 1) {
			/* the same stages with the bookkeeping on component pairs
			 * (2j, 2j+1; ND is even): each stage sum, stage state and
			 * compensated update is one packed f32x2 instruction per
			 * pair.  The operations and roundings are those of the
			 * lane-wise form below, except that a product feeding an
			 * add is not contracted into an FMA here */
			constexpr int NP = ND / 2;
			V kk[ND], t[ND];
			float2 H[NP], S2[NP];
			const float2 hh2 = make_float2(hh, hh), hs2 = make_float2(hs, hs);
			const float2 two2 = make_float2(2.0f, 2.0f);
#pragma unroll
			for(int j = 0; j < NP; ++j)
				H[j] = make_float2(hi[2 * j], hi[2 * j + 1]);
			rhs<V, NF>(rc, hi, kk);
#pragma unroll
			for(int j = 0; j < NP; ++j) {
				S2[j] = make_float2(kk[2 * j], kk[2 * j + 1]);
				const float2 s = __ffma2_rn(hh2, S2[j], H[j]);
				t[2 * j] = s.x;
				t[2 * j + 1] = s.y;
			}
			rhs<V, NF>(rc, t, kk);
#pragma unroll
			for(int j = 0; j < NP; ++j) {
				const float2 K = make_float2(kk[2 * j], kk[2 * j + 1]);
				S2[j] = __ffma2_rn(two2, K, S2[j]);
				const float2 s = __ffma2_rn(hh2, K, H[j]);
				t[2 * j] = s.x;
				t[2 * j + 1] = s.y;
			}
			rhs<V, NF>(rc, t, kk);
#pragma unroll
			for(int j = 0; j < NP; ++j) {
				const float2 K = make_float2(kk[2 * j], kk[2 * j + 1]);
				S2[j] = __ffma2_rn(two2, K, S2[j]);
				const float2 s = __ffma2_rn(hs2, K, H[j]);
				t[2 * j] = s.x;
				t[2 * j + 1] = s.y;
			}
			rhs<V, NF>(rc, t, kk);
			const float2 h62 = make_float2(hs * (1.0f / 6.0f), hs * (1.0f / 6.0f));
#pragma unroll
			for(int j = 0; j < NP; ++j) {
				const float2 K   = make_float2(kk[2 * j], kk[2 * j + 1]);
				const float2 inc = __fmul2_rn(h62, __fadd2_rn(S2[j], K));
				const float2 yv  = sub2(inc, make_float2(lo[2 * j], lo[2 * j + 1]));
				const float2 tv  = __fadd2_rn(H[j], yv);
				const float2 c   = sub2(sub2(tv, H[j]), yv);
				hi[2 * j] = tv.x;
				hi[2 * j + 1] = tv.y;
				lo[2 * j] = c.x;
				lo[2 * j + 1] = c.y;
			}
		} else {
			V kk[ND], t[ND], sum[ND];
			rhs<V, NF>(rc, hi, kk);
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				sum[i] = kk[i];
				t[i] = fmav(hh, kk[i], hi[i]);
			}
			rhs<V, NF>(rc, t, kk);
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				sum[i] = fmav(bc<V>(2.0f), kk[i], sum[i]);
				t[i] = fmav(hh, kk[i], hi[i]);
			}
			rhs<V, NF>(rc, t, kk);
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				sum[i] = fmav(bc<V>(2.0f), kk[i], sum[i]);
				t[i] = fmav(hs, kk[i], hi[i]);
			}
			rhs<V, NF>(rc, t, kk);
			const V h6 = hs * bc<V>(1.0f / 6.0f);
#pragma unroll
			for(int i = 0; i < ND; ++i) {
				V inc = h6 * (sum[i] + kk[i]);
				/* Kahan: value = hi - lo */
				V yv = inc - lo[i];
				V tv = hi[i] + yv;
				lo[i] = (tv - hi[i]) - yv;
				hi[i] = tv;
			}
		}
#pragma unroll
		for(int k = 0; k < L; ++k) {
			if(dh[k] == 0)
				continue;
			++cnt;
			Slot &s = S[k];
			s.h += dh[k];
			if(s.h >= s.n) {
				if(++s.dump >= s.dump_end) {
					store_slot<V, ND>(s, k, hi, lo);
					s.active = false;
				} else {
					start_dump(s);
				}
			}
		}
	}

#pragma unroll
	for(int o = 16; o > 0; o >>= 1)
		cnt += __shfl_xor_sync(FULL, cnt, o);
	if(lane == 0 && cnt)
		atomicAdd(steps, cnt);
}

template <int NF, typename V, bool ROLLED>
cudaError_t
launch_nf(const MixedTable &T, unsigned int *queue, unsigned long long *steps,
          cudaStream_t st, const MixedLaunch &cfg)
{
	const int maxb = Lanes<V>::N == 1 ? 256 : 128;
	int block = cfg.block > 0 ? cfg.block : maxb;
	if(block > maxb || block % 32)
		return cudaErrorInvalidValue;
	int per_sm = cfg.blocks_per_sm;
	int occ = 0;
	cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
		&occ, mixed_kernel<NF, V, ROLLED>, block, 0);
	if(e != cudaSuccess)
		return e;
	if(per_sm <= 0 || per_sm > occ)
		per_sm = occ > 0 ? occ : 1;
	const unsigned long long rays_per_block = (unsigned long long)block * Lanes<V>::N;
	long long want = (long long)per_sm * (cfg.sms > 0 ? cfg.sms : 148);
	long long need = (long long)((T.total + rays_per_block - 1) / rays_per_block);
	unsigned grid = (unsigned)(want < need ? want : need);
	if(grid == 0)
		grid = 1;
	mixed_kernel<NF, V, ROLLED><<<grid, block, 0, st>>>(T, queue, steps);
	return cudaGetLastError();
}

template <typename V>
cudaError_t
launch_v(const MixedTable &T, int n_freq, unsigned int *queue, unsigned long long *steps,
         cudaStream_t st, const MixedLaunch &cfg)
{
#define LNF(NF) (cfg.rk4_rolled ? launch_nf<NF, V, true>(T, queue, steps, st, cfg) \
                                : launch_nf<NF, V, false>(T, queue, steps, st, cfg))
	switch(n_freq) {
	case 0: return LNF(0);
	case 1: return LNF(1);
	case 2: return LNF(2);
	case 3: return LNF(3);
	case 4: return LNF(4);
	case 5: return LNF(5);
	case 6: return LNF(6);
	case 7: return LNF(7);
	case 8: return LNF(8);
	default: return cudaErrorInvalidValue;
	}
#undef LNF
}

template <int NF, typename V>
cudaError_t
occ_nf(int block, bool rolled, int *out)
{
	return rolled ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
	                    out, mixed_kernel<NF, V, true>, block, 0)
	              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
	                    out, mixed_kernel<NF, V, false>, block, 0);
}

} /* namespace */

cudaError_t
launch_mixed_table(const MixedTable &T, int n_freq, unsigned int *queue,
                   unsigned long long *steps, cudaStream_t st, const MixedLaunch &cfg)
{
	cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned int), st);
	if(e != cudaSuccess)
		return e;
	if(cfg.rays_per_thread == 2)
		return launch_v<F2>(T, n_freq, queue, steps, st, cfg);
	return launch_v<float>(T, n_freq, queue, steps, st, cfg);
}

cudaError_t
mixed_occupancy(int n_freq, const MixedLaunch &cfg, int *blocks_per_sm)
{
	const bool two = cfg.rays_per_thread == 2;
	const int block = cfg.block > 0 ? cfg.block : (two ? 128 : 256);
#define OCC(NF) (two ? occ_nf<NF, F2>(block, cfg.rk4_rolled, blocks_per_sm) \
                     : occ_nf<NF, float>(block, cfg.rk4_rolled, blocks_per_sm))
	switch(n_freq) {
	case 0: return OCC(0);
	case 1: return OCC(1);
	case 2: return OCC(2);
	case 3: return OCC(3);
	case 4: return OCC(4);
	case 5: return OCC(5);
	case 6: return OCC(6);
	case 7: return OCC(7);
	case 8: return OCC(8);
	default: return cudaErrorInvalidValue;
	}
#undef OCC
}

/* Per-render constants of the thermal emissivities (rt.cl:80-170), FP64 on
 * the host; log K_2(1/te) exactly as rt.cl:70-78 and 166-167 compute it. */
static void
thermal_fast(const RenderParams &p, ThermalFast *t)
{
	const double c = 2.99792458e+10, h = 6.62606957e-27, G = 6.67384800e-08,
	             Ry = 2.17987197e-11, e = 4.80320425e-10, me = 9.10938291e-28,
	             msun = 1.98910000e+33, pi = 3.14159265358979323846,
	             sqrt2 = 1.41421356237309504880, eps = GRAY_EPSILON;
	const double te = p.flow_te, b = p.flow_b;
	static const double LOGK2[GRAY_LOGK2_N] = {GRAY_LOGK2_VALUES};
	t->kf2 = h / (me * c) / c / (te + eps);
	t->kB = 2.0 * h / (c * c);
	t->kB2 = 2.0 * h / (c * c) / t->kf2;
	t->ky = h / (me * c * c) / te;
	t->xg = me * c * c / Ry * te;
	t->sxg = sqrt(t->xg);
	t->g1 = p.th.g1; t->g2 = p.th.g2; t->g3 = p.th.g3; t->g4 = p.th.g4; t->g5 = p.th.g5;
	t->kff = p.m_adm * p.th.ff_f * p.th.ff_f;
	t->sqte = sqrt(te);
	t->knus = te * te * b * (e / (9 * pi * me * c));
	double log_K2 = 0.0;
	if(te > 1e+2) {
		log_K2 = log(2 * te * te - 0.5);
	} else if(te > 1e-1) {
		const double hh = log(te / 1e-1) * p.th.lk_scale;
		int i = (int)hh;
		if(i > 59)
			i = 59;
		const double d = hh - i;
		log_K2 = (1 - d) * LOGK2[i] + d * LOGK2[i + 1];
	}
	t->ksyn = p.m_adm * ((G * msun / (c * c)) * (sqrt2 * pi * e * e / (3 * c))) * exp(-log_K2);
	t->b = b;
	t->syn = te > 1e-1 && b != 0.0;
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
	m->dump_begin = 0;
	m->dump_end = (int)n_dump;
	m->a_d = p.a;
	m->aa_d = p.aa;
	m->rp_d = p.rp;
	m->data = data;
	m->info = info;
	m->n_rays = p.n_rays;
	m->t_init = t_init;
	m->dt_dump = dt_dump;
	m->n_sub = n_sub;
	for(int i = 0; i < GRAY_MAX_FREQ; ++i)
		m->nu_hz[i] = p.nu[i];
	m->thermal = p.flow == GRAY_FLOW_THERMAL;
	if(m->thermal)
		thermal_fast(p, &m->tf);
}

size_t
mixed_render_bytes(void)
{
	return sizeof(MixedRender);
}
