/*
 * Mixed-precision persistent geodesic kernel (analytic Kerr-Schild + torus
 * transfer).  One launch integrates a window of dump intervals of every ray
 * of one or many renders:
 *
 *  - persistent warps pull rays from a global queue; a warp ballot finds the
 *    lanes whose ray terminated (horizon capture, or its dump window done)
 *    and refills exactly those lanes, so captured rays do not idle SIMD
 *    lanes while their neighbours keep integrating;
 *  - the geodesic equation (KS.cl:263-378) is integrated in Hamiltonian
 *    form, on the event x^mu and the covariant momentum k_mu: k_t is
 *    conserved and the force needs no gradient of l, so a step costs about
 *    a third fewer operations than the second-order form in u^mu; u^mu
 *    (the state in HBM) is converted to k_mu in FP64 when a ray is loaded
 *    and back when it is stored;
 *  - the RHS, RK4 stages (RK4.cl:37-47) and transfer (rt.cl:185-198 form
 *    with the analytic torus) run in FP32 with the approximate
 *    rcp/rsqrt/ex2/lg2 instructions in place of IEEE divide and
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
 *    boundaries are hit exactly as in the FP64 kernel; far from the hole,
 *    where the step is surely the cap, the step rule reads no radius root;
 *  - each ray's render constants live in registers (loaded when the ray is
 *    loaded), not re-read from the table every RHS.
 */
#include <climits>
#include <cstring>
#include <type_traits>

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

/* Register layout of a ray in the mixed kernel: the event x^mu, the spatial
 * covariant momentum k_i, then -I_nu and the optical depth of the first
 * frequency.  The intensities are held negated (exactly, at load and store)
 * because the transfer's dI_nu/dl is minus a power of 2: the registers then
 * integrate that power of 2 itself.  k_t is conserved (the metric does not
 * depend on t) and lives in RC.  For the torus every frequency's absorption is the same function
 * of the ray times nu_i^-2 (alpha_nu = kappa n nu^-2 at the fluid-frame
 * frequency, dtau_i = -alpha shift), so tau_i - tau_i(0) = (nu_0/nu_i)^2
 * (tau_0 - tau_0(0)) holds exactly and only tau_0 is integrated. */
template <int NF>
struct Layout {
	static constexpr int NI = 7 + (NF > 0 ? NF + 1 : 0); /* integrated reals     */
	static constexpr int I0 = 7;                        /* first -I_nu          */
	static constexpr int TAU = 7 + NF;                  /* tau of frequency 0   */
	static constexpr int ND = 8 + 2 * NF;               /* reals in HBM per ray */
};

template <typename V, int NF>
struct RC {
	V a, aa, risco, ihr2, ktau, kt;
	/* log2(n0 r_+^1.5 nu_i^-0.7) plus the frequency's optical-depth
	 * offset, and the factor turning tau_0 into -log2(e) tau_i */
	V lgnu[NF > 0 ? NF : 1], tcoef[NF > 0 ? NF : 1];
};

/* (nu_0/nu_i)^2: tau_i - tau_i(0) = (nu_0/nu_i)^2 (tau_0 - tau_0(0)); the
 * offset tau_i(0) - (nu_0/nu_i)^2 tau_0(0), zero for rays that start at the
 * camera, is folded into the frequency's constant. */
__device__ __forceinline__ double
tau_ratio(const MixedRender &c, int i)
{
	const double q = c.nu_hz[0] / c.nu_hz[i];
	return q * q;
}

/* The render's constants into lane k of rc.  With UNI (a one-render
 * launch) only the per-ray part is held in registers: k_t and the
 * frequencies' optical-depth offsets; uni_rc() supplies the rest from the
 * kernel parameter at each step. */
template <typename V, int NF, bool UNI>
__device__ __forceinline__ void
load_rc(RC<V, NF> &rc, int k, const MixedRender &c, double kt, const double *tau0)
{
	if constexpr(!UNI) {
		setl(rc.a, k, c.a);
		setl(rc.aa, k, c.aa);
		setl(rc.risco, k, c.risco);
		setl(rc.ihr2, k, c.ihr2_log2e);
		setl(rc.ktau, k, c.ktau);
	}
	setl(rc.kt, k, (float)kt);
#pragma unroll
	for(int i = 0; i < NF; ++i) {
		const double q = tau_ratio(c, i);
		const double off = tau0[i] - q * tau0[0];
		setl(rc.lgnu[i], k, (c.ln0t + log2f(c.nupow[i])) - (float)(1.4426950408889634 * off));
		if constexpr(!UNI)
			setl(rc.tcoef[i], k, c.tcoef[i]);
	}
}

/* The constants of a step: rc as loaded, or with UNI the render-wide ones
 * taken from the kernel parameter, which the compiler reads as constant
 * bank operands instead of keeping them live in registers. */
template <typename V, int NF, bool UNI>
__device__ __forceinline__ RC<V, NF>
step_rc(const RC<V, NF> &rc, const MixedRender &R)
{
	if constexpr(!UNI) {
		return rc;
	} else {
		RC<V, NF> o = rc;
		o.a = bc<V>(R.a);
		o.aa = bc<V>(R.aa);
		o.risco = bc<V>(R.risco);
		o.ihr2 = bc<V>(R.ihr2_log2e);
		o.ktau = bc<V>(R.ktau);
#pragma unroll
		for(int i = 0; i < NF; ++i)
			o.tcoef[i] = bc<V>(R.tcoef[i]);
		return o;
	}
}

/* -------------------------------------------------------------- the RHS */

template <typename V>
struct Aux {
	V r, ir, f, iss, R2, lz; /* lz = z / r */
};

/* The geodesic equation of KS.cl:263-378 in Hamiltonian form.  With
 * g^{mu nu} = eta^{mu nu} - f l^mu l^nu (l^mu = (-1, l_x, l_y, l_z)) and
 * L = l^mu k_mu, Hamilton's equations for H = g^{mu nu} k_mu k_nu / 2 are
 *   dx^mu/dl = eta^{mu nu} k_nu - f L l^mu
 *   dk_i/dl  = f L d_i L + L^2 d_i f / 2,   dk_t/dl = 0,
 * the same geodesics as the reference's second-order form in u^mu (the
 * state is mapped u <-> k with down() in FP64 when a ray is loaded and
 * stored).  f, l and r share the reference's radius root and gradient; the
 * r-dependence of L and f enters through d_i r once:
 *   d_i L = dL/dr d_i r + (explicit part),  dL/dr = iss (x k_x + y k_y
 *   - 2 r (l_x k_x + l_y k_y)) - l_z k_z / r,
 * so dk_i = G d_i r + f L (explicit d_i L) [+ L^2 df/dz|_r / 2 for z] with
 * G = f L dL/dr + L^2 df/dr / 2, and no gradient of l is formed. */
template <typename V, int NF>
__device__ __forceinline__ void
ks_ham(const RC<V, NF> &c, const V *s, V *ds, Aux<V> &aux)
{
	const V a = c.a, aa = c.aa, kt = c.kt;
	const V x = s[1], y = s[2], z = s[3];
	const V kx = s[4], ky = s[5], kz = s[6];
	const V half = bc<V>(0.5f), two = bc<V>(2.0f);

	V zz  = z * z;
	V azz = aa * zz;
	V R2  = fmav(x, x, y * y);       /* also the torus's cylindrical radius */
	V kk  = half * ((R2 + zz) - aa);
	V d2  = fmav(kk, kk, azz);
	V idd = rsqv(d2);
	V rr  = fmav(d2, idd, kk);       /* r^2 = sqrt(d2) + kk */
	V ir  = rsqv(rr);
	V r   = rr * ir;
	V ss  = rr + aa;
	V iss = rcpv(ss);
	V hrd = half * (ir * idd);       /* d_x r = hrd r^2 x, d_z r = hrd ss z */
	V t   = (two * rr) * rcpv(fmav(rr, rr, azz)); /* f / r */
	V f   = t * r;
	V tt2 = t * fmav(-(two * rr), t, bc<V>(3.0f)); /* df/dr */
	V fz  = -((t * t) * (aa * (z * ir)));          /* df/dz at fixed r */

	V lx = iss * fmav(x, r, y * a);
	V ly = iss * fmav(y, r, -(x * a));
	V lz = z * ir;
	V P  = fmav(ly, ky, lx * kx);
	V L  = fmav(lz, kz, P - kt);
	V Q  = fmav(y, ky, x * kx);
	V dLdr = fmav(iss, fmav(-(two * r), P, Q), -((lz * ir) * kz));
	V fL  = f * L;
	V hLL = (half * L) * L;
	V G   = fmav(fL, dLdr, hLL * tt2);
	V Gxy = G * (hrd * rr);
	V Gz  = G * (hrd * ss);
	V fLi = fL * iss;

	ds[0] = fL - kt;
	ds[1] = fmav(-fL, lx, kx);
	ds[2] = fmav(-fL, ly, ky);
	ds[3] = fmav(-fL, lz, kz);
	ds[4] = fmav(Gxy, x, fLi * fmav(r, kx, -(a * ky)));
	ds[5] = fmav(Gxy, y, fLi * fmav(r, ky, a * kx));
	ds[6] = fmav(Gz, z, fmav(fL * ir, kz, hLL * fz));

	aux.r = r; aux.ir = ir; aux.f = f; aux.iss = iss; aux.R2 = R2; aux.lz = lz;
}

/* Torus flow + transfer (the FP64 kernel's model), branch-free: the
 * emission is masked to zero outside r_isco, where the Keplerian flow is
 * not timelike, or where the shift is not positive.  The shift is -k_mu
 * u^mu_fluid with k_mu straight from the state.  Every factor is folded into
 * one power of 2 per output, with the density n = n0 r_+^1.5 2^ln in log2,
 * ln = -1.5 lg2 r - z^2 log2(e) / (2 (h r)^2):
 *   dtau_0  = -kappa nu_0^-2 n0 r_+^1.5 2^(ln - lg2 shift)
 *   d(-I_i) = 2^(ln + lg2(n0 r_+^1.5 nu_i^-0.7) - 2.7 lg2 shift - log2(e) tau_i)
 * (dI_i = -n nu_i^-0.7 shift^-2.7 e^-tau_i).  Where the emission is masked
 * ln = -inf, which makes every output exactly 0. */
template <typename V, int NF>
__device__ __forceinline__ void
torus_rt(const RC<V, NF> &c, const V *s, const Aux<V> &x, V *ds)
{
	typedef Layout<NF> Y;
	typedef typename MaskOf<V>::T M;
	const V one = bc<V>(1.0f), zero = bc<V>(0.0f);
	const V q1 = s[1], q2 = s[2];
	const V kx = s[4], ky = s[5];
	V irs = rsqv(x.r);                 /* r^-1/2 */
	V sr  = x.r * irs;                 /* r^1/2  */
	V Om  = rcpv(fmav(x.r, sr, c.a));
	V vv  = fmav(Om * Om, x.R2, -one);
	V lv  = fmav(-((c.a * Om) * x.R2), x.iss, one);
	V D   = -fmav(x.f * lv, lv, vv);
	M ok  = andv(gtv(x.r, c.risco), gtv(D, zero));
	V utf = rsqv(selv(ok, D, one));
	V shift = -(utf * fmav(Om, fmav(q1, ky, -(q2 * kx)), c.kt));
	ok = andv(ok, gtv(shift, zero));
	V lsh = lg2v(selv(ok, shift, one));
	V gz  = -((x.lz * x.lz) * c.ihr2);  /* log2 of the Gaussian: -(z/r)^2 log2(e) / (2 h^2) */
	V ln  = selv(ok, fmav(bc<V>(-1.5f), lg2v(x.r), gz), bc<V>(-INFINITY));
	ds[Y::TAU] = c.ktau * ex2v(ln - lsh);
	V g27 = fmav(bc<V>(-2.7f), lsh, ln);
#pragma unroll
	for(int i = 0; i < NF; ++i)
		ds[Y::I0 + i] = ex2v(fmav(s[Y::TAU], c.tcoef[i], g27 + c.lgnu[i]));
}

template <typename V, int NF>
__device__ __forceinline__ void
rhs(const RC<V, NF> &c, const V *s, V *ds)
{
	Aux<V> aux;
	ks_ham<V, NF>(c, s, ds, aux);
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

/* f and l_mu = (1, l_x, l_y, l_z) at an event (KS.cl:282-333) */
__device__ __forceinline__ void
fl_d(double a, const double *q, double *f, double *l)
{
	double aa = a * a;
	double zz = q[3] * q[3];
	double kk = 0.5 * (fma(q[1], q[1], fma(q[2], q[2], zz)) - aa);
	double rr = sqrt(fma(kk, kk, aa * zz)) + kk;
	double r  = sqrt(rr);
	*f = 2.0 * rr * r / fma(rr, rr, aa * zz);
	double iss = 1.0 / (rr + aa);
	l[0] = iss * fma(q[1], r, q[2] * a);
	l[1] = iss * fma(q[2], r, -(q[1] * a));
	l[2] = q[3] / r;
}

/* KS.cl:91-114 down(): k_mu = g_mu_nu u^nu = eta u + f (l.u) l */
__device__ __forceinline__ void
down_d(double a, const double *q, const double *u, double *k)
{
	double f, l[3];
	fl_d(a, q, &f, l);
	double flu = f * fma(l[2], u[3], fma(l[1], u[2], fma(l[0], u[1], u[0])));
	k[0] = flu - u[0];
	k[1] = fma(flu, l[0], u[1]);
	k[2] = fma(flu, l[1], u[2]);
	k[3] = fma(flu, l[2], u[3]);
}

/* its inverse: u^mu = g^{mu nu} k_nu = eta k - f (l^nu k_nu) l^mu */
__device__ __forceinline__ void
up_d(double a, const double *q, const double *k, double *u)
{
	double f, l[3];
	fl_d(a, q, &f, l);
	double fL = f * fma(l[2], k[3], fma(l[1], k[2], fma(l[0], k[1], -k[0])));
	u[0] = fL - k[0];
	u[1] = fma(-fL, l[0], k[1]);
	u[2] = fma(-fL, l[1], k[2]);
	u[3] = fma(-fL, l[2], k[3]);
}

/* KS.cl:164-168 null constraint g(u,u) from the final state */
__device__ __forceinline__ double
getuu_d(double a, const double *s)
{
	double k[4];
	down_d(a, s, s + 4, k);
	return fma(k[3], s[7], fma(k[2], s[6], fma(k[1], s[5], k[0] * s[4])));
}

/* ------------------------------------------------------ slot bookkeeping */

/* Scalar state of one ray slot (a thread has Lanes<V>::N slots). */
struct Slot {
	const MixedRender *c;
	unsigned int ray;  /* a render has at most 2^31 rays */
	int dump, dump_end, h, n, dh_cap;
	float cdt;   /* n / |dt| */
	float r2_far; /* x^2+y^2+z^2-a^2 beyond which the step is surely dh_cap */
	float dtn;   /* dt / n   */
	float rp, eps_stop, cdt_scale;
	double aa_d, rp_d;
	bool active;
};

/* Per-dump constants, computed in FP64 exactly like the host loop of
 * sim-org/gray.c:251-252 and driver.cl:93; n is the render's ticks per
 * dump interval. */
__device__ __forceinline__ void
start_dump(Slot &S, const MixedRender &c, int n)
{
	double t      = c.t_init + (double)S.dump * c.dt_dump;
	double target = c.t_init + (double)(S.dump + 1) * c.dt_dump;
	double dt     = target - t;
	double dts    = dt / (double)c.n_sub;
	S.dh_cap = (int)(dts / dt * (double)n);
	S.cdt    = (float)((double)n / fabs(dt));
	S.dtn    = (float)(dt / (double)n);
	S.h      = 0;
	/* eps at which the tick rule reaches dh_cap, with 1% to spare for the
	 * FP32 rounding of the exact rule: r^2 >= x^2+y^2+z^2-a^2 (KS.cl:48-55),
	 * so beyond this the step is dh_cap whatever eps rounds to */
	const double e_cap = sqrt((double)S.dh_cap / (0.01 * (double)S.cdt));
	const double r_far = 1.01 * ((double)c.rp_d + e_cap) + 1.0;
	S.r2_far = (float)(r_far * r_far);
}

/* A slot's render-wide values: from the slot (loaded with the ray) or, with
 * UNI, from the kernel parameter. */
template <bool UNI>
struct SlotView {
	const Slot &S;
	const MixedRender &R;
	__device__ __forceinline__ const MixedRender &render() const { return UNI ? R : *S.c; }
	__device__ __forceinline__ int n() const { return UNI ? R.n_ticks : S.n; }
	__device__ __forceinline__ int dump_end() const { return UNI ? R.dump_end : S.dump_end; }
	__device__ __forceinline__ float rp() const { return UNI ? R.rp : S.rp; }
	__device__ __forceinline__ float eps_stop() const { return UNI ? R.eps_stop : S.eps_stop; }
	__device__ __forceinline__ float cdt_scale() const { return UNI ? R.cdt_scale : S.cdt_scale; }
	__device__ __forceinline__ double aa_d() const { return UNI ? R.aa_d : S.aa_d; }
	__device__ __forceinline__ double rp_d() const { return UNI ? R.rp_d : S.rp_d; }
};

/* Final state to HBM in the reference's layout: x^mu, u^mu (from k_mu in
 * FP64), I_nu, tau_nu (tau_i rebuilt from tau_0) and g(u,u).  The ray's
 * state as it was loaded is still in HBM: k_t is recomputed from it (the
 * same FP64 value the load computed) and the initial tau_i are read from it
 * before they are overwritten.  Called once per ray and dump window, so it
 * is kept out of line: its FP64 temporaries do not add to the register
 * count of the stepping loop. */
__device__ __noinline__ void
store_ray(const MixedRender &c, unsigned int ray, int nf, const float *hi, const float *lo)
{
	const long long nr = c.n_rays;
	double q[4], k[4], u[4];
	{
		double s0[8];
		for(int i = 0; i < 8; ++i)
			s0[i] = c.data[i * nr + ray];
		down_d(c.a_d, s0, s0 + 4, k);
	}
	for(int i = 0; i < 4; ++i)
		q[i] = (double)hi[i] + (double)lo[i];
	for(int i = 1; i < 4; ++i)
		k[i] = (double)hi[3 + i] + (double)lo[3 + i];
	up_d(c.a_d, q, k, u);
	for(int i = 0; i < 4; ++i) {
		c.data[i * nr + ray] = q[i];
		c.data[(4 + i) * nr + ray] = u[i];
	}
	if(nf > 0) {
		const double tau = (double)hi[7 + nf] + (double)lo[7 + nf];
		const double tau00 = c.data[(8 + nf) * nr + ray];
		for(int i = 1; i < nf; ++i) {
			double *p = c.data + (8 + nf + i) * nr + ray;
			*p = fma(tau_ratio(c, i), tau - tau00, *p);
		}
		c.data[(8 + nf) * nr + ray] = tau;
		for(int i = 0; i < nf; ++i)
			c.data[(8 + i) * nr + ray] = -((double)hi[7 + i] + (double)lo[7 + i]);
	}
	double s[8] = {q[0], q[1], q[2], q[3], u[0], u[1], u[2], u[3]};
	c.info[ray] = getuu_d(c.a_d, s);
}

template <typename V, int NF>
__device__ __forceinline__ void
store_slot(const MixedRender &c, const Slot &S, int k, const V *hi, const V *lo)
{
	constexpr int NI = Layout<NF>::NI;
	float h[NI], l[NI];
#pragma unroll
	for(int i = 0; i < NI; ++i) {
		h[i] = getl(hi[i], k);
		l[i] = getl(lo[i], k);
	}
	store_ray(c, S.ray, NF, h, l);
}

template <int L, typename C>
__device__ __forceinline__ void
flush_steps(C &cnt, unsigned long long *steps)
{
	if(L == 1 && cnt >= 0x80000000u) {
		atomicAdd(steps, (unsigned long long)cnt);
		cnt = 0;
	}
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
template <typename V, bool UNI>
__device__ __forceinline__ int
ticks(const SlotView<UNI> &v, int k, const V *hi, const V *lo)
{
	const Slot &S = v.S;
	float x = getl(hi[1], k), y = getl(hi[2], k), z = getl(hi[3], k);
	float aa = (float)v.aa_d();
	float zz = z * z;
	float q2 = fmaf(x, x, fmaf(y, y, zz));
	if(q2 - aa >= S.r2_far) /* far from the hole: the capped step */
		return S.dh_cap < v.n() - S.h ? S.dh_cap : v.n() - S.h;
	float kk = 0.5f * (q2 - aa);
	float rr = sqrt_a(fmaf(kk, kk, aa * zz)) + kk;
	float eps = sqrt_a(rr) - v.rp();
	if(eps < 1.0f) {
		double xd = (double)x + (double)getl(lo[1], k);
		double yd = (double)y + (double)getl(lo[2], k);
		double zd = (double)z + (double)getl(lo[3], k);
		eps = (float)(sqrt(getrr_d(v.aa_d(), xd, yd, zd)) - v.rp_d());
	}
	if(!(eps >= v.eps_stop()))
		return 0;
	float want = v.cdt_scale() * eps * eps * S.cdt; /* 0.01 eps^2 n / |dt| */
	int dh = want < (float)S.dh_cap ? (int)want : S.dh_cap;
	return dh < v.n() - S.h ? dh : v.n() - S.h;
}

/* One RK4 step (RK4.cl:37-47) of size hs on the NI integrated reals with
 * the compensated update (value = hi + lo).  With one ray per thread the
 * stage sums, stage states and update run on pairs of components (2j,
 * 2j+1) in packed f32x2, one instruction per pair; an odd last component
 * runs scalar.  The update adds h/6 (k1 + 2 k2 + 2 k3 + k4) to the low part
 * with one fused multiply-add and renormalises (Fast2Sum).  (Pairing the
 * components the RHS reads apart from those it does not, so that whole
 * pairs of stage states drop out, measured 6% slower.) */
template <typename V, int NF>
__device__ __forceinline__ void
rk4_packed(const RC<V, NF> &rc, V *hi, V *lo, V hs)
{
	constexpr int NI = Layout<NF>::NI;
	constexpr int NP = NI / 2;
	constexpr bool TAIL = NI & 1;
	constexpr int LAST = NI - 1;
	const V hh = bc<V>(0.5f) * hs;
	V kk[NI], t[NI];
	float2 H[NP], S2[NP];
	float tS = 0.0f;
	const float2 hh2 = make_float2(hh, hh), hs2 = make_float2(hs, hs);
	const float2 two2 = make_float2(2.0f, 2.0f);
#define PA(j) (2 * (j))
#define PB(j) (2 * (j) + 1)
#pragma unroll
	for(int j = 0; j < NP; ++j)
		H[j] = make_float2(hi[PA(j)], hi[PB(j)]);
	rhs<V, NF>(rc, hi, kk);
#pragma unroll
	for(int j = 0; j < NP; ++j) {
		S2[j] = make_float2(kk[PA(j)], kk[PB(j)]);
		const float2 s = __ffma2_rn(hh2, S2[j], H[j]);
		t[PA(j)] = s.x;
		t[PB(j)] = s.y;
	}
	if(TAIL) {
		tS = kk[LAST];
		t[LAST] = fmaf(hh, kk[LAST], hi[LAST]);
	}
#pragma unroll
	for(int st = 1; st < 3; ++st) {
		rhs<V, NF>(rc, t, kk);
		const float2 c2 = st == 1 ? hh2 : hs2;
#pragma unroll
		for(int j = 0; j < NP; ++j) {
			const float2 K = make_float2(kk[PA(j)], kk[PB(j)]);
			S2[j] = __ffma2_rn(two2, K, S2[j]);
			const float2 s = __ffma2_rn(c2, K, H[j]);
			t[PA(j)] = s.x;
			t[PB(j)] = s.y;
		}
		if(TAIL) {
			tS = fmaf(2.0f, kk[LAST], tS);
			t[LAST] = fmaf(st == 1 ? hh : hs, kk[LAST], hi[LAST]);
		}
	}
	rhs<V, NF>(rc, t, kk);
	const float h6 = hs * (1.0f / 6.0f);
	const float2 h62 = make_float2(h6, h6);
#pragma unroll
	for(int j = 0; j < NP; ++j) {
		const float2 K  = make_float2(kk[PA(j)], kk[PB(j)]);
		const float2 yv = __ffma2_rn(h62, __fadd2_rn(S2[j], K), make_float2(lo[PA(j)], lo[PB(j)]));
		const float2 tv = __fadd2_rn(H[j], yv);
		const float2 c  = sub2(yv, sub2(tv, H[j]));
		hi[PA(j)] = tv.x;
		hi[PB(j)] = tv.y;
		lo[PA(j)] = c.x;
		lo[PB(j)] = c.y;
	}
#undef PA
#undef PB
	if(TAIL) {
		const float yv = fmaf(h6, tS + kk[LAST], lo[LAST]);
		const float tv = hi[LAST] + yv;
		lo[LAST] = yv - (tv - hi[LAST]);
		hi[LAST] = tv;
	}
}

/* UNI: the table holds one render, passed again by value as R1 (a kernel
 * parameter); its constants are then not held per ray.  Otherwise R1 is
 * unused. */
template <int NF, typename V, bool ROLLED, bool UNI>
__global__ void __launch_bounds__(Lanes<V>::N == 1 ? 256 : 128, Lanes<V>::N == 1 ? 2 : 1)
mixed_kernel(const MixedTable T, const __grid_constant__ MixedRender R1,
             unsigned int *__restrict__ queue, unsigned long long *__restrict__ steps)
{
	typedef Layout<NF> Y;
	constexpr int NI = Y::NI;
	constexpr int L = Lanes<V>::N;
	const unsigned FULL = 0xffffffffu;
	const int lane = threadIdx.x & 31;

	V hi[NI], lo[NI];
	RC<V, NF> rc;
	Slot S[L];
	bool exhausted = false;
	/* accepted steps of this thread; with one slot a 32-bit count, flushed
	 * at a ray's events (store, dump boundary) once it reaches 2^31: between
	 * two events a ray takes at most one interval's ticks (< 2^31) */
	typename std::conditional<L == 1, unsigned int, unsigned long long>::type cnt = 0;
#pragma unroll
	for(int k = 0; k < L; ++k)
		S[k].active = false;
#pragma unroll
	for(int i = 0; i < NI; ++i) {
		hi[i] = bc<V>(0.0f);
		lo[i] = bc<V>(0.0f);
	}
	rc = RC<V, NF>();

	for(;;) {
		/* refill the slots whose ray finished (warp-ballot compaction);
		 * one vote per step while every slot of the warp is busy */
		bool full = true;
#pragma unroll
		for(int k = 0; k < L; ++k)
			full &= S[k].active;
		if(!__all_sync(FULL, full)) {
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
				const int rdx = UNI ? 0 : find_render(T, g);
				const MixedRender &c = UNI ? R1 : T.renders[rdx];
				Slot &s = S[k];
				s.ray = (unsigned int)(UNI ? g : g - T.prefix[rdx]);
				s.dump = c.dump_begin;
				if constexpr(!UNI) {
					s.c = &c;
					s.n = c.n_ticks;
					s.dump_end = c.dump_end;
					s.rp = c.rp;
					s.eps_stop = c.eps_stop;
					s.cdt_scale = c.cdt_scale;
					s.aa_d = c.aa_d;
					s.rp_d = c.rp_d;
				}
				const long long nr = c.n_rays;
				double s0[8], k0[4], tau0[NF > 0 ? NF : 1];
#pragma unroll
				for(int i = 0; i < 8; ++i)
					s0[i] = c.data[i * nr + s.ray];
				if(s.dump >= c.dump_end) { /* empty window: state unchanged */
					c.info[s.ray] = getuu_d(c.a_d, s0);
					continue;
				}
				down_d(c.a_d, s0, s0 + 4, k0);
				double v[NI];
				v[0] = s0[0]; v[1] = s0[1]; v[2] = s0[2]; v[3] = s0[3];
				v[4] = k0[1]; v[5] = k0[2]; v[6] = k0[3];
#pragma unroll
				for(int i = 0; i < NF; ++i) {
					v[Y::I0 + i] = -c.data[(8 + i) * nr + s.ray];
					tau0[i] = c.data[(8 + NF + i) * nr + s.ray];
				}
				if(NF > 0)
					v[Y::TAU] = tau0[0];
				load_rc<V, NF, UNI>(rc, k, c, k0[0], tau0);
#pragma unroll
				for(int i = 0; i < NI; ++i) {
					float h = (float)v[i];
					setl(hi[i], k, h);
					setl(lo[i], k, (float)(v[i] - (double)h));
				}
				start_dump(s, c, c.n_ticks);
				s.active = true;
			}
			bool any = false;
#pragma unroll
			for(int k = 0; k < L; ++k)
				any |= S[k].active;
			if(!__any_sync(FULL, any))
				break;
		}

		/* step control per slot; finished slots store and free */
		int dh[L];
		bool step = false;
#pragma unroll
		for(int k = 0; k < L; ++k) {
			dh[k] = 0;
			if(!S[k].active)
				continue;
			const SlotView<UNI> v{S[k], R1};
			dh[k] = ticks<V, UNI>(v, k, hi, lo);
			if(dh[k] == 0) {
				store_slot<V, NF>(v.render(), S[k], k, hi, lo);
				S[k].active = false;
				flush_steps<L>(cnt, steps);
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
		if constexpr(ROLLED) {
			/* one RHS body, looped over the stages (less code, same
			 * arithmetic) */
			const V hh = bc<V>(0.5f) * hs;
			V kk[NI], t[NI], sum[NI];
#pragma unroll
			for(int i = 0; i < NI; ++i)
				t[i] = hi[i];
#pragma unroll 1
			for(int st = 0; st < 4; ++st) {
				rhs<V, NF>(rc, t, kk);
				const V wg = bc<V>((st == 1 || st == 2) ? 2.0f : 1.0f);
				const V cg = st < 2 ? hh : hs;
#pragma unroll
				for(int i = 0; i < NI; ++i) {
					if(st < 3)
						sum[i] = st == 0 ? kk[i] : fmav(wg, kk[i], sum[i]);
					t[i] = fmav(cg, kk[i], hi[i]);
				}
			}
			const V h6 = hs * bc<V>(1.0f / 6.0f);
#pragma unroll
			for(int i = 0; i < NI; ++i) {
				V yv = fmav(h6, sum[i] + kk[i], lo[i]);
				V tv = hi[i] + yv;
				lo[i] = yv - (tv - hi[i]);
				hi[i] = tv;
			}
		} else if constexpr(L == 1) {
			rk4_packed<V, NF>(step_rc<V, NF, UNI>(rc, R1), hi, lo, hs);
		} else {
			const V hh = bc<V>(0.5f) * hs;
			V kk[NI], t[NI], sum[NI];
			rhs<V, NF>(rc, hi, kk);
#pragma unroll
			for(int i = 0; i < NI; ++i) {
				sum[i] = kk[i];
				t[i] = fmav(hh, kk[i], hi[i]);
			}
			rhs<V, NF>(rc, t, kk);
#pragma unroll
			for(int i = 0; i < NI; ++i) {
				sum[i] = fmav(bc<V>(2.0f), kk[i], sum[i]);
				t[i] = fmav(hh, kk[i], hi[i]);
			}
			rhs<V, NF>(rc, t, kk);
#pragma unroll
			for(int i = 0; i < NI; ++i) {
				sum[i] = fmav(bc<V>(2.0f), kk[i], sum[i]);
				t[i] = fmav(hs, kk[i], hi[i]);
			}
			rhs<V, NF>(rc, t, kk);
			const V h6 = hs * bc<V>(1.0f / 6.0f);
#pragma unroll
			for(int i = 0; i < NI; ++i) {
				/* compensated: value = hi + lo */
				V yv = fmav(h6, sum[i] + kk[i], lo[i]);
				V tv = hi[i] + yv;
				lo[i] = yv - (tv - hi[i]);
				hi[i] = tv;
			}
		}
#pragma unroll
		for(int k = 0; k < L; ++k) {
			if(dh[k] == 0)
				continue;
			++cnt;
			Slot &s = S[k];
			const SlotView<UNI> v{s, R1};
			s.h += dh[k];
			if(s.h >= v.n()) {
				flush_steps<L>(cnt, steps);
				if(++s.dump >= v.dump_end()) {
					store_slot<V, NF>(v.render(), s, k, hi, lo);
					s.active = false;
				} else {
					start_dump(s, v.render(), v.n());
				}
			}
		}
	}

	unsigned long long total = cnt;
#pragma unroll
	for(int o = 16; o > 0; o >>= 1)
		total += __shfl_xor_sync(FULL, total, o);
	if(lane == 0 && total)
		atomicAdd(steps, total);
}

template <int NF, typename V, bool ROLLED, bool UNI>
cudaError_t
launch_nf(const MixedTable &T, const MixedRender &R1, unsigned int *queue,
          unsigned long long *steps, cudaStream_t st, const MixedLaunch &cfg)
{
	const int maxb = Lanes<V>::N == 1 ? 256 : 128;
	int block = cfg.block > 0 ? cfg.block : maxb;
	if(block > maxb || block % 32)
		return cudaErrorInvalidValue;
	int per_sm = cfg.blocks_per_sm;
	int occ = 0;
	cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
		&occ, mixed_kernel<NF, V, ROLLED, UNI>, block, 0);
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
	mixed_kernel<NF, V, ROLLED, UNI><<<grid, block, 0, st>>>(T, R1, queue, steps);
	return cudaGetLastError();
}

/* The one-render form is built for the scalar, unrolled kernel alone: the
 * other forms are autotuner alternatives. */
template <typename V>
cudaError_t
launch_v(const MixedTable &T, const MixedRender *one, int n_freq, unsigned int *queue,
         unsigned long long *steps, cudaStream_t st, const MixedLaunch &cfg)
{
	MixedRender none;
	memset(&none, 0, sizeof(none));
	const bool uni = one && T.n_renders == 1 && Lanes<V>::N == 1 && !cfg.rk4_rolled;
	const MixedRender &R1 = uni ? *one : none;
#define LNF(NF) (cfg.rk4_rolled ? launch_nf<NF, V, true, false>(T, R1, queue, steps, st, cfg) \
                 : uni ? launch_nf<NF, V, false, Lanes<V>::N == 1>(T, R1, queue, steps, st, cfg) \
                       : launch_nf<NF, V, false, false>(T, R1, queue, steps, st, cfg))
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
	                    out, mixed_kernel<NF, V, true, false>, block, 0)
	              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
	                    out, mixed_kernel<NF, V, false, false>, block, 0);
}

} /* namespace */

cudaError_t
launch_mixed_table(const MixedTable &T, int n_freq, unsigned int *queue,
                   unsigned long long *steps, cudaStream_t st, const MixedLaunch &cfg,
                   const MixedRender *one)
{
	cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned int), st);
	if(e != cudaSuccess)
		return e;
	if(cfg.rays_per_thread == 2)
		return launch_v<F2>(T, one, n_freq, queue, steps, st, cfg);
	return launch_v<float>(T, one, n_freq, queue, steps, st, cfg);
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
	/* the density scale n0 r_+^1.5 (zero without the torus flow) in log2,
	 * and -kappa nu_0^-2 n0 r_+^1.5 */
	const float n0t = p.flow == GRAY_FLOW_TORUS ? m->n0_rp15 : 0.0f;
	m->ln0t = n0t > 0.0f ? log2f(n0t) : -INFINITY;
	m->ktau = p.n_freq > 0 ? -(m->kappa * m->nuinv2[0]) * n0t : 0.0f;
	for(int i = 0; i < GRAY_MAX_FREQ; ++i) {
		m->tcoef[i] = 0.0f;
		if(i < p.n_freq) {
			const double q = p.nu[0] / p.nu[i];
			m->tcoef[i] = (float)(-1.4426950408889634 * (q * q));
		}
	}
	m->flow = p.flow;
	m->dump_begin = 0;
	m->dump_end = (int)n_dump;
	m->n_ticks = (int)((INT_MAX / n_sub) * n_sub);
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
