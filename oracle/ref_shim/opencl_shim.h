/*
 * OpenCL C on the host, for compiling the reference's own kernel sources
 * (luxsrc/gray sim-org/*.cl) as C++ -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference's path cannot run here: there is no OpenCL platform and no
 * lux runtime.  Its kernel sources are plain OpenCL C, though, and this
 * header supplies what they use from OpenCL and lux, so that the same
 * source text compiles with g++ and runs on the CPU:
 *  - `real` (double here: the FP64 path), `whole`, the lux literal macro K();
 *  - vector types real4/real8/real16/int4 with component names .x-.w and
 *    .s0-.sf, component-wise arithmetic, and the multi-component swizzles
 *    the sources use (.s123, .s0123, .s489, ...), readable and assignable;
 *  - the built-ins they call (dot, clamp, convert_int4, sincos, sign, cbrt,
 *    asinh, sinh, floor, ...), component-wise where OpenCL defines them so;
 *  - image3d_t and read_imagef with CLK_FILTER_LINEAR |
 *    CLK_ADDRESS_CLAMP_TO_EDGE on unnormalised coordinates, following the
 *    OpenCL specification's linear filter.  The filter weights and the sum
 *    are computed in double, as the CPU restatement (gray_oracle.c)
 *    documents its choice; an OpenCL device rounds them to float;
 *  - get_global_id() from the host loop that plays the NDRange.
 * Address-space qualifiers compile away.  Nothing here is a restatement of
 * the reference's arithmetic: that comes from its .cl files, included as
 * they are.
 */
#ifndef GRAY_OPENCL_SHIM_H
#define GRAY_OPENCL_SHIM_H

#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdint>

#undef M_PI
#undef M_SQRT2

typedef double real;
typedef long whole;
#define K(x) ((real)(x))

#define __kernel
#define __global
#define __local
#define __constant
#define __private
#define __read_only
#define __write_only

/* ---------------------------------------------------------- vector types */

template <typename T, int N> struct VecOf;

#define GRAY_VEC_OPS(V, T, N)                                                        \
	inline V operator+(V a, V b) { for(int i = 0; i < N; ++i) a.v[i] += b.v[i]; return a; } \
	inline V operator-(V a, V b) { for(int i = 0; i < N; ++i) a.v[i] -= b.v[i]; return a; } \
	inline V operator*(V a, V b) { for(int i = 0; i < N; ++i) a.v[i] *= b.v[i]; return a; } \
	inline V operator/(V a, V b) { for(int i = 0; i < N; ++i) a.v[i] /= b.v[i]; return a; } \
	inline V operator+(V a, T s) { for(int i = 0; i < N; ++i) a.v[i] += s; return a; }      \
	inline V operator-(V a, T s) { for(int i = 0; i < N; ++i) a.v[i] -= s; return a; }      \
	inline V operator*(V a, T s) { for(int i = 0; i < N; ++i) a.v[i] *= s; return a; }      \
	inline V operator/(V a, T s) { for(int i = 0; i < N; ++i) a.v[i] /= s; return a; }      \
	inline V operator+(T s, V a) { for(int i = 0; i < N; ++i) a.v[i] = s + a.v[i]; return a; } \
	inline V operator-(T s, V a) { for(int i = 0; i < N; ++i) a.v[i] = s - a.v[i]; return a; } \
	inline V operator*(T s, V a) { for(int i = 0; i < N; ++i) a.v[i] = s * a.v[i]; return a; } \
	inline V operator/(T s, V a) { for(int i = 0; i < N; ++i) a.v[i] = s / a.v[i]; return a; } \
	inline V operator-(V a) { for(int i = 0; i < N; ++i) a.v[i] = -a.v[i]; return a; }     \
	inline V &operator+=(V &a, V b) { return a = a + b; }                                    \
	inline V &operator-=(V &a, V b) { return a = a - b; }                                    \
	inline V &operator*=(V &a, V b) { return a = a * b; }                                    \
	inline V &operator/=(V &a, V b) { return a = a / b; }                                    \
	inline V &operator*=(V &a, T s) { return a = a * s; }                                    \
	inline V &operator/=(V &a, T s) { return a = a / s; }                                    \
	template <> struct VecOf<T, N> { typedef V type; };

/* A swizzle of components I... of a vector: converts to the vector type of
 * that length and assigns from one. */
template <typename V, typename T, int... I>
struct Swz {
	V *p;
	typedef typename VecOf<T, (int)sizeof...(I)>::type R;
	operator R() const
	{
		R r;
		const int idx[] = {I...};
		for(int k = 0; k < (int)sizeof...(I); ++k)
			r.v[k] = p->v[idx[k]];
		return r;
	}
	Swz &operator=(const R &x)
	{
		const int idx[] = {I...};
		for(int k = 0; k < (int)sizeof...(I); ++k)
			p->v[idx[k]] = x.v[k];
		return *this;
	}
	template <int... J>
	Swz &operator=(const Swz<V, T, J...> &o) { return *this = (R)o; }
	Swz &operator+=(const R &x) { return *this = (R) * this + x; }
	Swz &operator-=(const R &x) { return *this = (R) * this - x; }
	Swz &operator*=(T s) { return *this = (R) * this * s; }
	Swz &operator/=(T s) { return *this = (R) * this / s; }
};

#define GRAY_SWZ_MEMBER(V, T)                                                        \
	template <int... I> Swz<V, T, I...> sw() { return Swz<V, T, I...>{this}; }        \
	template <int... I> typename VecOf<T, (int)sizeof...(I)>::type sw() const        \
	{                                                                                \
		typename VecOf<T, (int)sizeof...(I)>::type r;                                \
		const int idx[] = {I...};                                                    \
		for(int k = 0; k < (int)sizeof...(I); ++k)                                   \
			r.v[k] = v[idx[k]];                                                      \
		return r;                                                                    \
	}

struct real2 {
	union { real v[2]; struct { real x, y; }; struct { real s0, s1; }; };
	GRAY_SWZ_MEMBER(real2, real)
};
struct real3 {
	union { real v[3]; struct { real x, y, z; }; struct { real s0, s1, s2; }; };
	GRAY_SWZ_MEMBER(real3, real)
};
struct real4 {
	union { real v[4]; struct { real x, y, z, w; }; struct { real s0, s1, s2, s3; }; };
	GRAY_SWZ_MEMBER(real4, real)
};
struct real8 {
	union { real v[8]; struct { real s0, s1, s2, s3, s4, s5, s6, s7; }; };
	GRAY_SWZ_MEMBER(real8, real)
};
struct real16 {
	union {
		real v[16];
		struct { real s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, sa, sb, sc, sd, se, sf; };
	};
	GRAY_SWZ_MEMBER(real16, real)
};
struct int4 {
	union { int v[4]; struct { int x, y, z, w; }; struct { int s0, s1, s2, s3; }; };
	GRAY_SWZ_MEMBER(int4, int)
};
GRAY_VEC_OPS(real2, real, 2)
GRAY_VEC_OPS(real3, real, 3)
GRAY_VEC_OPS(real4, real, 4)
GRAY_VEC_OPS(real8, real, 8)
GRAY_VEC_OPS(real16, real, 16)
GRAY_VEC_OPS(int4, int, 4)

/* the multi-component swizzles the reference sources use */
#define s012 sw<0, 1, 2>()
#define s123 sw<1, 2, 3>()
#define s126 sw<1, 2, 6>()
#define s37b sw<3, 7, 11>()
#define s489 sw<4, 8, 9>()
#define scde sw<12, 13, 14>()
#define s0123 sw<0, 1, 2, 3>()
#define s4567 sw<4, 5, 6, 7>()
#define s89ab sw<8, 9, 10, 11>()
#define scdef sw<12, 13, 14, 15>()
#define s048c sw<0, 4, 8, 12>()
#define s159d sw<1, 5, 9, 13>()
#define s26ae sw<2, 6, 10, 14>()
#define s37bf sw<3, 7, 11, 15>()

/* ------------------------------------------------------------- built-ins */

#define GRAY_CW1(f)                                                                  \
	inline real4 f(real4 a) { for(int i = 0; i < 4; ++i) a.v[i] = std::f(a.v[i]); return a; }
GRAY_CW1(cbrt)
GRAY_CW1(asinh)
GRAY_CW1(sinh)
GRAY_CW1(floor)
#undef GRAY_CW1

inline real dot(real3 a, real3 b) { return a.v[0] * b.v[0] + a.v[1] * b.v[1] + a.v[2] * b.v[2]; }
inline real dot(real4 a, real4 b)
{
	return a.v[0] * b.v[0] + a.v[1] * b.v[1] + a.v[2] * b.v[2] + a.v[3] * b.v[3];
}
inline int4 clamp(int4 x, int4 lo, int4 hi)
{
	for(int i = 0; i < 4; ++i)
		x.v[i] = x.v[i] < lo.v[i] ? lo.v[i] : x.v[i] > hi.v[i] ? hi.v[i] : x.v[i];
	return x;
}
inline real4 clamp(real4 x, real4 lo, real4 hi)
{
	for(int i = 0; i < 4; ++i)
		x.v[i] = std::fmin(std::fmax(x.v[i], lo.v[i]), hi.v[i]);
	return x;
}
inline int4 convert_int4(real4 a) /* round toward zero, the default */
{
	int4 r;
	for(int i = 0; i < 4; ++i) /* out of range or NaN: saturate, NaN to 0 */
		r.v[i] = a.v[i] != a.v[i]        ? 0
		         : a.v[i] >= 2147483647.0  ? INT_MAX
		         : a.v[i] <= -2147483648.0 ? INT_MIN
		                                   : (int)a.v[i];
	return r;
}
inline real sincos(real x, real *c)
{
	*c = std::cos(x);
	return std::sin(x);
}
inline real sign(real x) { return x > 0 ? 1.0 : x < 0 ? -1.0 : x; }
using std::cbrt;
using std::asinh;
using std::sinh;
using std::floor;
using std::sqrt;
using std::fabs;
using std::pow;
using std::exp;
using std::log;
using std::fmin;
using std::fmax;
inline real min(real a, real b) { return std::fmin(a, b); }
inline real max(real a, real b) { return std::fmax(a, b); }

/* ------------------------------------------------------------------ images */

typedef int sampler_t;
#define CLK_NORMALIZED_COORDS_FALSE 0
#define CLK_ADDRESS_CLAMP_TO_EDGE 2
#define CLK_FILTER_LINEAR 16

#ifdef GRAY_SHIM_NO_IMAGES
/* A program that reads no image (the analytic spacetime): the image type is
 * empty, so the 102 image arguments every kernel function passes on
 * (preamble.cl's SPACETIME_PROTOTYPE_ARGS) cost nothing to copy, as in an
 * OpenCL build where they are handles. */
struct image3d_t {
};
inline real4 read_imagef(image3d_t, sampler_t, real4)
{
	return real4{0, 0, 0, 1};
}
#else
/* a 3-D single-channel FP32 image: one field of a grid level, read from
 * an interleaved [z][y][x][stride] array at offset comp */
struct image3d_t {
	const float *base;
	int nx, ny, nz, stride, comp;
};

/* OpenCL linear filter on unnormalised coordinates with clamp-to-edge:
 * u' = u - 1/2, i0 = floor(u'), i1 = i0 + 1, a = u' - i0, indices clamped
 * to [0, n-1]; the eight texels weighted (1-a or a)(1-b or b)(1-c or c).
 * The result is in .x, as read_imagef returns the red channel there. */
inline real4 read_imagef(image3d_t im, sampler_t, real4 c)
{
	const int n[3] = {im.nx, im.ny, im.nz};
	int i0[3], i1[3];
	real w[3];
	for(int k = 0; k < 3; ++k) {
		const real u = c.v[k] - 0.5;
		const real fl = std::floor(u);
		w[k] = u - fl;
		int a = (int)fl, b = a + 1;
		i0[k] = a < 0 ? 0 : a > n[k] - 1 ? n[k] - 1 : a;
		i1[k] = b < 0 ? 0 : b > n[k] - 1 ? n[k] - 1 : b;
	}
	auto T = [&](int x, int y, int z) {
		return (real)im.base[(((size_t)z * im.ny + y) * im.nx + x) * im.stride + im.comp];
	};
	const real ax = 1 - w[0], ay = 1 - w[1], az = 1 - w[2];
	real4 r = {0, 0, 0, 1};
	r.v[0] = ax * ay * az * T(i0[0], i0[1], i0[2]) + w[0] * ay * az * T(i1[0], i0[1], i0[2]) +
	         ax * w[1] * az * T(i0[0], i1[1], i0[2]) + w[0] * w[1] * az * T(i1[0], i1[1], i0[2]) +
	         ax * ay * w[2] * T(i0[0], i0[1], i1[2]) + w[0] * ay * w[2] * T(i1[0], i0[1], i1[2]) +
	         ax * w[1] * w[2] * T(i0[0], i1[1], i1[2]) + w[0] * w[1] * w[2] * T(i1[0], i1[1], i1[2]);
	return r;
}
#endif /* GRAY_SHIM_NO_IMAGES */

/* --------------------------------------------------------------- work items */

extern thread_local size_t gray_shim_gid[2];
inline size_t get_global_id(int d) { return gray_shim_gid[d]; }

#endif /* GRAY_OPENCL_SHIM_H */
