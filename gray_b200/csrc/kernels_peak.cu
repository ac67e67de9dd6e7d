/*
 * CUDA-core peak microbenchmark: independent FMA chains per thread, enough
 * warps to fill every SM.  Gives the FP32 and FP64 denominators of the
 * roofline of the geodesic kernels (which are CUDA-core bound, not
 * tensor-core or HBM bound).  FP32 is measured both with scalar FFMA and
 * with the packed f32x2 FMA of sm_100; the larger rate is reported.
 */
#include "gray_internal.h"

namespace {

constexpr int CHAINS = 8;

__global__ void __launch_bounds__(256)
fma32_kernel(float *out, int iters, float a, float b)
{
	float v[CHAINS];
#pragma unroll
	for(int c = 0; c < CHAINS; ++c)
		v[c] = threadIdx.x * 1e-3f + c;
	for(int i = 0; i < iters; ++i) {
#pragma unroll
		for(int c = 0; c < CHAINS; ++c)
			v[c] = fmaf(v[c], a, b);
	}
	float s = 0.0f;
#pragma unroll
	for(int c = 0; c < CHAINS; ++c)
		s += v[c];
	if(s == 12345.678f)
		out[0] = s; /* keeps the chains alive */
}

__global__ void __launch_bounds__(256)
fma32x2_kernel(float *out, int iters, float a, float b)
{
	float2 v[CHAINS];
	const float2 A = make_float2(a, a), B = make_float2(b, b);
#pragma unroll
	for(int c = 0; c < CHAINS; ++c)
		v[c] = make_float2(threadIdx.x * 1e-3f + c, c + 0.5f);
	for(int i = 0; i < iters; ++i) {
#pragma unroll
		for(int c = 0; c < CHAINS; ++c)
			v[c] = __ffma2_rn(v[c], A, B);
	}
	float s = 0.0f;
#pragma unroll
	for(int c = 0; c < CHAINS; ++c)
		s += v[c].x + v[c].y;
	if(s == 12345.678f)
		out[0] = s;
}

__global__ void __launch_bounds__(256)
fma64_kernel(double *out, int iters, double a, double b)
{
	double v[CHAINS];
#pragma unroll
	for(int c = 0; c < CHAINS; ++c)
		v[c] = threadIdx.x * 1e-3 + c;
	for(int i = 0; i < iters; ++i) {
#pragma unroll
		for(int c = 0; c < CHAINS; ++c)
			v[c] = fma(v[c], a, b);
	}
	double s = 0.0;
#pragma unroll
	for(int c = 0; c < CHAINS; ++c)
		s += v[c];
	if(s == 12345.678)
		out[0] = s;
}

/* L1 load bandwidth with the numerical kernel's load instruction: 32-byte
 * loads (ld.global.nc.v8.f32) from a 16 KiB window that stays resident in
 * L1, a warp's 32 lanes reading 32 consecutive rows (1 KiB, fully used
 * lines), so that the L1 data path, not its tag lookups, is the limit: the
 * ceiling of any gather that hits in L1.  Each load feeds an add chain so
 * that it is not dead. */
__global__ void __launch_bounds__(256)
l1_gather_kernel(const float *__restrict__ buf, float *out, int iters)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
	for(int i = 0; i < iters; ++i) {
		/* 512 rows of 32 bytes; warp w reads rows 32 (i + w) .. + 31 */
		const int row = (32 * (i + warp) + lane) & 511;
		const float *src = buf + row * 8;
		float v[8];
		asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
		             : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]),
		               "=f"(v[6]), "=f"(v[7])
		             : "l"(src));
		acc[i & 3] += (v[0] + v[1]) + (v[2] + v[3]) + ((v[4] + v[5]) + (v[6] + v[7]));
	}
	const float s = acc[0] + acc[1] + acc[2] + acc[3];
	if(s == 12345.678f)
		out[0] = s;
}

/* Bytes/s of the best of 5 timed launches of the L1 load pattern. */
cudaError_t
measure_l1(int sms, cudaStream_t st, double *bps)
{
	const int block = 256, iters = 1 << 15, reps = 5;
	const unsigned grid = (unsigned)sms * 8;
	const size_t window = 16384; /* 128 lines x 128 bytes */
	float *buf = nullptr;
	cudaEvent_t e0, e1;
	cudaError_t e = cudaMalloc((void **)&buf, window + 64);
	if(e != cudaSuccess)
		return e;
	e = cudaMemsetAsync(buf, 0, window + 64, st);
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	double best = 0.0;
	for(int r = 0; r < reps + 1 && e == cudaSuccess; ++r) {
		cudaEventRecord(e0, st);
		l1_gather_kernel<<<grid, block, 0, st>>>(buf, buf + window / sizeof(float), iters);
		cudaEventRecord(e1, st);
		e = cudaEventSynchronize(e1);
		if(e != cudaSuccess)
			break;
		float ms = 0.0f;
		cudaEventElapsedTime(&ms, e0, e1);
		const double bytes = (double)grid * block * iters * 32.0;
		if(r > 0 && ms > 0.0f && bytes / (ms * 1e-3) > best)
			best = bytes / (ms * 1e-3);
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(buf);
	*bps = best;
	return e;
}

} /* namespace */

/* Returns FLOP/s (FMA = 2 FLOP) of the best of `reps` timed launches; with
 * GRAY_PEAK_L1_GATHER, the L1 load bandwidth in bytes/s. */
cudaError_t
measure_peak(int precision, int sms, cudaStream_t st, double *flops)
{
	if(precision == GRAY_PEAK_L1_GATHER)
		return measure_l1(sms, st, flops);
	const int block = 256, iters = 1 << 14, reps = 5;
	const unsigned grid = (unsigned)sms * 8;
	void *buf = nullptr;
	cudaEvent_t e0, e1;
	cudaError_t e = cudaMalloc(&buf, 64);
	if(e != cudaSuccess)
		return e;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	double best = 0.0;
	const double threads = (double)grid * block;
	const int variants = precision == GRAY_PREC_FP64 ? 1 : 2;
	for(int var = 0; var < variants && e == cudaSuccess; ++var) {
		for(int r = 0; r < reps + 1 && e == cudaSuccess; ++r) {
			cudaEventRecord(e0, st);
			if(precision == GRAY_PREC_FP64)
				fma64_kernel<<<grid, block, 0, st>>>((double *)buf, iters, 0.999999, 1e-7);
			else if(var == 0)
				fma32_kernel<<<grid, block, 0, st>>>((float *)buf, iters, 0.999999f, 1e-7f);
			else
				fma32x2_kernel<<<grid, block, 0, st>>>((float *)buf, iters, 0.999999f, 1e-7f);
			cudaEventRecord(e1, st);
			e = cudaEventSynchronize(e1);
			if(e != cudaSuccess)
				break;
			float ms = 0.0f;
			cudaEventElapsedTime(&ms, e0, e1);
			double fl = threads * iters * CHAINS * 2.0 * (var == 1 ? 2.0 : 1.0);
			if(r > 0 && ms > 0.0f && fl / (ms * 1e-3) > best)
				best = fl / (ms * 1e-3);
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(buf);
	*flops = best;
	return e;
}
