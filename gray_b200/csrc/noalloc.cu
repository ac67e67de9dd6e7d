/*
 * Allocation-free entry point of the mixed-precision persistent kernel.
 *
 * Some callers cannot call cudaMalloc: an application whose own allocator
 * already owns the device memory (a serving process or a visualisation host
 * that reserves HBM up front and forbids side allocations so its accounting
 * stays exact), or a latency-critical loop that cannot afford the implicit
 * device-wide synchronisation of cudaMalloc/cudaFree.  They hand in the
 * ray-state and diagnostic buffers they already own; the small scratch the
 * kernel needs beyond those (render table, prefix sums, ray queue, step
 * counter) lives in the file-scope device array below, which every GPU that
 * loads this library holds until the process exits.
 */
#include <cstring>
#include <mutex>

#include "gray_internal.h"
#include "mixed_table.h"

namespace {

struct NoallocScratch {
	MixedRender renders[GRAY_NOALLOC_MAX_RENDERS];
	unsigned long long prefix[GRAY_NOALLOC_MAX_RENDERS];
	unsigned long long steps;
	unsigned int queue;
};
static_assert(sizeof(NoallocScratch) <= GRAY_NOALLOC_SCRATCH_BYTES,
              "no-alloc scratch layout exceeds its static array");

/* The scratch itself.  In host code this name is only a stand-in for the
 * device symbol: its device address comes from cudaGetSymbolAddress. */
static __device__ __align__(256) unsigned char g_noalloc_scratch[GRAY_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
NoallocScratch *g_addr[MAX_DEVICES] = {nullptr};

/* Once per device, with that device current: look up the scratch's device
 * address.  Called by the first gray_run_mixed_noalloc on each device. */
cudaError_t
scratch_for(int device, NoallocScratch **out)
{
	std::lock_guard<std::mutex> lk(g_mu);
	if(!g_addr[device]) {
		void *p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if(e != cudaSuccess)
			return e;
		g_addr[device] = (NoallocScratch *)p;
	}
	*out = g_addr[device];
	return cudaSuccess;
}

int
status_of(cudaError_t e)
{
	return e == cudaSuccess ? GRAY_OK : GRAY_ECUDA;
}

} /* namespace */

extern "C" int
gray_run_mixed_noalloc(int device, const gray_render_desc *descs, int n_renders,
                       double *const *state_dev, double *const *info_dev,
                       void *cuda_stream, uint64_t *steps_host)
{
	int n_dev = 0;
	if(!descs || !state_dev || !info_dev)
		return GRAY_EINVAL;
	if(n_renders < 1 || n_renders > GRAY_NOALLOC_MAX_RENDERS)
		return GRAY_EINVAL; /* beyond the static scratch: at most GRAY_NOALLOC_MAX_RENDERS */
	/* arguments first, so a bad call is refused before any device is touched */
	unsigned long long total = 0;
	for(int i = 0; i < n_renders; ++i) {
		const gray_render_desc &d = descs[i];
		int st = gray_internal_check_desc(&d);
		if(st)
			return st;
		if(d.spacetime != GRAY_ST_KERR || d.n_freq != descs[0].n_freq ||
		   d.flow != descs[0].flow || !state_dev[i] || !info_dev[i])
			return GRAY_EINVAL;
		total += (unsigned long long)d.n_width * (d.n_rows ? d.n_rows : d.n_height);
	}
	if(total > (1ull << 31))
		return GRAY_EINVAL; /* the ray queue is a 32-bit counter */
	if(cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev ||
	   device >= MAX_DEVICES) {
		cudaGetLastError();
		return GRAY_ENODEV;
	}

	int prev = 0;
	cudaGetDevice(&prev);
	if(cudaSetDevice(device) != cudaSuccess)
		return GRAY_ENODEV;
	cudaStream_t st = (cudaStream_t)cuda_stream;
	NoallocScratch *S = nullptr;
	int sms = 0;
	cudaError_t e = scratch_for(device, &S);
	if(e == cudaSuccess)
		e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);

	/* host image of the render table and its prefix sums */
	MixedRender table[GRAY_NOALLOC_MAX_RENDERS];
	unsigned long long prefix[GRAY_NOALLOC_MAX_RENDERS];
	memset(table, 0, sizeof(table));
	unsigned long long acc = 0;
	int n_freq = descs[0].n_freq;
	for(int i = 0; i < n_renders && e == cudaSuccess; ++i) {
		RenderParams p;
		gray_internal_make_params(&descs[i], &p);
		e = launch_icond64(p, state_dev[i], info_dev[i], st);
		fill_mixed_render(p, state_dev[i], info_dev[i], descs[i].t_init, descs[i].dt_dump,
		                  (long long)descs[i].n_dump, (long long)descs[i].n_sub, &table[i]);
		prefix[i] = acc;
		acc += (unsigned long long)p.n_rays;
	}
	if(e == cudaSuccess)
		e = cudaMemcpyAsync(S->renders, table, sizeof(MixedRender) * n_renders,
		                    cudaMemcpyHostToDevice, st);
	if(e == cudaSuccess)
		e = cudaMemcpyAsync(S->prefix, prefix, sizeof(unsigned long long) * n_renders,
		                    cudaMemcpyHostToDevice, st);
	/* the array keeps the last call's contents: the step counter restarts
	 * at 0 here, the ray queue in launch_mixed_table */
	if(e == cudaSuccess)
		e = cudaMemsetAsync(&S->steps, 0, sizeof(S->steps), st);
	if(e == cudaSuccess) {
		MixedTable T;
		T.renders = S->renders;
		T.prefix = S->prefix;
		T.n_renders = n_renders;
		T.total = total;
		/* the context's default plan: one ray per thread, 256 threads */
		MixedLaunch cfg = {256, 0, sms, 1};
		e = launch_mixed_table(T, n_freq, &S->queue, &S->steps, st, cfg,
		                       n_renders == 1 ? &table[0] : nullptr);
	}
	if(e == cudaSuccess && steps_host) {
		unsigned long long v = 0;
		e = cudaMemcpyAsync(&v, &S->steps, sizeof(v), cudaMemcpyDeviceToHost, st);
		if(e == cudaSuccess)
			e = cudaStreamSynchronize(st);
		*steps_host = v;
	}
	cudaSetDevice(prev);
	return status_of(e);
}
