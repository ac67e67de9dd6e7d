/*
 * Continuous-batching render server.
 *
 * A scheduler thread owns two streams.  Each iteration it
 *   1. admits queued requests (FIFO) while the admitted state fits the HBM
 *      budget and the table has room: allocates their state and launches
 *      their camera initial conditions;
 *   2. builds one render table per kind -- analytic renders grouped by
 *      n_freq, numerical renders on the context's grid -- each entry with
 *      the next window of dump intervals, and runs one persistent launch
 *      per group (analytic on one stream, numerical on the other);
 *   3. advances the windows; renders whose last interval is done are copied
 *      to host memory and their device state freed, which lets queued
 *      requests in on the next iteration.
 * Requests therefore join while others are mid-render and their rays share
 * the persistent launches.  Every entry point but the scheduler's own work
 * takes the server mutex only briefly.
 */
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <utility>
#include <vector>

#include "ctx_internal.h"

namespace {

/* one table per kind and frequency count: analytic n_freq 0..8 are groups
 * 0..8, numerical n_freq 0..8 are groups 9..17 */
constexpr int NUM_GROUP = GRAY_MAX_FREQ + 1;
constexpr int GROUPS = 2 * NUM_GROUP;

double
now_s()
{
	using namespace std::chrono;
	static const steady_clock::time_point t0 = steady_clock::now();
	return duration<double>(steady_clock::now() - t0).count();
}

/* An allocator whose value-construction leaves the elements uninitialised:
 * a finished render's host buffers are overwritten by the device copy at
 * once, so zero-filling them first (over 100 MB for a 1024^2 render) would
 * only hold up the scheduler. */
template <typename T>
struct NoInit : std::allocator<T> {
	template <typename U>
	struct rebind {
		typedef NoInit<U> other;
	};
	NoInit() = default;
	template <typename U>
	NoInit(const NoInit<U> &) noexcept {}
	template <typename U, typename... A>
	void construct(U *p, A &&...a)
	{
		::new((void *)p) U(std::forward<A>(a)...);
	}
	template <typename U>
	void construct(U *p) noexcept
	{
		::new((void *)p) U;
	}
};

struct Request {
	uint64_t id = 0;
	gray_render_desc desc;
	RenderParams p;
	int state = GRAY_REQ_QUEUED;
	int status = GRAY_OK;
	double t_submit = 0, t_admit = 0, t_done = 0;
	double *d_data = nullptr, *d_info = nullptr;
	size_t bytes = 0;
	int next_dump = 0;
	int window = 0;  /* dump intervals of the current iteration */
	std::atomic<bool> cancel{false}; /* set by gray_serve_cancel, read by the scheduler */
	/* a finished render's state and info: a block of the server's pinned
	 * pool (hres, at hres_off) or, when the pool has no room, vectors */
	char *hres = nullptr;
	size_t hres_off = 0;
	std::vector<double, NoInit<double>> h_data, h_info;

	int group() const
	{
		return p.spacetime == GRAY_ST_NUMERICAL ? NUM_GROUP + p.n_freq : p.n_freq;
	}
	size_t data_count() const { return (size_t)p.n_rays * p.n_data; }
	size_t result_bytes() const { return (data_count() + (size_t)p.n_rays) * sizeof(double); }
	const double *res_data() const { return hres ? (const double *)hres : h_data.data(); }
	const double *res_info() const
	{
		return hres ? (const double *)hres + data_count() : h_info.data();
	}
};

/* Estimated seconds of one dump interval of a render on the shared device:
 * its steps per interval times the longer of one ray's step latency (a
 * small render's rays each run alone in a warp) and its rays' share of the
 * device's throughput.  The figures are B200 measurements of the mixed
 * kernels (analytic, numerical); they only size windows and never change a
 * result. */
constexpr double STEP_LATENCY_S[2] = {1.5e-6, 9e-6};
constexpr double STEP_COST_S[2] = {1.0 / 4.5e10, 1.0 / 1.4e10};
constexpr double MIN_ITER_S = 0.05;

/* steps of one ray per interval: the analytic cap |dt|/n_sub
 * (phys.cl:60-61; more near the horizon); the numerical spacetime's step
 * is min(|dt|/n_sub, 0.01) (dyst.cl:43-53 gives eps = 1) */
double
interval_steps(const Request *r)
{
	const double n_sub = (double)r->desc.n_sub;
	return r->p.spacetime == GRAY_ST_NUMERICAL
	           ? std::max(n_sub, std::fabs(r->desc.dt_dump) / 0.01)
	           : n_sub;
}

double
interval_s(const Request *r)
{
	const int k = r->p.spacetime == GRAY_ST_NUMERICAL ? 1 : 0;
	return interval_steps(r) *
	       std::max(STEP_LATENCY_S[k], (double)r->p.n_rays * STEP_COST_S[k]);
}

} /* namespace */

struct Server {
	gray_ctx *c = nullptr;
	gray_serve_config cfg;
	size_t budget = 0;
	std::thread th;
	std::mutex mu;
	std::condition_variable cv;
	bool stop = false, drain = false;
	std::deque<Request *> pending;
	std::map<uint64_t, Request *> reqs;
	std::vector<Request *> inflight;
	size_t inflight_bytes = 0;
	uint64_t next_id = 1;
	gray_serve_stats stats;
	/* device: table | prefix | 2 counters per group */
	void *dblock = nullptr;
	/* the requests' device state: stream-ordered allocations from a pool
	 * that keeps its memory, so admitting and retiring a render neither
	 * maps nor unmaps HBM nor synchronises the device (cudaMalloc and
	 * cudaFree of large states stalled the scheduler for up to a second) */
	cudaMemPool_t pool = nullptr;
	/* pinned host pool for finished renders' results: the scheduler's copy
	 * out of HBM then runs at full speed into memory that is already
	 * mapped, instead of faulting in fresh pageable pages (which stalled
	 * every other request for up to a second per large render) */
	char *hpool = nullptr;
	size_t hpool_bytes = 0;
	std::map<size_t, size_t> hfree; /* offset -> bytes of each free block */
	size_t dbytes = 0;
	MixedRender *d_tab = nullptr;
	unsigned long long *d_pre = nullptr;
	unsigned int *d_queue = nullptr;          /* [GROUPS] (64-byte spaced) */
	unsigned long long *d_steps = nullptr;    /* [GROUPS] */
	MixedRender *h_tab = nullptr;             /* pinned staging */
	unsigned long long *h_pre = nullptr;
	unsigned long long *h_steps = nullptr;
	cudaStream_t s[2] = {nullptr, nullptr};
	cudaEvent_t copied = nullptr, e0 = nullptr, e1 = nullptr, e2 = nullptr;
	int thread_status = GRAY_OK;
};

namespace {

constexpr size_t HPOOL_BYTES = size_t(2) << 30;

size_t
pool_round(size_t bytes)
{
	return (bytes + 255) & ~size_t(255);
}

/* First fit in the pinned pool (S->mu held); nullptr when nothing fits. */
char *
pool_take(Server *S, size_t bytes, size_t *off)
{
	bytes = pool_round(bytes);
	for(auto it = S->hfree.begin(); it != S->hfree.end(); ++it) {
		if(it->second < bytes)
			continue;
		const size_t at = it->first, rest = it->second - bytes;
		S->hfree.erase(it);
		if(rest) {
			try {
				S->hfree[at + bytes] = rest;
			} catch(const std::bad_alloc &) {
				/* the remainder is lost to the pool until the server stops */
			}
		}
		*off = at;
		return S->hpool + at;
	}
	return nullptr;
}

/* Return a block to the pool, merged with free neighbours (S->mu held). */
void
pool_give(Server *S, size_t off, size_t bytes)
{
	bytes = pool_round(bytes);
	auto next = S->hfree.lower_bound(off);
	if(next != S->hfree.end() && off + bytes == next->first) {
		bytes += next->second;
		next = S->hfree.erase(next);
	}
	if(next != S->hfree.begin()) {
		auto prev = std::prev(next);
		if(prev->first + prev->second == off) {
			prev->second += bytes;
			return;
		}
	}
	try {
		S->hfree[off] = bytes;
	} catch(const std::bad_alloc &) {
		/* lost to the pool until the server stops */
	}
}

void
release(Server *S, Request *r)
{
	if(r->d_data) {
		cudaFreeAsync(r->d_data, S->s[0]); /* after the stream's copies of it */
		gi_unreserve(S->c, r->bytes);
		r->d_data = r->d_info = nullptr;
		S->inflight_bytes -= r->bytes;
	}
}

/* The SMs of the two kinds' persistent launches, which run at the same
 * time on their two streams.  Each launch sizes its grid to its SM count,
 * so with both kinds in flight neither grid takes the whole device and the
 * other kind's launch does not wait for it to drain.  While the numerical
 * renders' rays fit on at most half the SMs at once (2 blocks of 256 per
 * SM), they get the SMs that hold them all: their windows were sized for
 * rays that run at once.  Otherwise the SMs are split by the kinds'
 * estimated work this iteration. */
void
split_sms(const Server *S, const unsigned long long *total, int *ana_sms, int *num_sms)
{
	const int sms = S->c->sms;
	double work[2] = {0.0, 0.0};
	for(const Request *r : S->inflight)
		work[r->p.spacetime == GRAY_ST_NUMERICAL ? 1 : 0] += r->window * interval_s(r);
	unsigned long long blocks = 0;
	for(int g = NUM_GROUP; g < GROUPS; ++g)
		blocks += (total[g] + 255) / 256;
	*ana_sms = *num_sms = sms;
	if(work[0] <= 0.0 || work[1] <= 0.0 || sms < 2)
		return;
	int n = (int)std::min<unsigned long long>((blocks + 1) / 2, (unsigned long long)sms);
	if(n > sms / 2)
		n = (int)std::lround(sms * work[1] / (work[0] + work[1]));
	n = std::max(1, std::min(sms - 1, n));
	*num_sms = n;
	*ana_sms = sms - n;
}

/* Device-side work of one iteration.  Returns a GRAY_* status. */
int
iterate(Server *S, std::vector<Request *> &fresh)
{
	gray_ctx *c = S->c;
	cudaError_t e = cudaSuccess;
	/* 1. admission: state + initial conditions of the fresh requests */
	for(Request *r : fresh) {
		/* on the stream of its kind's launches, which use it first; the
		 * retiring copies on s[0] wait for s[1] */
		cudaStream_t st_ = S->s[r->group() >= NUM_GROUP ? 1 : 0];
		int st = gi_reserve(c, r->bytes);
		if(!st && cudaMallocFromPoolAsync((void **)&r->d_data, r->bytes, S->pool, st_) !=
		              cudaSuccess) {
			cudaGetLastError();
			gi_unreserve(c, r->bytes);
			st = GRAY_ENOMEM;
		}
		if(st) {
			std::lock_guard<std::mutex> lk(S->mu);
			r->state = GRAY_REQ_FAILED;
			r->status = st;
			r->t_done = now_s();
			S->inflight_bytes -= r->bytes;
			r->d_data = nullptr;
			S->stats.failed++;
			continue;
		}
		r->d_info = r->d_data + (size_t)r->p.n_rays * r->p.n_data;
		r->next_dump = 0;
		/* in flight before its first launch, so that a failure below frees
		 * it with the rest (the capacity was reserved at start) */
		S->inflight.push_back(r);
		e = r->group() >= NUM_GROUP
		        ? launch_dyst_icond(r->p, c->grid->gp, r->d_data, r->d_info, st_)
		        : launch_icond64(r->p, r->d_data, r->d_info, st_);
		if(e != cudaSuccess)
			return gi_from_cuda(e);
	}
	if(S->inflight.empty())
		return GRAY_OK;

	/* 2. one table per group, entries with the next window of dumps.  The
	 * iteration lasts dumps_per_iter intervals of the admitted render with
	 * the longest estimated interval (and at least MIN_ITER_S); every render
	 * advances as many intervals as fit in that time (at most the ones it
	 * has left), so small renders finish in an iteration or two while a
	 * newcomer waits at most about one iteration for admission */
	const int dpi = S->cfg.dumps_per_iter;
	double t_iter = MIN_ITER_S;
	for(Request *r : S->inflight)
		t_iter = std::max(t_iter, dpi * interval_s(r));
	for(Request *r : S->inflight) {
		const double w = t_iter / interval_s(r);
		const int left = (int)r->desc.n_dump - r->next_dump;
		/* left = 0 (no dump intervals): an empty window, the render is done */
		r->window = left <= 0 ? 0 : (w < (double)left ? std::max(dpi, (int)w) : left);
	}
	int count[GROUPS] = {0}, start[GROUPS];
	for(Request *r : S->inflight)
		count[r->group()]++;
	for(int g = 0, acc = 0; g < GROUPS; ++g) {
		start[g] = acc;
		acc += count[g];
	}
	int fill[GROUPS];
	unsigned long long total[GROUPS] = {0};
	memcpy(fill, start, sizeof(fill));
	/* within a group, the renders whose rays take longest this iteration
	 * (window x steps per interval) first in the queue: a small render's
	 * few long rays then start with the iteration instead of after a large
	 * render's many short ones (longest processing time first) */
	std::vector<Request *> order(S->inflight);
	std::stable_sort(order.begin(), order.end(), [](const Request *a, const Request *b) {
		return a->window * interval_steps(a) > b->window * interval_steps(b);
	});
	for(Request *r : order) {
		int g = r->group(), k = fill[g]++;
		MixedRender &m = S->h_tab[k];
		memset(&m, 0, sizeof(m));
		fill_mixed_render(r->p, r->d_data, r->d_info, r->desc.t_init, r->desc.dt_dump,
		                  (long long)r->desc.n_dump, (long long)r->desc.n_sub, &m);
		m.dump_begin = r->next_dump;
		m.dump_end = r->next_dump + r->window;
		S->h_pre[k] = total[g];
		total[g] += (unsigned long long)r->p.n_rays;
	}
	const size_t n = S->inflight.size();
	if((e = cudaMemcpyAsync(S->d_tab, S->h_tab, n * sizeof(MixedRender), cudaMemcpyHostToDevice,
	                        S->s[0])) != cudaSuccess ||
	   (e = cudaMemcpyAsync(S->d_pre, S->h_pre, n * sizeof(unsigned long long),
	                        cudaMemcpyHostToDevice, S->s[0])) != cudaSuccess ||
	   (e = cudaMemsetAsync(S->d_steps, 0, GROUPS * sizeof(unsigned long long), S->s[0])) !=
	       cudaSuccess ||
	   (e = cudaEventRecord(S->copied, S->s[0])) != cudaSuccess ||
	   (e = cudaStreamWaitEvent(S->s[1], S->copied, 0)) != cudaSuccess ||
	   (e = cudaEventRecord(S->e0, S->s[0])) != cudaSuccess)
		return gi_from_cuda(e);
	MixedLaunch cfg = c->mixed;
	cfg.sms = c->sms;
	int num_sms = c->sms;
	split_sms(S, total, &cfg.sms, &num_sms);
	for(int g = 0; g < GROUPS; ++g) {
		if(!count[g])
			continue;
		MixedTable T;
		T.renders = S->d_tab + start[g];
		T.prefix = S->d_pre + start[g];
		T.n_renders = count[g];
		T.total = total[g];
		unsigned int *q = (unsigned int *)((char *)S->d_queue + 64 * g);
		if(g >= NUM_GROUP) {
			MixedLaunch dc = cfg;
			dc.block = 256;
			dc.sms = num_sms;
			e = launch_dyst_mixed_table(T, c->grid->gp, g - NUM_GROUP, q, S->d_steps + g,
			                            S->s[1], dc);
		} else {
			e = launch_mixed_table(T, g, q, S->d_steps + g, S->s[0], cfg,
			                       count[g] == 1 ? &S->h_tab[start[g]] : nullptr);
		}
		if(e != cudaSuccess)
			return gi_from_cuda(e);
	}
	if((e = cudaEventRecord(S->e2, S->s[1])) != cudaSuccess ||
	   (e = cudaStreamWaitEvent(S->s[0], S->e2, 0)) != cudaSuccess ||
	   (e = cudaEventRecord(S->e1, S->s[0])) != cudaSuccess ||
	   (e = cudaMemcpyAsync(S->h_steps, S->d_steps, GROUPS * sizeof(unsigned long long),
	                        cudaMemcpyDeviceToHost, S->s[0])) != cudaSuccess ||
	   (e = cudaStreamSynchronize(S->s[0])) != cudaSuccess)
		return gi_from_cuda(e);
	float ms = 0.0f;
	cudaEventElapsedTime(&ms, S->e0, S->e1);

	/* 3. advance windows, retire finished renders */
	std::vector<Request *> keep, done;
	for(Request *r : S->inflight) {
		r->next_dump += r->window;
		if(r->next_dump >= (int)r->desc.n_dump || r->cancel)
			done.push_back(r);
		else
			keep.push_back(r);
	}
	for(Request *r : done) {
		if(!r->cancel) {
			const size_t nr = (size_t)r->p.n_rays, nd = r->data_count();
			{
				std::lock_guard<std::mutex> lk(S->mu);
				if(S->hpool)
					r->hres = pool_take(S, r->result_bytes(), &r->hres_off);
			}
			double *hd, *hi;
			if(r->hres) {
				hd = (double *)r->hres;
				hi = hd + nd;
			} else {
				r->h_data.resize(nd);
				r->h_info.resize(nr);
				hd = r->h_data.data();
				hi = r->h_info.data();
			}
			if((e = cudaMemcpyAsync(hd, r->d_data, nd * sizeof(double), cudaMemcpyDeviceToHost,
			                        S->s[0])) != cudaSuccess ||
			   (e = cudaMemcpyAsync(hi, r->d_info, nr * sizeof(double), cudaMemcpyDeviceToHost,
			                        S->s[0])) != cudaSuccess ||
			   (e = cudaStreamSynchronize(S->s[0])) != cudaSuccess)
				return gi_from_cuda(e);
		}
		std::lock_guard<std::mutex> lk(S->mu);
		release(S, r);
		r->t_done = now_s();
		if(r->cancel) {
			r->state = GRAY_REQ_CANCELLED;
			S->stats.cancelled++;
		} else {
			r->state = GRAY_REQ_DONE;
			S->stats.completed++;
		}
	}
	{
		std::lock_guard<std::mutex> lk(S->mu);
		S->inflight.swap(keep);
		S->stats.iterations++;
		S->stats.busy_s += ms * 1e-3;
		for(int g = 0; g < GROUPS; ++g)
			S->stats.ray_steps[g >= NUM_GROUP ? 1 : 0] += S->h_steps[g];
	}
	S->cv.notify_all();
	return GRAY_OK;
}

void
loop(Server *S)
{
	cudaSetDevice(S->c->device);
	for(;;) {
		std::vector<Request *> fresh;
		try { /* admission below never grows it past this */
			fresh.reserve((size_t)S->cfg.max_inflight);
		} catch(const std::bad_alloc &) {
			std::this_thread::sleep_for(std::chrono::milliseconds(20));
			continue;
		}
		{
			std::unique_lock<std::mutex> lk(S->mu);
			if(S->inflight.empty())
				S->cv.wait_for(lk, std::chrono::milliseconds(20), [&] {
					return S->stop || !S->pending.empty();
				});
			if(S->stop && (!S->drain || (S->pending.empty() && S->inflight.empty())))
				break;
			/* FIFO admission under the budget and the table size */
			size_t slots = S->inflight.size();
			while(!S->pending.empty() && slots < (size_t)S->cfg.max_inflight) {
				Request *r = S->pending.front();
				if(r->cancel) {
					S->pending.pop_front();
					r->state = GRAY_REQ_CANCELLED;
					r->t_done = now_s();
					S->stats.cancelled++;
					continue;
				}
				if(S->inflight_bytes + r->bytes > S->budget)
					break; /* wait until running renders free memory */
				S->pending.pop_front();
				S->inflight_bytes += r->bytes;
				r->state = GRAY_REQ_RUNNING;
				r->t_admit = now_s();
				fresh.push_back(r);
				++slots;
			}
		}
		int st;
		try { /* a failed host allocation ends serving like a device error */
			st = iterate(S, fresh);
		} catch(const std::bad_alloc &) {
			st = GRAY_ENOMEM;
		}
		if(st) {
			/* device failure: fail everything in flight and stop serving */
			std::lock_guard<std::mutex> lk(S->mu);
			S->thread_status = st;
			for(Request *r : S->inflight) {
				release(S, r);
				if(r->state != GRAY_REQ_RUNNING)
					continue; /* retired (done or cancelled) before the failure */
				r->state = GRAY_REQ_FAILED;
				r->status = st;
				S->stats.failed++;
			}
			S->inflight.clear();
			/* admitted this iteration but not reached before the failure */
			for(Request *r : fresh) {
				if(r->state != GRAY_REQ_RUNNING)
					continue;
				S->inflight_bytes -= r->bytes;
				r->state = GRAY_REQ_FAILED;
				r->status = st;
				S->stats.failed++;
			}
			for(Request *r : S->pending) {
				r->state = GRAY_REQ_FAILED;
				r->status = st;
				S->stats.failed++;
			}
			S->pending.clear();
			S->stop = true;
			break;
		}
	}
	S->cv.notify_all();
}

void
free_server(Server *S)
{
	gray_ctx *c = S->c;
	for(Request *r : S->inflight)
		release(S, r);
	for(int i = 0; i < 2; ++i)
		if(S->s[i])
			cudaStreamSynchronize(S->s[i]);
	if(S->pool)
		cudaMemPoolDestroy(S->pool);
	for(auto &kv : S->reqs)
		delete kv.second;
	if(S->dblock)
		gi_dfree(c, S->dblock, S->dbytes);
	if(S->h_tab)
		cudaFreeHost(S->h_tab);
	if(S->hpool) /* after the requests whose results it held */
		cudaFreeHost(S->hpool);
	for(int i = 0; i < 2; ++i)
		if(S->s[i])
			cudaStreamDestroy(S->s[i]);
	if(S->copied) cudaEventDestroy(S->copied);
	if(S->e0) cudaEventDestroy(S->e0);
	if(S->e1) cudaEventDestroy(S->e1);
	if(S->e2) cudaEventDestroy(S->e2);
	delete S;
}

} /* namespace */

void
gi_serve_shutdown(gray_ctx *c)
{
	if(!c || !c->server)
		return;
	Server *S = c->server;
	{
		std::lock_guard<std::mutex> lk(S->mu);
		S->stop = true;
		S->drain = false;
	}
	S->cv.notify_all();
	if(S->th.joinable())
		S->th.join();
	free_server(S);
	c->server = nullptr;
}

extern "C" double
gray_serve_clock(void)
{
	return now_s();
}

extern "C" int
gray_serve_start(gray_ctx *c, const gray_serve_config *cfg)
{
	if(!c || !cfg)
		return GRAY_EINVAL;
	if(c->server)
		return GRAY_ESTATE;
	if(cfg->max_inflight < 0 || cfg->dumps_per_iter < 0 || cfg->max_inflight > (1 << 16))
		return GRAY_EINVAL;
	if(cudaSetDevice(c->device) != cudaSuccess)
		return GRAY_ECUDA;
	Server *S = new(std::nothrow) Server;
	if(!S)
		return GRAY_ENOMEM;
	S->c = c;
	S->cfg = *cfg;
	if(!S->cfg.max_inflight)
		S->cfg.max_inflight = 1024;
	if(!S->cfg.dumps_per_iter)
		S->cfg.dumps_per_iter = 1;
	S->budget = cfg->hbm_budget ? cfg->hbm_budget : c->budget;
	memset(&S->stats, 0, sizeof(S->stats));
	const size_t n = (size_t)S->cfg.max_inflight;
	const size_t tab = (n * sizeof(MixedRender) + 255) / 256 * 256;
	const size_t pre = (n * sizeof(unsigned long long) + 255) / 256 * 256;
	const size_t cnt = 64 * GROUPS + 8 * GROUPS;
	S->dbytes = tab + pre + cnt + 256;
	int st = gi_dalloc(c, &S->dblock, S->dbytes);
	cudaError_t e = cudaSuccess;
	if(!st) {
		S->d_tab = (MixedRender *)S->dblock;
		S->d_pre = (unsigned long long *)((char *)S->dblock + tab);
		S->d_queue = (unsigned int *)((char *)S->dblock + tab + pre);
		S->d_steps = (unsigned long long *)((char *)S->dblock + tab + pre + 64 * GROUPS);
		void *h = nullptr;
		e = cudaMallocHost(&h, tab + pre + 8 * GROUPS);
		if(e == cudaSuccess) {
			S->h_tab = (MixedRender *)h;
			S->h_pre = (unsigned long long *)((char *)h + tab);
			S->h_steps = (unsigned long long *)((char *)h + tab + pre);
		}
		if(e == cudaSuccess) {
			/* the result pool; without it results go to pageable memory */
			S->hpool_bytes = std::min(HPOOL_BYTES, pool_round(S->budget));
			if(cudaHostAlloc((void **)&S->hpool, S->hpool_bytes, cudaHostAllocDefault) ==
			   cudaSuccess) {
				try {
					S->hfree[0] = S->hpool_bytes;
				} catch(const std::bad_alloc &) {
					cudaFreeHost(S->hpool);
					S->hpool = nullptr;
				}
			} else {
				cudaGetLastError();
				S->hpool = nullptr;
			}
		}
		if(e == cudaSuccess) {
			cudaMemPoolProps pp;
			memset(&pp, 0, sizeof(pp));
			pp.allocType = cudaMemAllocationTypePinned;
			pp.location.type = cudaMemLocationTypeDevice;
			pp.location.id = c->device;
			e = cudaMemPoolCreate(&S->pool, &pp);
			uint64_t keep = UINT64_MAX; /* the budget bounds what it holds */
			if(e == cudaSuccess)
				e = cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep);
		}
		for(int i = 0; i < 2 && e == cudaSuccess; ++i)
			e = cudaStreamCreateWithFlags(&S->s[i], cudaStreamNonBlocking);
		if(e == cudaSuccess) e = cudaEventCreateWithFlags(&S->copied, cudaEventDisableTiming);
		if(e == cudaSuccess) e = cudaEventCreate(&S->e0);
		if(e == cudaSuccess) e = cudaEventCreate(&S->e1);
		if(e == cudaSuccess) e = cudaEventCreateWithFlags(&S->e2, cudaEventDisableTiming);
		if(e != cudaSuccess)
			st = gi_from_cuda(e);
	}
	if(st) {
		free_server(S);
		return st;
	}
	c->server = S;
	try {
		S->inflight.reserve(n); /* admission never grows it past this */
		S->th = std::thread(loop, S);
	} catch(...) {
		c->server = nullptr;
		free_server(S);
		return GRAY_ENOMEM;
	}
	return GRAY_OK;
}

extern "C" int
gray_serve_submit(gray_ctx *c, const gray_render_desc *d, uint64_t *id)
{
	if(!c || !c->server || !id)
		return c && !c->server ? GRAY_ESTATE : GRAY_EINVAL;
	int st = gray_internal_check_desc(d);
	if(st)
		return st;
	if(d->precision != GRAY_PREC_MIXED)
		return GRAY_EINVAL; /* the server runs the mixed-precision kernels */
	if(d->spacetime == GRAY_ST_NUMERICAL && !gi_grid_ready(c))
		return GRAY_ESTATE;
	if(d->n_dump > (uint64_t)INT32_MAX)
		return GRAY_EINVAL;
	Request *r = new(std::nothrow) Request;
	if(!r)
		return GRAY_ENOMEM;
	r->desc = *d;
	gray_internal_make_params(d, &r->p);
	r->bytes = (size_t)r->p.n_rays * (r->p.n_data + 1) * sizeof(double);
	Server *S = c->server;
	{
		std::lock_guard<std::mutex> lk(S->mu);
		if(S->stop) {
			delete r;
			return GRAY_ESTATE;
		}
		r->id = S->next_id;
		r->t_submit = now_s();
		try { /* no exception may cross the C ABI */
			S->reqs[r->id] = r;
			if(r->bytes <= S->budget)
				S->pending.push_back(r);
		} catch(const std::bad_alloc &) {
			S->reqs.erase(r->id);
			delete r;
			return GRAY_ENOMEM;
		}
		++S->next_id;
		if(r->bytes > S->budget) { /* can never be admitted */
			r->state = GRAY_REQ_FAILED;
			r->status = GRAY_EBUDGET;
			r->t_done = r->t_submit;
			S->stats.failed++;
		}
		*id = r->id;
	}
	S->cv.notify_all();
	return GRAY_OK;
}

extern "C" int
gray_serve_poll(gray_ctx *c, uint64_t id, gray_request_status *out)
{
	if(!c || !out)
		return GRAY_EINVAL;
	if(!c->server)
		return GRAY_ESTATE;
	Server *S = c->server;
	std::lock_guard<std::mutex> lk(S->mu);
	auto it = S->reqs.find(id);
	if(it == S->reqs.end())
		return GRAY_ENOTFOUND;
	const Request *r = it->second;
	out->state = r->state;
	out->status = r->status;
	out->t_submit = r->t_submit;
	out->t_admit = r->t_admit;
	out->t_done = r->t_done;
	out->n_rays = (uint64_t)r->p.n_rays;
	return GRAY_OK;
}

extern "C" int
gray_serve_result(gray_ctx *c, uint64_t id, void *data, size_t data_bytes, void *info,
                  size_t info_bytes)
{
	if(!c)
		return GRAY_EINVAL;
	if(!c->server)
		return GRAY_ESTATE;
	Server *S = c->server;
	Request *r = nullptr;
	{
		std::lock_guard<std::mutex> lk(S->mu);
		auto it = S->reqs.find(id);
		if(it == S->reqs.end())
			return GRAY_ENOTFOUND;
		r = it->second;
		if(r->state == GRAY_REQ_QUEUED || r->state == GRAY_REQ_RUNNING)
			return GRAY_ESTATE;
		if(r->state == GRAY_REQ_DONE) {
			if(data && data_bytes != r->data_count() * sizeof(double))
				return GRAY_ESIZE;
			if(info && info_bytes != (size_t)r->p.n_rays * sizeof(double))
				return GRAY_ESIZE;
		}
		S->reqs.erase(it); /* the request is this caller's from here on */
	}
	/* the copies run without the server mutex: the scheduler never waits
	 * for a client's memcpy */
	if(r->state == GRAY_REQ_DONE) {
		if(data)
			memcpy(data, r->res_data(), data_bytes);
		if(info)
			memcpy(info, r->res_info(), info_bytes);
	}
	int st = r->state == GRAY_REQ_DONE ? GRAY_OK
	         : r->state == GRAY_REQ_FAILED ? (r->status ? r->status : GRAY_ECUDA)
	                                        : GRAY_ESTATE;
	if(r->hres) {
		std::lock_guard<std::mutex> lk(S->mu);
		pool_give(S, r->hres_off, r->result_bytes());
	}
	delete r;
	return st;
}

extern "C" int
gray_serve_cancel(gray_ctx *c, uint64_t id)
{
	if(!c)
		return GRAY_EINVAL;
	if(!c->server)
		return GRAY_ESTATE;
	Server *S = c->server;
	std::lock_guard<std::mutex> lk(S->mu);
	auto it = S->reqs.find(id);
	if(it == S->reqs.end())
		return GRAY_ENOTFOUND;
	it->second->cancel = true; /* retired at the next iteration boundary */
	S->cv.notify_all();
	return GRAY_OK;
}

extern "C" int
gray_serve_get_stats(gray_ctx *c, gray_serve_stats *out)
{
	if(!c || !out)
		return GRAY_EINVAL;
	if(!c->server)
		return GRAY_ESTATE;
	std::lock_guard<std::mutex> lk(c->server->mu);
	*out = c->server->stats;
	return c->server->thread_status;
}

extern "C" int
gray_serve_stop(gray_ctx *c, int drain)
{
	if(!c)
		return GRAY_EINVAL;
	if(!c->server)
		return GRAY_ESTATE;
	Server *S = c->server;
	{
		std::lock_guard<std::mutex> lk(S->mu);
		S->stop = true;
		S->drain = drain != 0;
	}
	S->cv.notify_all();
	if(S->th.joinable())
		S->th.join();
	int st = S->thread_status;
	free_server(S);
	c->server = nullptr;
	return st;
}
