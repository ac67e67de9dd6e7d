/*
 * Dynamic spacetimes: a render integrated across a time series of grid
 * snapshots, the "slow light" loop of sim-org/gray.c:147-294.
 *
 * The reference reads each snapshot pair from HDF5 into two image sets and,
 * when a dump time leaves the pair, copies one set over the other and reads
 * the next snapshot, all between dumps with the device idle.  Here the pair
 * sequence is known before the first interval (it depends only on the
 * times), so the snapshot the next interval needs is read by the caller's
 * loader and copied to the device on a second stream while the current
 * interval runs, into a third device level.  Moving the pair by one
 * snapshot relabels the levels instead of copying 51 fields.
 */
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx_internal.h"

namespace {

/* sim-org/gray.c:41-57: the first k with times[k] <= t <= times[k+1]
 * (-1 when there is none; the reference would read past the series) */
int64_t
find_snapshot(const double *times, uint64_t n, double t)
{
	for(uint64_t k = 0; k + 1 < n; ++k)
		if(t >= times[k] && t <= times[k + 1])
			return (int64_t)k;
	return -1;
}

/* sim-org/gray.c:183-293: the pair of every interval and of t_init */
int
schedule(const double *times, uint64_t n, double t_init, double dt_dump, uint64_t n_dump,
         int fast_light, int64_t *first, int64_t *pairs, bool *frozen)
{
	if(!times || n == 0 || (n_dump && !pairs))
		return GRAY_EINVAL;
	for(uint64_t k = 0; k < n; ++k)
		if(!std::isfinite(times[k]) || (k && !(times[k] > times[k - 1])))
			return GRAY_EINVAL;
	if(!std::isfinite(t_init) || !std::isfinite(dt_dump))
		return GRAY_EINVAL;
	int64_t snap;
	*frozen = n == 1 || fast_light;
	if(n == 1) {
		snap = 0;
	} else if(fast_light) {
		snap = find_snapshot(times, n, t_init);
	} else {
		/* sim-org/gray.c:193-205 (i_init = 0) */
		const double lo = times[0], hi = times[n - 1];
		const double t_final = t_init + dt_dump * (double)n_dump;
		if(t_init < lo || t_init > hi || t_final < lo || t_final > hi)
			return GRAY_EINVAL;
		snap = find_snapshot(times, n, t_init);
	}
	if(snap < 0)
		return GRAY_EINVAL;
	*first = snap;
	for(uint64_t i = 0; i < n_dump;) {
		pairs[i] = snap;
		const double target = t_init + (double)(++i) * dt_dump;
		if(!*frozen && (target < times[snap] || target > times[snap + 1])) {
			snap = find_snapshot(times, n, target);
			if(snap < 0)
				return GRAY_EINVAL;
		}
	}
	return GRAY_OK;
}

/* The three device levels of a series run and what each holds. */
struct Levels {
	gray_ctx *c;
	const gray_snapshot_source *src;
	size_t npts;
	float *buf[3];
	int64_t held[3];
	cudaEvent_t ready[3];    /* the copy that filled buf[b]              */
	cudaStream_t copy = nullptr;
	cudaEvent_t staged = nullptr; /* the last copy out of the staging    */
	uint64_t loads = 0;

	int find(int64_t k) const
	{
		for(int b = 0; b < 3; ++b)
			if(held[b] == k)
				return b;
		return -1;
	}

	/* Read snapshot k into the staging buffer and copy it into level b on
	 * the copy stream, after `after` (the compute work that may still read
	 * level b).  The loader runs on this thread while the GPU computes. */
	int load(int b, int64_t k, cudaEvent_t after)
	{
		cudaError_t e = cudaEventSynchronize(staged); /* staging free again */
		if(e != cudaSuccess)
			return gi_from_cuda(e);
		held[b] = -1;
		if(src->load(src->user, (uint64_t)k, c->grid->staging) != 0)
			return GRAY_ESOURCE;
		++loads;
		if(after && (e = cudaStreamWaitEvent(copy, after, 0)) != cudaSuccess)
			return gi_from_cuda(e);
		e = cudaMemcpy2DAsync(buf[b], GRAY_NSTRIDE * sizeof(float), c->grid->staging,
		                      GRAY_NCOMP * sizeof(float), GRAY_NCOMP * sizeof(float), npts,
		                      cudaMemcpyHostToDevice, copy);
		if(e == cudaSuccess)
			e = cudaEventRecord(ready[b], copy);
		if(e == cudaSuccess)
			e = cudaEventRecord(staged, copy);
		if(e != cudaSuccess)
			return gi_from_cuda(e);
		held[b] = k;
		return GRAY_OK;
	}

	/* A level not holding any of the snapshots in keep[0..nk) */
	int free_level(const int64_t *keep, int nk) const
	{
		for(int b = 0; b < 3; ++b) {
			bool used = false;
			for(int j = 0; j < nk; ++j)
				used |= held[b] == keep[j];
			if(!used)
				return b;
		}
		return -1;
	}

	/* Make snapshots k (and k + 1 unless frozen) resident, order the
	 * compute stream after their copies and point the grid at them. */
	int use_pair(int64_t k, bool frozen, const double *times)
	{
		const int64_t need[2] = {k, k + 1};
		const int nn = frozen ? 1 : 2;
		for(int j = 0; j < nn; ++j) {
			if(find(need[j]) >= 0)
				continue;
			int b = free_level(need, nn);
			/* the level may still be read by work already on the stream */
			cudaEvent_t after = nullptr;
			cudaError_t e = cudaEventCreateWithFlags(&after, cudaEventDisableTiming);
			if(e == cudaSuccess)
				e = cudaEventRecord(after, c->stream);
			if(e != cudaSuccess) {
				if(after)
					cudaEventDestroy(after);
				return gi_from_cuda(e);
			}
			int st = load(b, need[j], after);
			cudaEventDestroy(after);
			if(st)
				return st;
		}
		int b0 = find(need[0]), b1 = frozen ? b0 : find(need[1]);
		cudaError_t e = cudaStreamWaitEvent(c->stream, ready[b0], 0);
		if(e == cudaSuccess && b1 != b0)
			e = cudaStreamWaitEvent(c->stream, ready[b1], 0);
		if(e != cudaSuccess)
			return gi_from_cuda(e);
		GridParams &gp = c->grid->gp;
		gp.lvl[0] = buf[b0];
		gp.lvl[1] = buf[b1];
		gp.box[0] = frozen ? 0.0f : (float)times[k];
		gp.box[4] = frozen ? 0.0f : (float)times[k + 1];
		gp.single = frozen ? 1 : gp.box[0] == gp.box[4];
		return GRAY_OK;
	}
};

} /* namespace */

extern "C" int
gray_series_schedule(const double *times, uint64_t n_times, double t_init, double dt_dump,
                     uint64_t n_dump, int fast_light, int64_t *pairs)
{
	int64_t first;
	bool frozen;
	return schedule(times, n_times, t_init, dt_dump, n_dump, fast_light, &first, pairs,
	                &frozen);
}

extern "C" int
gray_run_series(gray_ctx *c, int id, const gray_grid_desc *gd,
                const gray_snapshot_source *src, int fast_light,
                int (*after_dump)(void *user, uint64_t i), double *ns, uint64_t *loads)
{
	if(loads)
		*loads = 0;
	Render *r = gi_find_render(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	if(!gd || !src || !src->load || !src->times)
		return GRAY_EINVAL;
	if(r->p.spacetime != GRAY_ST_NUMERICAL)
		return GRAY_EINVAL;
	if(c->server)
		return GRAY_ESTATE; /* the server's renders read the grid */
	const gray_render_desc &d = r->desc;
	std::vector<int64_t> pairs;
	try { /* no exception may cross the C ABI */
		pairs.resize(d.n_dump ? d.n_dump : 1);
	} catch(const std::exception &) {
		return GRAY_ENOMEM;
	}
	int64_t first;
	bool frozen;
	int st = schedule(src->times, src->n_times, d.t_init, d.dt_dump, d.n_dump, fast_light,
	                  &first, pairs.data(), &frozen);
	if(st)
		return st;
	gray_grid_desc g2 = *gd;
	g2.box[0] = g2.box[4] = 0.0f;
	if((st = gi_check_grid(&g2)) != GRAY_OK)
		return st;
	cudaError_t e = cudaSetDevice(c->device);
	if(e != cudaSuccess)
		return gi_from_cuda(e);
	if((st = gi_ensure_grid(c, &g2)) != GRAY_OK)
		return st;
	Grid *g = c->grid;
	const size_t npts = (size_t)gd->nx * gd->ny * gd->nz;
	const size_t level_bytes = npts * GRAY_NSTRIDE * sizeof(float);
	if(!g->spare && (st = gi_dalloc(c, (void **)&g->spare, level_bytes)) != GRAY_OK)
		return st;
	if(!g->staging &&
	   cudaMallocHost((void **)&g->staging, npts * GRAY_NCOMP * sizeof(float)) != cudaSuccess) {
		g->staging = nullptr;
		return GRAY_ENOMEM;
	}

	Levels L;
	L.c = c;
	L.src = src;
	L.npts = npts;
	L.buf[0] = g->lvl[0];
	L.buf[1] = g->lvl[1];
	L.buf[2] = g->spare;
	for(int b = 0; b < 3; ++b) {
		L.held[b] = -1; /* what an earlier load left there is not known */
		L.ready[b] = nullptr;
	}
	cudaEvent_t before = nullptr; /* recorded before each interval's launch */
	e = cudaStreamCreateWithFlags(&L.copy, cudaStreamNonBlocking);
	for(int b = 0; b < 3 && e == cudaSuccess; ++b)
		e = cudaEventCreateWithFlags(&L.ready[b], cudaEventDisableTiming);
	if(e == cudaSuccess)
		e = cudaEventCreateWithFlags(&L.staged, cudaEventDisableTiming);
	if(e == cudaSuccess)
		e = cudaEventCreateWithFlags(&before, cudaEventDisableTiming);
	if(e == cudaSuccess)
		e = cudaEventRecord(L.staged, L.copy);
	st = e == cudaSuccess ? GRAY_OK : gi_from_cuda(e);

	if(!st)
		st = gi_timed_begin(c);
	if(!st)
		st = L.use_pair(first, frozen, src->times);
	if(!st) /* the levels the grid parameters point at hold the pair */
		g->loaded[0] = g->loaded[1] = true;
	if(!st)
		st = gi_icond(c, r);
	for(uint64_t i = 0; i < d.n_dump && !st;) {
		const int64_t k = pairs[i];
		if((st = L.use_pair(k, frozen, src->times)) != GRAY_OK)
			break;
		if((e = cudaEventRecord(before, c->stream)) != cudaSuccess) {
			st = gi_from_cuda(e);
			break;
		}
		const double t      = d.t_init + (double)i * d.dt_dump;
		const double target = d.t_init + (double)(++i) * d.dt_dump;
		if((st = gi_evolve_interval(c, r, t, target, d.n_sub)) != GRAY_OK)
			break;
		/* prefetch a snapshot of the next pair into the level this
		 * interval does not read, once the intervals before it are done */
		if(!frozen && i < d.n_dump) {
			const int64_t now[2] = {k, k + 1};
			const int64_t nk = pairs[i];
			for(int64_t s = nk; s <= nk + 1; ++s) {
				if(L.find(s) >= 0)
					continue;
				int b = L.free_level(now, 2);
				if(b < 0 || (st = L.load(b, s, before)) != GRAY_OK)
					break;
				break; /* one spare level: the other waits for use_pair */
			}
			if(st)
				break;
		}
		if(after_dump) {
			if((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
				st = gi_from_cuda(e);
				break;
			}
			if(after_dump(src->user, i) != 0) {
				st = GRAY_ESOURCE;
				break;
			}
		}
	}
	if(!st)
		st = gi_timed_end(c, ns);
	/* drain the copies before the events and the stream go away */
	if(L.copy)
		cudaStreamSynchronize(L.copy);
	if(st)
		cudaStreamSynchronize(c->stream);

	/* the levels of the last pair become the grid's levels 0 and 1 */
	if(!st) {
		const int64_t k = d.n_dump ? pairs[d.n_dump - 1] : first;
		int b0 = L.find(k), b1 = frozen ? b0 : L.find(k + 1);
		float *lv0 = L.buf[b0], *lv1 = L.buf[b1];
		float *rest = nullptr;
		for(int b = 0; b < 3; ++b)
			if(L.buf[b] != lv0 && L.buf[b] != lv1)
				rest = rest ? rest : L.buf[b];
		if(frozen) { /* one snapshot: level 1 is a copy (sim-org/gray.c:219-224) */
			float *other = rest;
			for(int b = 0; b < 3; ++b)
				if(L.buf[b] != lv0 && L.buf[b] != other)
					rest = L.buf[b];
			lv1 = other;
			e = cudaMemcpyAsync(lv1, lv0, level_bytes, cudaMemcpyDeviceToDevice, c->stream);
			if(e == cudaSuccess)
				e = cudaStreamSynchronize(c->stream);
			if(e != cudaSuccess)
				st = gi_from_cuda(e);
		}
		g->lvl[0] = lv0;
		g->lvl[1] = lv1;
		g->spare = rest;
		g->gp.lvl[0] = lv0;
		g->gp.lvl[1] = lv1;
		g->loaded[0] = g->loaded[1] = true;
		g->desc.box[0] = g->gp.box[0];
		g->desc.box[4] = g->gp.box[4];
	} else {
		/* contents unknown after a failure: the grid must be reloaded */
		g->gp.lvl[0] = g->lvl[0];
		g->gp.lvl[1] = g->lvl[1];
		g->loaded[0] = g->loaded[1] = false;
	}
	if(loads)
		*loads = L.loads;
	for(int b = 0; b < 3; ++b)
		if(L.ready[b])
			cudaEventDestroy(L.ready[b]);
	if(L.staged)
		cudaEventDestroy(L.staged);
	if(before)
		cudaEventDestroy(before);
	if(L.copy)
		cudaStreamDestroy(L.copy);
	return st;
}
