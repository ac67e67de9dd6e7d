/*
 * C ABI of libgray_cuda (include/gray_cuda.h): contexts, renders, device
 * memory under an HBM budget, and the launch sequence of the reference's
 * host glue (sim-org/icond.c, evolve.c, gray.c:243-294, io.c:39-72).
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "ctx_internal.h"

namespace {

int
from_cuda(cudaError_t e)
{
	if(e == cudaSuccess)
		return GRAY_OK;
	if(e == cudaErrorMemoryAllocation)
		return GRAY_ENOMEM;
	return GRAY_ECUDA;
}

#define CK(call)                                   \
	do {                                           \
		cudaError_t e_ = (call);                   \
		if(e_ != cudaSuccess)                      \
			return from_cuda(e_);                  \
	} while(0)

int
dalloc(gray_ctx *c, void **p, size_t bytes)
{
	std::lock_guard<std::mutex> lk(c->mem_mu);
	if(c->used + bytes > c->budget)
		return GRAY_EBUDGET;
	cudaError_t e = cudaMalloc(p, bytes);
	if(e != cudaSuccess) {
		*p = nullptr;
		cudaGetLastError();
		return GRAY_ENOMEM;
	}
	c->used += bytes;
	return GRAY_OK;
}

void
dfree(gray_ctx *c, void *p, size_t bytes)
{
	if(p) {
		std::lock_guard<std::mutex> lk(c->mem_mu);
		cudaFree(p);
		c->used -= bytes;
	}
}

Render *
find(gray_ctx *c, int id)
{
	if(!c)
		return nullptr;
	auto it = c->renders.find(id);
	return it == c->renders.end() ? nullptr : it->second;
}

/* Bardeen-Press-Teukolsky prograde ISCO (M = 1) */
double
risco_of(double a)
{
	double z1 = 1.0 + cbrt(1.0 - a * a) * (cbrt(1.0 + a) + cbrt(1.0 - a));
	double z2 = sqrt(3.0 * a * a + z1 * z1);
	return 3.0 + z2 - sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
}

int
check_desc(const gray_render_desc *d)
{
	if(!d)
		return GRAY_EINVAL;
	if(!(d->a_spin > -1.0 && d->a_spin < 1.0))
		return GRAY_EINVAL;
	if(d->n_width == 0 || d->n_height == 0 || d->n_sub == 0)
		return GRAY_EINVAL;
	if(d->n_width > (1u << 20) || d->n_height > (1u << 20))
		return GRAY_EINVAL;
	if(d->n_rows == 0 ? d->row_begin != 0
	                  : d->row_begin >= d->n_height || d->n_rows > d->n_height - d->row_begin)
		return GRAY_EINVAL;
	if((uint64_t)d->n_width * (d->n_rows ? d->n_rows : d->n_height) > (1ull << 31))
		return GRAY_EINVAL;
	if(d->n_sub > (uint64_t)INT32_MAX)
		return GRAY_EINVAL;
	/* the persistent kernels count dump intervals in 32-bit integers */
	if(d->n_dump > (uint64_t)INT32_MAX)
		return GRAY_EINVAL;
	if(d->n_freq < 0 || d->n_freq > GRAY_MAX_FREQ)
		return GRAY_EINVAL;
	if(d->flow != GRAY_FLOW_NONE && d->flow != GRAY_FLOW_TORUS &&
	   d->flow != GRAY_FLOW_THERMAL)
		return GRAY_EINVAL;
	if(d->term != GRAY_TERM_EPS && d->term != GRAY_TERM_RPLUS)
		return GRAY_EINVAL;
	if(d->precision != GRAY_PREC_FP64 && d->precision != GRAY_PREC_MIXED)
		return GRAY_EINVAL;
	if(d->spacetime != GRAY_ST_KERR && d->spacetime != GRAY_ST_NUMERICAL)
		return GRAY_EINVAL;
	/* the torus is an analytic-spacetime model, the thermal flow reads the
	 * grid's density: each transfer belongs to one kind of spacetime */
	if(d->n_freq > 0 && d->spacetime == GRAY_ST_NUMERICAL && d->flow != GRAY_FLOW_THERMAL)
		return GRAY_EINVAL;
	if(d->n_freq > 0 && d->spacetime == GRAY_ST_KERR && d->flow == GRAY_FLOW_THERMAL)
		return GRAY_EINVAL;
	if(d->flow == GRAY_FLOW_THERMAL &&
	   !(std::isfinite(d->m_adm) && std::isfinite(d->flow_te) && d->flow_te > 0.0 &&
	     std::isfinite(d->flow_b)))
		return GRAY_EINVAL;
	for(int i = 0; i < d->n_freq; ++i)
		if(!(d->nu[i] > 0.0))
			return GRAY_EINVAL;
	if(!std::isfinite(d->dt_dump) || !std::isfinite(d->t_init))
		return GRAY_EINVAL;
	/* driver.cl:93 divides by the interval: a zero one has no step count */
	if(d->n_dump > 0 && d->dt_dump == 0.0)
		return GRAY_EINVAL;
	return GRAY_OK;
}

void
make_params(const gray_render_desc *d, RenderParams *p)
{
	memset(p, 0, sizeof(*p));
	p->a  = d->a_spin;
	p->aa = d->a_spin * d->a_spin;
	p->rp = 1.0 + sqrt(1.0 - d->a_spin * d->a_spin);
	p->risco = risco_of(d->a_spin);
	p->eps_stop = d->term == GRAY_TERM_RPLUS ? 0.01 * p->rp : 0.01;
	const double deg2rad = 3.14159265358979323846264338327950288 / 180.0;
	p->ci = cos(deg2rad * d->i_obs);
	p->si = sin(deg2rad * d->i_obs);
	p->cj = cos(deg2rad * d->j_obs);
	p->sj = sin(deg2rad * d->j_obs);
	p->w_img = d->w_img;
	p->h_img = d->h_img;
	p->r_obs = d->r_obs;
	p->w_rays = (long long)d->n_width;
	p->h_rays = (long long)d->n_height;
	p->row0 = (long long)d->row_begin;
	p->n_rays = p->w_rays * (long long)(d->n_rows ? d->n_rows : d->n_height);
	p->spacetime = d->spacetime;
	p->flow = d->n_freq > 0 ? d->flow : GRAY_FLOW_NONE;
	p->n_freq = d->n_freq;
	p->n_data = 8 + 2 * d->n_freq;
	p->torus_n0 = d->torus_n0;
	p->torus_kappa = d->torus_kappa;
	p->torus_hr = d->torus_hr;
	for(int i = 0; i < d->n_freq; ++i) {
		p->nupow[i]  = pow(d->nu[i], -0.7);
		p->nuinv2[i] = 1.0 / (d->nu[i] * d->nu[i]);
		p->nupow_f[i]  = (float)p->nupow[i];
		p->nuinv2_f[i] = (float)p->nuinv2[i];
		p->nu[i] = d->nu[i];
	}
	p->m_adm = d->m_adm;
	p->flow_te = d->flow_te;
	p->flow_b = d->flow_b;
	gray_thermal_consts(&p->th);
}

int
timed_begin(gray_ctx *c)
{
	CK(cudaEventRecord(c->ev0, c->stream));
	return GRAY_OK;
}

int
timed_end(gray_ctx *c, double *ns)
{
	CK(cudaEventRecord(c->ev1, c->stream));
	if(ns) {
		CK(cudaEventSynchronize(c->ev1));
		float ms = 0.0f;
		CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
		*ns = (double)ms * 1e6;
	}
	return GRAY_OK;
}

int
grid_ready(gray_ctx *c)
{
	if(!c->grid || !c->grid->loaded[0])
		return 0;
	if(!c->grid->gp.single && !c->grid->loaded[1])
		return 0;
	return 1;
}

} /* namespace */

/* Shared with other translation units (ctx_internal.h, gray_internal.h). */
int
gi_from_cuda(cudaError_t e)
{
	return from_cuda(e);
}

int
gi_dalloc(gray_ctx *c, void **p, size_t bytes)
{
	return dalloc(c, p, bytes);
}

int
gi_reserve(gray_ctx *c, size_t bytes)
{
	std::lock_guard<std::mutex> lk(c->mem_mu);
	if(c->used + bytes > c->budget)
		return GRAY_EBUDGET;
	c->used += bytes;
	return GRAY_OK;
}

void
gi_unreserve(gray_ctx *c, size_t bytes)
{
	std::lock_guard<std::mutex> lk(c->mem_mu);
	c->used -= bytes;
}

void
gi_dfree(gray_ctx *c, void *p, size_t bytes)
{
	dfree(c, p, bytes);
}

int
gi_grid_ready(gray_ctx *c)
{
	return grid_ready(c);
}

/* rt.cl:95-143 constants that need libm, from volatile inputs so that the
 * compiler folds none of them (the CPU oracle evaluates the same way) */
void
gray_thermal_consts(ThermalConsts *t)
{
	volatile double three = 3.0, four = 4.0, twelve = 12.0, pi = 3.14159265358979323846,
	                e_gaunt = 1.78107241799;
	const double c = 2.99792458e+10, G = 6.67384800e-08, kB = 1.38064881e-16,
	             me = 9.10938291e-28, msun = 1.98910000e+33;
	volatile double ff_in = G * msun / (c * c) * 6.8e-38, mec2_kb = me * c * c / kB;
	volatile double tmax_tmin = 1e+2 / 1e-1;
	t->g1 = sqrt(three / pi);
	t->g2 = sqrt(three) / pi;
	t->g3 = log(four / e_gaunt);
	t->g4 = log(four / pow(e_gaunt, 2.5));
	t->g5 = sqrt(twelve);
	t->ff_f = sqrt(ff_in / (4 * pi * sqrt(mec2_kb)));
	t->lk_scale = 60.0 / log(tmax_tmin);
}

int
gray_internal_check_desc(const gray_render_desc *d)
{
	return check_desc(d);
}

void
gray_internal_make_params(const gray_render_desc *d, RenderParams *p)
{
	make_params(d, p);
}

/* ------------------------------------------------------------------------ */

extern "C" const char *
gray_strerror(int s)
{
	switch(s) {
	case GRAY_OK:        return "success";
	case GRAY_EINVAL:    return "invalid argument or configuration";
	case GRAY_ENOMEM:    return "out of memory";
	case GRAY_ECUDA:     return "CUDA runtime error";
	case GRAY_ENODEV:    return "no usable CUDA device";
	case GRAY_EBUDGET:   return "request exceeds the HBM budget";
	case GRAY_ETIMEOUT:  return "bounded device wait timed out";
	case GRAY_ENOTFOUND: return "unknown render or request id";
	case GRAY_ESTATE:    return "call out of order";
	case GRAY_ESIZE:     return "buffer size mismatch";
	case GRAY_ESOURCE:   return "a caller callback failed";
	default:             return "unknown status";
	}
}

extern "C" int
gray_abi_version(void)
{
	return GRAY_ABI_VERSION;
}

extern "C" gray_ctx *
gray_create(int device, size_t hbm_budget, int *status)
{
	int st = GRAY_OK, n = 0;
	gray_ctx *c = nullptr;
	cudaDeviceProp prop;
	size_t fr = 0, tot = 0;

	if(cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
		cudaGetLastError();
		st = GRAY_ENODEV;
		goto out;
	}
	if(cudaSetDevice(device) != cudaSuccess ||
	   cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
		st = GRAY_ENODEV;
		goto out;
	}
	if(prop.major < 10) { /* built for sm_100a only */
		st = GRAY_ENODEV;
		goto out;
	}
	c = new(std::nothrow) gray_ctx;
	if(!c) {
		st = GRAY_ENOMEM;
		goto out;
	}
	c->device = device;
	c->sms = prop.multiProcessorCount;
	if(cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
		st = GRAY_ECUDA;
		goto fail;
	}
	c->budget = hbm_budget ? hbm_budget : (size_t)(0.9 * (double)fr);
	if(cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
	   cudaEventCreate(&c->ev0) != cudaSuccess ||
	   cudaEventCreate(&c->ev1) != cudaSuccess) {
		st = GRAY_ECUDA;
		goto fail;
	}
	c->stream = c->own;
	c->mixed.sms = c->sms;
	goto out;
fail:
	gray_destroy(c);
	c = nullptr;
out:
	if(status)
		*status = st;
	return c;
}

static void
free_grid(gray_ctx *c)
{
	if(!c->grid)
		return;
	Grid *g = c->grid;
	size_t npts = (size_t)g->desc.nx * g->desc.ny * g->desc.nz;
	for(int l = 0; l < 2; ++l)
		dfree(c, g->lvl[l], npts * GRAY_NSTRIDE * sizeof(float));
	if(g->spare)
		dfree(c, g->spare, npts * GRAY_NSTRIDE * sizeof(float));
	if(g->staging)
		cudaFreeHost(g->staging);
	const int n[3] = {g->desc.nx, g->desc.ny, g->desc.nz};
	for(int a = 0; a < 3; ++a) {
		dfree(c, g->nodes[a], (n[a] + 1) * sizeof(double));
		dfree(c, g->nodes_f[a], (n[a] + 1) * sizeof(float));
	}
	delete g;
	c->grid = nullptr;
}

extern "C" void
gray_destroy(gray_ctx *c)
{
	if(!c)
		return;
	gi_serve_shutdown(c);
	cudaSetDevice(c->device);
	if(c->stream)
		cudaStreamSynchronize(c->stream);
	for(auto &kv : c->batches) {
		Batch *b = kv.second;
		if(b->exec)
			cudaGraphExecDestroy(b->exec);
		dfree(c, b->block, b->bytes);
		delete b;
	}
	c->batches.clear();
	for(auto &kv : c->renders) {
		Render *r = kv.second;
		dfree(c, r->d_data, r->bytes);
		delete r;
	}
	c->renders.clear();
	free_grid(c);
	if(c->ev0) cudaEventDestroy(c->ev0);
	if(c->ev1) cudaEventDestroy(c->ev1);
	if(c->own) cudaStreamDestroy(c->own);
	delete c;
}

extern "C" int
gray_set_stream(gray_ctx *c, void *stream)
{
	if(!c)
		return GRAY_EINVAL;
	c->stream = stream ? (cudaStream_t)stream : c->own;
	return GRAY_OK;
}

extern "C" int
gray_sync(gray_ctx *c)
{
	if(!c)
		return GRAY_EINVAL;
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	return GRAY_OK;
}

extern "C" size_t
gray_hbm_used(const gray_ctx *c)
{
	return c ? c->used : 0;
}

/* One device block per render: data | info | steps | queue */
extern "C" int
gray_render_create(gray_ctx *c, const gray_render_desc *d, int *id)
{
	if(!c || !id)
		return GRAY_EINVAL;
	int st = check_desc(d);
	if(st)
		return st;
	CK(cudaSetDevice(c->device));
	Render *r = new(std::nothrow) Render;
	if(!r)
		return GRAY_ENOMEM;
	r->desc = *d;
	make_params(d, &r->p);
	const size_t nr = (size_t)r->p.n_rays;
	const size_t data_b = nr * r->p.n_data * sizeof(double);
	const size_t info_b = nr * sizeof(double);
	const size_t tab_b = (sizeof(MixedRender) + 255) / 256 * 256;
	r->bytes = data_b + info_b + 256 + tab_b;
	void *base = nullptr;
	st = dalloc(c, &base, r->bytes);
	if(st) {
		delete r;
		return st;
	}
	r->d_data  = (double *)base;
	r->d_info  = (double *)((char *)base + data_b);
	r->d_steps = (unsigned long long *)((char *)base + data_b + info_b);
	r->d_queue = (unsigned int *)((char *)base + data_b + info_b + 128);
	r->d_prefix = (unsigned long long *)((char *)base + data_b + info_b + 192);
	r->d_table = (MixedRender *)((char *)base + data_b + info_b + 256);
	cudaError_t e = cudaMemsetAsync((char *)base + data_b + info_b, 0, 256, c->stream);
	if(e != cudaSuccess) {
		dfree(c, base, r->bytes);
		delete r;
		return from_cuda(e);
	}
	try {
		c->renders[c->next_id] = r;
	} catch(const std::bad_alloc &) {
		dfree(c, base, r->bytes);
		delete r;
		return GRAY_ENOMEM;
	}
	*id = c->next_id++;
	return GRAY_OK;
}

extern "C" int
gray_render_destroy(gray_ctx *c, int id)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	for(auto &kv : c->batches)
		for(int bid : kv.second->ids)
			if(bid == id)
				return GRAY_ESTATE; /* still part of a batch */
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	dfree(c, r->d_data, r->bytes);
	c->renders.erase(id);
	delete r;
	return GRAY_OK;
}

static int
icond_impl(gray_ctx *c, Render *r)
{
	CK(cudaMemsetAsync(r->d_steps, 0, 2 * sizeof(unsigned long long), c->stream));
	if(r->p.spacetime == GRAY_ST_NUMERICAL) {
		if(!grid_ready(c))
			return GRAY_ESTATE;
		CK(launch_dyst_icond(r->p, c->grid->gp, r->d_data, r->d_info, c->stream));
	} else {
		CK(launch_icond64(r->p, r->d_data, r->d_info, c->stream));
	}
	r->has_state = true;
	return GRAY_OK;
}

extern "C" int
gray_icond(gray_ctx *c, int id)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	CK(cudaSetDevice(c->device));
	return icond_impl(c, r);
}

/* Build the one-entry render table of a mixed render and launch the
 * persistent kernel over n_dump intervals starting at t_init. */
static int
run_mixed(gray_ctx *c, Render *r, double t_init, double dt_dump, long long n_dump,
          long long n_sub)
{
	MixedRender m;
	memset(&m, 0, sizeof(m));
	fill_mixed_render(r->p, r->d_data, r->d_info, t_init, dt_dump, n_dump, n_sub, &m);
	CK(cudaMemcpyAsync(r->d_table, &m, sizeof(m), cudaMemcpyHostToDevice, c->stream));
	MixedTable T;
	T.renders = r->d_table;
	T.prefix = r->d_prefix; /* zeroed at creation: the one render starts at 0 */
	T.n_renders = 1;
	T.total = (unsigned long long)r->p.n_rays;
	if(r->p.spacetime == GRAY_ST_NUMERICAL) {
		if(!grid_ready(c))
			return GRAY_ESTATE;
		CK(launch_dyst_mixed_table(T, c->grid->gp, r->p.n_freq, r->d_queue, r->d_steps,
		                           c->stream, c->mixed, r->d_steps + 1));
	} else {
		CK(launch_mixed_table(T, r->p.n_freq, r->d_queue, r->d_steps, c->stream, c->mixed, &m));
	}
	return GRAY_OK;
}

static int
evolve_interval(gray_ctx *c, Render *r, double t, double target, uint64_t n_sub)
{
	const double dt = target - t;
	if(r->p.spacetime == GRAY_ST_NUMERICAL) {
		if(!grid_ready(c))
			return GRAY_ESTATE;
		if(r->desc.precision == GRAY_PREC_FP64) {
			CK(launch_dyst_evolve64(r->p, c->grid->gp, r->d_data, r->d_info, dt,
			                        (long long)n_sub, r->d_steps, c->stream));
			return GRAY_OK;
		}
		return run_mixed(c, r, t, dt, 1, (long long)n_sub);
	}
	if(r->desc.precision == GRAY_PREC_FP64) {
		CK(launch_evolve64(r->p, r->d_data, r->d_info, dt, (long long)n_sub,
		                   r->d_steps, c->stream, c->evolve64_block));
		return GRAY_OK;
	}
	return run_mixed(c, r, t, dt, 1, (long long)n_sub);
}

extern "C" int
gray_evolve(gray_ctx *c, int id, double t, double target, uint64_t n_sub, double *ns)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	if(!r->has_state)
		return GRAY_ESTATE;
	if(n_sub == 0 || n_sub > (uint64_t)INT32_MAX || !std::isfinite(t) ||
	   !std::isfinite(target))
		return GRAY_EINVAL;
	CK(cudaSetDevice(c->device));
	int st = timed_begin(c);
	if(st)
		return st;
	if(target != t) { /* an empty interval leaves the state as it is */
		st = evolve_interval(c, r, t, target, n_sub);
		if(st)
			return st;
	}
	return timed_end(c, ns);
}

static int
evolve_all_impl(gray_ctx *c, Render *r)
{
	const gray_render_desc &d = r->desc;
	int st;
	if(d.precision == GRAY_PREC_MIXED) {
		st = run_mixed(c, r, d.t_init, d.dt_dump, (long long)d.n_dump, (long long)d.n_sub);
		if(st)
			return st;
	} else {
		/* sim-org/gray.c:248-257 */
		for(uint64_t i = 0; i < d.n_dump;) {
			double t      = d.t_init + (double)i * d.dt_dump;
			double target = d.t_init + (double)(++i) * d.dt_dump;
			st = evolve_interval(c, r, t, target, d.n_sub);
			if(st)
				return st;
		}
	}
	return GRAY_OK;
}

extern "C" int
gray_run(gray_ctx *c, int id, double *ns)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	CK(cudaSetDevice(c->device));
	int st = timed_begin(c);
	if(!st)
		st = icond_impl(c, r);
	if(!st)
		st = evolve_all_impl(c, r);
	if(!st)
		st = timed_end(c, ns);
	return st;
}

extern "C" int
gray_evolve_all(gray_ctx *c, int id, double *ns)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	if(!r->has_state)
		return GRAY_ESTATE;
	CK(cudaSetDevice(c->device));
	int st = timed_begin(c);
	if(!st)
		st = evolve_all_impl(c, r);
	if(!st)
		st = timed_end(c, ns);
	return st;
}

extern "C" int
gray_read_state(gray_ctx *c, int id, void *data, size_t data_bytes, void *info,
                size_t info_bytes, int layout)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	if(!r->has_state)
		return GRAY_ESTATE;
	if(layout != GRAY_LAYOUT_SOA && layout != GRAY_LAYOUT_AOS)
		return GRAY_EINVAL;
	const size_t nr = (size_t)r->p.n_rays;
	const size_t db = nr * r->p.n_data * sizeof(double);
	if(data && data_bytes != db)
		return GRAY_ESIZE;
	if(info && info_bytes != nr * sizeof(double))
		return GRAY_ESIZE;
	CK(cudaSetDevice(c->device));
	if(data) {
		if(layout == GRAY_LAYOUT_SOA) {
			CK(cudaMemcpyAsync(data, r->d_data, db, cudaMemcpyDeviceToHost, c->stream));
		} else {
			void *tmp = nullptr;
			int st = dalloc(c, &tmp, db);
			if(st)
				return st;
			cudaError_t e = launch_transpose(r->d_data, (double *)tmp, (long long)nr,
			                                 r->p.n_data, 1, c->stream);
			if(e == cudaSuccess)
				e = cudaMemcpyAsync(data, tmp, db, cudaMemcpyDeviceToHost, c->stream);
			if(e == cudaSuccess)
				e = cudaStreamSynchronize(c->stream);
			dfree(c, tmp, db);
			if(e != cudaSuccess)
				return from_cuda(e);
		}
	}
	if(info)
		CK(cudaMemcpyAsync(info, r->d_info, nr * sizeof(double), cudaMemcpyDeviceToHost,
		                   c->stream));
	CK(cudaStreamSynchronize(c->stream));
	return GRAY_OK;
}

extern "C" int
gray_write_state(gray_ctx *c, int id, const void *data, size_t data_bytes, int layout)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	if(!data || (layout != GRAY_LAYOUT_SOA && layout != GRAY_LAYOUT_AOS))
		return GRAY_EINVAL;
	const size_t nr = (size_t)r->p.n_rays;
	const size_t db = nr * r->p.n_data * sizeof(double);
	if(data_bytes != db)
		return GRAY_ESIZE;
	CK(cudaSetDevice(c->device));
	if(layout == GRAY_LAYOUT_SOA) {
		CK(cudaMemcpyAsync(r->d_data, data, db, cudaMemcpyHostToDevice, c->stream));
	} else {
		void *tmp = nullptr;
		int st = dalloc(c, &tmp, db);
		if(st)
			return st;
		cudaError_t e = cudaMemcpyAsync(tmp, data, db, cudaMemcpyHostToDevice, c->stream);
		if(e == cudaSuccess)
			e = launch_transpose((const double *)tmp, r->d_data, (long long)nr,
			                     r->p.n_data, 0, c->stream);
		if(e == cudaSuccess)
			e = cudaStreamSynchronize(c->stream);
		dfree(c, tmp, db);
		if(e != cudaSuccess)
			return from_cuda(e);
	}
	if(r->p.spacetime == GRAY_ST_KERR)
		CK(launch_getuu64(r->p, r->d_data, r->d_info, c->stream));
	CK(cudaMemsetAsync(r->d_steps, 0, 2 * sizeof(unsigned long long), c->stream));
	CK(cudaStreamSynchronize(c->stream));
	r->has_state = true;
	return GRAY_OK;
}

extern "C" int
gray_read_kdown(gray_ctx *c, int id, double *k, size_t bytes)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	if(!r->has_state)
		return GRAY_ESTATE;
	if(!k)
		return GRAY_EINVAL;
	if(r->p.spacetime != GRAY_ST_KERR)
		return GRAY_EINVAL;
	const size_t nr = (size_t)r->p.n_rays;
	if(bytes != nr * 4 * sizeof(double))
		return GRAY_ESIZE;
	CK(cudaSetDevice(c->device));
	void *tmp = nullptr;
	int st = dalloc(c, &tmp, bytes);
	if(st)
		return st;
	cudaError_t e = launch_kdown64(r->p, r->d_data, (double *)tmp, c->stream);
	if(e == cudaSuccess)
		e = cudaMemcpyAsync(k, tmp, bytes, cudaMemcpyDeviceToHost, c->stream);
	if(e == cudaSuccess)
		e = cudaStreamSynchronize(c->stream);
	dfree(c, tmp, bytes);
	return from_cuda(e);
}

extern "C" int
gray_read_coords(gray_ctx *c, int id, int system, double r_match, int flags, double *out,
                 size_t bytes)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	if(!r->has_state)
		return GRAY_ESTATE;
	if(!out || (system != GRAY_COORDS_SPH_KS && system != GRAY_COORDS_BL) ||
	   (flags & ~GRAY_COORDS_AS_WRITTEN))
		return GRAY_EINVAL;
	if(r->p.spacetime != GRAY_ST_KERR)
		return GRAY_EINVAL;
	if(system == GRAY_COORDS_BL && !(std::isfinite(r_match) && r_match > r->p.rp))
		return GRAY_EINVAL;
	const size_t nr = (size_t)r->p.n_rays;
	if(bytes != nr * 8 * sizeof(double))
		return GRAY_ESIZE;
	CK(cudaSetDevice(c->device));
	void *tmp = nullptr;
	int st = dalloc(c, &tmp, bytes);
	if(st)
		return st;
	cudaError_t e = launch_coords64(r->p, r->d_data, (double *)tmp, system, r_match,
	                                (flags & GRAY_COORDS_AS_WRITTEN) ? 1 : 0, c->stream);
	if(e == cudaSuccess)
		e = cudaMemcpyAsync(out, tmp, bytes, cudaMemcpyDeviceToHost, c->stream);
	if(e == cudaSuccess)
		e = cudaStreamSynchronize(c->stream);
	dfree(c, tmp, bytes);
	return from_cuda(e);
}

extern "C" int
gray_ray_steps(gray_ctx *c, int id, uint64_t *steps)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	if(!steps)
		return GRAY_EINVAL;
	CK(cudaSetDevice(c->device));
	unsigned long long v = 0;
	CK(cudaMemcpyAsync(&v, r->d_steps, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	*steps = v;
	return GRAY_OK;
}

/* ---- numerical spacetime ------------------------------------------- */

static int
check_grid(const gray_grid_desc *g)
{
	if(!g || g->nx < 2 || g->ny < 2 || g->nz < 2)
		return GRAY_EINVAL;
	if((long long)g->nx * g->ny * g->nz > (1ll << 28))
		return GRAY_EINVAL;
	for(int a = 1; a <= 3; ++a)
		if(!(g->box[a] < g->box[a + 4]))
			return GRAY_EINVAL;
	if(!(g->box[4] >= g->box[0]))
		return GRAY_EINVAL;
	return GRAY_OK;
}

static int
same_shape(const gray_grid_desc *a, const gray_grid_desc *b)
{
	return a->nx == b->nx && a->ny == b->ny && a->nz == b->nz &&
	       memcmp(a->box + 1, b->box + 1, 3 * sizeof(float)) == 0 &&
	       memcmp(a->box + 5, b->box + 5, 3 * sizeof(float)) == 0;
}

/* (Re)creates the grid when the shape changes; computes the fisheye
 * constants and node tables of interp.cl:89-121 on the host in FP64. */
static int
ensure_grid(gray_ctx *c, const gray_grid_desc *gd)
{
	if(c->grid && !same_shape(&c->grid->desc, gd))
		free_grid(c);
	if(!c->grid) {
		Grid *g = new(std::nothrow) Grid;
		if(!g)
			return GRAY_ENOMEM;
		g->desc = *gd;
		c->grid = g;
		size_t npts = (size_t)gd->nx * gd->ny * gd->nz;
		for(int l = 0; l < 2; ++l) {
			int st = dalloc(c, (void **)&g->lvl[l], npts * GRAY_NSTRIDE * sizeof(float));
			if(st) {
				free_grid(c);
				return st;
			}
		}
		const int n[3] = {gd->nx, gd->ny, gd->nz};
		GridParams &gp = g->gp;
		memset(&gp, 0, sizeof(gp));
		for(int a = 0; a < 3; ++a) {
			double lo = gd->box[a + 1], hi = gd->box[a + 5];
			double B = cbrt(asinh(lo));
			double A = (cbrt(asinh(hi)) - B) / (double)(n[a] - 1);
			gp.A[a] = A;
			gp.B[a] = B;
			std::vector<double> nd;
			std::vector<float> nf;
			try {
				nd.resize(n[a] + 1);
				nf.resize(n[a] + 1);
			} catch(const std::bad_alloc &) {
				free_grid(c);
				return GRAY_ENOMEM;
			}
			for(int i = 0; i <= n[a]; ++i) {
				double f = fma(A, (double)i, B);
				nd[i] = sinh((f * f) * f);
				nf[i] = (float)nd[i];
			}
			int st = dalloc(c, (void **)&g->nodes[a], (n[a] + 1) * sizeof(double));
			if(!st)
				st = dalloc(c, (void **)&g->nodes_f[a], (n[a] + 1) * sizeof(float));
			if(st) {
				free_grid(c);
				return st;
			}
			CK(cudaMemcpy(g->nodes[a], nd.data(), (n[a] + 1) * sizeof(double),
			              cudaMemcpyHostToDevice));
			CK(cudaMemcpy(g->nodes_f[a], nf.data(), (n[a] + 1) * sizeof(float),
			              cudaMemcpyHostToDevice));
			gp.nodes[a] = g->nodes[a];
			gp.nodes_f[a] = g->nodes_f[a];
		}
		gp.nx = gd->nx; gp.ny = gd->ny; gp.nz = gd->nz;
		gp.lvl[0] = g->lvl[0];
		gp.lvl[1] = g->lvl[1];
	}
	Grid *g = c->grid;
	g->desc.box[0] = gd->box[0];
	g->desc.box[4] = gd->box[4];
	g->desc.bug_gzz = gd->bug_gzz;
	g->desc.physics = gd->physics;
	memcpy(g->gp.box, g->desc.box, sizeof(g->gp.box));
	g->gp.bug_gzz = gd->bug_gzz;
	g->gp.physics = gd->physics;
	g->gp.single = gd->box[0] == gd->box[4];
	return GRAY_OK;
}

extern "C" int
gray_load_spacetime_interleaved(gray_ctx *c, const gray_grid_desc *gd,
                                const float *fields, int level)
{
	if(!c || !fields || (level != 0 && level != 1))
		return GRAY_EINVAL;
	int st = check_grid(gd);
	if(st)
		return st;
	CK(cudaSetDevice(c->device));
	st = ensure_grid(c, gd);
	if(st)
		return st;
	const size_t npts = (size_t)gd->nx * gd->ny * gd->nz;
	/* host rows of 51 -> device rows of GRAY_NSTRIDE (pitched copy) */
	CK(cudaMemcpy2DAsync(c->grid->lvl[level], GRAY_NSTRIDE * sizeof(float), fields,
	                     GRAY_NCOMP * sizeof(float), GRAY_NCOMP * sizeof(float), npts,
	                     cudaMemcpyHostToDevice, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	c->grid->loaded[level] = true;
	return GRAY_OK;
}

extern "C" int
gray_load_spacetime(gray_ctx *c, const gray_grid_desc *gd, const float *const *fields,
                    int level)
{
	if(!c || !fields || (level != 0 && level != 1))
		return GRAY_EINVAL;
	for(int i = 0; i < GRAY_NCOMP; ++i)
		if(!fields[i])
			return GRAY_EINVAL;
	int st = check_grid(gd);
	if(st)
		return st;
	CK(cudaSetDevice(c->device));
	st = ensure_grid(c, gd);
	if(st)
		return st;
	const size_t npts = (size_t)gd->nx * gd->ny * gd->nz;
	/* stage one field at a time and scatter it into the interleaved rows */
	CK(cudaMemcpy2DAsync(c->grid->lvl[level], GRAY_NSTRIDE * sizeof(float), fields[0],
	                     sizeof(float), sizeof(float), npts, cudaMemcpyHostToDevice,
	                     c->stream));
	for(int i = 1; i < GRAY_NCOMP; ++i)
		CK(cudaMemcpy2DAsync(c->grid->lvl[level] + i, GRAY_NSTRIDE * sizeof(float),
		                     fields[i], sizeof(float), sizeof(float), npts,
		                     cudaMemcpyHostToDevice, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	c->grid->loaded[level] = true;
	return GRAY_OK;
}

extern "C" int
gray_make_boosted_ks(gray_ctx *c, const gray_grid_desc *gd, double a, double v,
                     int axis, double t, int level)
{
	if(!c || (level != 0 && level != 1) || axis < 1 || axis > 3)
		return GRAY_EINVAL;
	if(!(a > -1.0 && a < 1.0) || !(v > -1.0 && v < 1.0))
		return GRAY_EINVAL;
	int st = check_grid(gd);
	if(st)
		return st;
	CK(cudaSetDevice(c->device));
	st = ensure_grid(c, gd);
	if(st)
		return st;
	CK(launch_boosted_ks(c->grid->gp, c->grid->lvl[level], a, v, axis, t, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	c->grid->loaded[level] = true;
	return GRAY_OK;
}

extern "C" int
gray_read_spacetime(gray_ctx *c, int level, float *fields, size_t bytes)
{
	if(!c || !fields || (level != 0 && level != 1))
		return GRAY_EINVAL;
	if(!c->grid || !c->grid->loaded[level])
		return GRAY_ESTATE;
	const gray_grid_desc &gd = c->grid->desc;
	const size_t npts = (size_t)gd.nx * gd.ny * gd.nz;
	if(bytes != npts * GRAY_NCOMP * sizeof(float))
		return GRAY_ESIZE;
	CK(cudaSetDevice(c->device));
	CK(cudaMemcpy2DAsync(fields, GRAY_NCOMP * sizeof(float), c->grid->lvl[level],
	                     GRAY_NSTRIDE * sizeof(float), GRAY_NCOMP * sizeof(float), npts,
	                     cudaMemcpyDeviceToHost, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	return GRAY_OK;
}

cudaError_t measure_peak(int precision, int sms, cudaStream_t st, double *flops);

extern "C" int
gray_measure_peak(gray_ctx *c, int precision, double *flops)
{
	if(!c || !flops || (precision != GRAY_PREC_FP64 && precision != GRAY_PREC_MIXED &&
	                    precision != GRAY_PEAK_L1_GATHER))
		return GRAY_EINVAL;
	CK(cudaSetDevice(c->device));
	CK(measure_peak(precision, c->sms, c->stream, flops));
	return GRAY_OK;
}

extern "C" int
gray_swap_levels(gray_ctx *c)
{
	if(!c || !c->grid)
		return GRAY_ESTATE;
	Grid *g = c->grid;
	float *t = g->lvl[0];
	g->lvl[0] = g->lvl[1];
	g->lvl[1] = t;
	bool b = g->loaded[0];
	g->loaded[0] = g->loaded[1];
	g->loaded[1] = b;
	g->gp.lvl[0] = g->lvl[0];
	g->gp.lvl[1] = g->lvl[1];
	return GRAY_OK;
}

/* internal helpers for the snapshot series (series.cu) */
Render *
gi_find_render(gray_ctx *c, int id)
{
	return find(c, id);
}

int
gi_icond(gray_ctx *c, Render *r)
{
	return icond_impl(c, r);
}

int
gi_evolve_interval(gray_ctx *c, Render *r, double t, double target, uint64_t n_sub)
{
	return evolve_interval(c, r, t, target, n_sub);
}

int
gi_check_grid(const gray_grid_desc *g)
{
	return check_grid(g);
}

int
gi_ensure_grid(gray_ctx *c, const gray_grid_desc *g)
{
	return ensure_grid(c, g);
}

int
gi_timed_begin(gray_ctx *c)
{
	return timed_begin(c);
}

int
gi_timed_end(gray_ctx *c, double *ns)
{
	return timed_end(c, ns);
}

/* ---- batches, plans, graphs ---------------------------------------- */

static Batch *
find_batch(gray_ctx *c, int id)
{
	if(!c)
		return nullptr;
	auto it = c->batches.find(id);
	return it == c->batches.end() ? nullptr : it->second;
}

static void
drop_graph(Batch *b)
{
	if(b->exec) {
		cudaGraphExecDestroy(b->exec);
		b->exec = nullptr;
	}
}

extern "C" int
gray_batch_create(gray_ctx *c, const int *ids, int n, int *batch_id)
{
	if(!c || !ids || n < 1 || !batch_id)
		return GRAY_EINVAL;
	Batch *b = new(std::nothrow) Batch;
	if(!b)
		return GRAY_ENOMEM;
	std::vector<unsigned long long> prefix;
	try { /* no exception may cross the C ABI */
		b->host_table.resize(n);
		b->ids.reserve(n);
		prefix.resize(n);
	} catch(const std::bad_alloc &) {
		delete b;
		return GRAY_ENOMEM;
	}
	for(int i = 0; i < n; ++i) {
		Render *r = find(c, ids[i]);
		if(!r) {
			delete b;
			return GRAY_ENOTFOUND;
		}
		for(int j = 0; j < i; ++j)
			if(ids[j] == ids[i]) {
				delete b;
				return GRAY_EINVAL; /* a render appears twice */
			}
		const gray_render_desc &d = r->desc;
		if(d.precision != GRAY_PREC_MIXED ||
		   (i > 0 && (d.spacetime != b->spacetime || d.n_freq != b->n_freq))) {
			delete b;
			return GRAY_EINVAL;
		}
		b->spacetime = d.spacetime;
		b->n_freq = d.n_freq;
		memset(&b->host_table[i], 0, sizeof(MixedRender));
		fill_mixed_render(r->p, r->d_data, r->d_info, d.t_init, d.dt_dump,
		                  (long long)d.n_dump, (long long)d.n_sub, &b->host_table[i]);
		prefix[i] = b->total;
		b->total += (unsigned long long)r->p.n_rays;
		b->ids.push_back(ids[i]);
	}
	if(b->total > (1ull << 31)) {
		delete b;
		return GRAY_EINVAL; /* the ray queue is a 32-bit counter */
	}
	CK(cudaSetDevice(c->device));
	const size_t tab = ((size_t)n * sizeof(MixedRender) + 255) / 256 * 256;
	const size_t pre = ((size_t)n * sizeof(unsigned long long) + 255) / 256 * 256;
	b->bytes = tab + pre + 256;
	int st = dalloc(c, &b->block, b->bytes);
	if(st) {
		delete b;
		return st;
	}
	b->d_table = (MixedRender *)b->block;
	b->d_prefix = (unsigned long long *)((char *)b->block + tab);
	b->d_queue = (unsigned int *)((char *)b->block + tab + pre);
	b->d_steps = (unsigned long long *)((char *)b->block + tab + pre + 128);
	cudaError_t e = cudaMemcpyAsync(b->d_table, b->host_table.data(),
	                                (size_t)n * sizeof(MixedRender), cudaMemcpyHostToDevice,
	                                c->stream);
	if(e == cudaSuccess)
		e = cudaMemcpyAsync(b->d_prefix, prefix.data(), (size_t)n * sizeof(unsigned long long),
		                    cudaMemcpyHostToDevice, c->stream);
	if(e == cudaSuccess)
		e = cudaMemsetAsync((char *)b->block + tab + pre, 0, 256, c->stream);
	if(e == cudaSuccess)
		e = cudaStreamSynchronize(c->stream);
	if(e != cudaSuccess) {
		dfree(c, b->block, b->bytes);
		delete b;
		return from_cuda(e);
	}
	try {
		c->batches[c->next_batch] = b;
	} catch(const std::bad_alloc &) {
		dfree(c, b->block, b->bytes);
		delete b;
		return GRAY_ENOMEM;
	}
	*batch_id = c->next_batch++;
	return GRAY_OK;
}

extern "C" int
gray_batch_destroy(gray_ctx *c, int id)
{
	Batch *b = find_batch(c, id);
	if(!b)
		return GRAY_ENOTFOUND;
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	drop_graph(b);
	dfree(c, b->block, b->bytes);
	c->batches.erase(id);
	delete b;
	return GRAY_OK;
}

/* Enqueue the batch: initial conditions of every render, counters reset,
 * one persistent launch over the whole table.  one: the host copy of the
 * table's entry when the batch holds one render (the one-render launch),
 * else null. */
static int
batch_enqueue(gray_ctx *c, Batch *b, const MixedLaunch &cfg, const MixedTable &T,
              const MixedRender *one)
{
	for(int id : b->ids) {
		Render *r = find(c, id);
		if(r->p.spacetime == GRAY_ST_NUMERICAL)
			CK(launch_dyst_icond(r->p, c->grid->gp, r->d_data, r->d_info, c->stream));
		else
			CK(launch_icond64(r->p, r->d_data, r->d_info, c->stream));
	}
	CK(cudaMemsetAsync(b->d_steps, 0, sizeof(unsigned long long), c->stream));
	if(b->spacetime == GRAY_ST_NUMERICAL)
		CK(launch_dyst_mixed_table(T, c->grid->gp, b->n_freq, b->d_queue, b->d_steps,
		                           c->stream, cfg));
	else
		CK(launch_mixed_table(T, b->n_freq, b->d_queue, b->d_steps, c->stream, cfg, one));
	return GRAY_OK;
}

static MixedTable
batch_table(const Batch *b)
{
	MixedTable T;
	T.renders = b->d_table;
	T.prefix = b->d_prefix;
	T.n_renders = (int)b->ids.size();
	T.total = b->total;
	return T;
}

static bool
same_cfg(const MixedLaunch &a, const MixedLaunch &b)
{
	return a.block == b.block && a.blocks_per_sm == b.blocks_per_sm && a.sms == b.sms &&
	       a.rays_per_thread == b.rays_per_thread && a.rk4_rolled == b.rk4_rolled;
}

extern "C" int
gray_batch_run(gray_ctx *c, int id, double *ns)
{
	Batch *b = find_batch(c, id);
	if(!b)
		return GRAY_ENOTFOUND;
	if(b->spacetime == GRAY_ST_NUMERICAL && !grid_ready(c))
		return GRAY_ESTATE;
	CK(cudaSetDevice(c->device));
	/* the graph holds its launches' arguments: recapture when the launch
	 * plan, the stream or (numerical) the grid it read has changed since,
	 * e.g. after gray_swap_levels, a series run or a reshaped grid */
	if(b->exec && (!same_cfg(b->graph_cfg, c->mixed) || b->graph_stream != c->stream ||
	               (b->spacetime == GRAY_ST_NUMERICAL &&
	                memcmp(&b->graph_gp, &c->grid->gp, sizeof(GridParams)) != 0)))
		drop_graph(b);
	if(!b->exec) {
		/* capture once; the graph is replayed by every later run */
		cudaGraph_t g = nullptr;
		CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
		int st = batch_enqueue(c, b, c->mixed, batch_table(b),
		                       b->host_table.size() == 1 ? &b->host_table[0] : nullptr);
		cudaError_t e = cudaStreamEndCapture(c->stream, &g);
		if(st) {
			if(g)
				cudaGraphDestroy(g);
			return st;
		}
		if(e != cudaSuccess)
			return from_cuda(e);
		e = cudaGraphInstantiate(&b->exec, g, 0);
		cudaGraphDestroy(g);
		if(e != cudaSuccess) {
			b->exec = nullptr;
			return from_cuda(e);
		}
		b->graph_cfg = c->mixed;
		b->graph_stream = c->stream;
		if(b->spacetime == GRAY_ST_NUMERICAL)
			memcpy(&b->graph_gp, &c->grid->gp, sizeof(GridParams));
	}
	int st = timed_begin(c);
	if(st)
		return st;
	CK(cudaGraphLaunch(b->exec, c->stream));
	for(int rid : b->ids)
		find(c, rid)->has_state = true;
	return timed_end(c, ns);
}

extern "C" int
gray_batch_steps(gray_ctx *c, int id, uint64_t *steps)
{
	Batch *b = find_batch(c, id);
	if(!b)
		return GRAY_ENOTFOUND;
	if(!steps)
		return GRAY_EINVAL;
	CK(cudaSetDevice(c->device));
	unsigned long long v = 0;
	CK(cudaMemcpyAsync(&v, b->d_steps, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	*steps = v;
	return GRAY_OK;
}

static int
check_plan(const gray_launch_plan *p)
{
	if(!p || (p->rays_per_thread != 1 && p->rays_per_thread != 2) ||
	   (p->rk4_rolled != 0 && p->rk4_rolled != 1))
		return GRAY_EINVAL;
	const int maxb = p->rays_per_thread == 2 ? 128 : 256;
	if(p->block < 32 || p->block > maxb || p->block % 32 || p->blocks_per_sm < 0)
		return GRAY_EINVAL;
	return GRAY_OK;
}

extern "C" int
gray_set_plan(gray_ctx *c, const gray_launch_plan *p)
{
	if(!c)
		return GRAY_EINVAL;
	int st = check_plan(p);
	if(st)
		return st;
	c->mixed.block = p->block;
	c->mixed.blocks_per_sm = p->blocks_per_sm;
	c->mixed.rays_per_thread = p->rays_per_thread;
	c->mixed.rk4_rolled = p->rk4_rolled;
	return GRAY_OK;
}

extern "C" int
gray_get_plan(const gray_ctx *c, gray_launch_plan *p)
{
	if(!c || !p)
		return GRAY_EINVAL;
	p->block = c->mixed.block;
	p->blocks_per_sm = c->mixed.blocks_per_sm;
	p->rays_per_thread = c->mixed.rays_per_thread;
	p->rk4_rolled = c->mixed.rk4_rolled;
	p->ns = 0.0;
	return GRAY_OK;
}

/* Candidates: rays per thread {2, 1} x block {64, 128(, 256)} x blocks per
 * SM {all that fit, half of them} x RK4 stages {unrolled, looped}.  Each is timed (best of two) over the
 * first two dump intervals of every render in the batch, launched directly
 * (not through the graph). */
extern "C" int
gray_plan(gray_ctx *c, int id, int flags, gray_launch_plan *best)
{
	Batch *b = find_batch(c, id);
	if(!b)
		return GRAY_ENOTFOUND;
	if(!best || (flags != GRAY_PLAN_ESTIMATE && flags != GRAY_PLAN_MEASURE))
		return GRAY_EINVAL;
	CK(cudaSetDevice(c->device));
	if(flags == GRAY_PLAN_ESTIMATE || b->spacetime == GRAY_ST_NUMERICAL) {
		/* the rule: 256 threads, one ray each (the numerical kernel has
		 * only this shape) */
		c->mixed = MixedLaunch{256, 0, c->sms, 1, 0};
		return gray_get_plan(c, best);
	}
	/* trial table: the first two dump intervals of every render */
	std::vector<MixedRender> trial;
	try {
		trial = b->host_table;
	} catch(const std::bad_alloc &) {
		return GRAY_ENOMEM;
	}
	for(auto &m : trial)
		m.dump_end = m.dump_begin + (m.dump_end - m.dump_begin > 2 ? 2 : m.dump_end - m.dump_begin);
	CK(cudaMemcpyAsync(b->d_table, trial.data(), trial.size() * sizeof(MixedRender),
	                   cudaMemcpyHostToDevice, c->stream));
	MixedTable T = batch_table(b);
	MixedLaunch cand[32];
	int nc = 0;
	for(int rolled = 0; rolled <= 1; ++rolled)
		for(int rpt = 2; rpt >= 1; --rpt)
			for(int blk = 64; blk <= (rpt == 2 ? 128 : 256); blk *= 2) {
				MixedLaunch m = {blk, 0, c->sms, rpt, rolled};
				int occ = 0;
				if(mixed_occupancy(b->n_freq, m, &occ) != cudaSuccess || occ <= 0)
					continue;
				cand[nc++] = m;
				if(occ >= 2) {
					m.blocks_per_sm = occ / 2;
					cand[nc++] = m;
				}
			}
	double best_ns = 1e300;
	MixedLaunch best_cfg = c->mixed;
	int st = GRAY_OK;
	for(int k = 0; k < nc && !st; ++k) {
		for(int rep = 0; rep < 2 && !st; ++rep) {
			double ns = 0.0;
			if((st = timed_begin(c)))
				break;
			if((st = batch_enqueue(c, b, cand[k], T, trial.size() == 1 ? &trial[0] : nullptr)))
				break;
			if((st = timed_end(c, &ns)))
				break;
			if(ns < best_ns) {
				best_ns = ns;
				best_cfg = cand[k];
			}
		}
	}
	/* restore the full schedule */
	cudaError_t e = cudaMemcpyAsync(b->d_table, b->host_table.data(),
	                                b->host_table.size() * sizeof(MixedRender),
	                                cudaMemcpyHostToDevice, c->stream);
	if(e == cudaSuccess)
		e = cudaStreamSynchronize(c->stream);
	if(st)
		return st;
	if(e != cudaSuccess)
		return from_cuda(e);
	c->mixed = best_cfg;
	gray_get_plan(c, best);
	best->ns = best_ns;
	return GRAY_OK;
}

extern "C" int
gray_gather_steps(gray_ctx *c, int id, uint64_t *steps)
{
	Render *r = find(c, id);
	if(!r)
		return GRAY_ENOTFOUND;
	if(!steps)
		return GRAY_EINVAL;
	CK(cudaSetDevice(c->device));
	unsigned long long v = 0;
	CK(cudaMemcpyAsync(&v, r->d_steps + 1, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	*steps = v;
	return GRAY_OK;
}
