/*
 * The context and its objects (renders, grid, batches, server), shared by
 * gray_api.cu and serve.cu.  Not part of the public ABI.
 */
#ifndef GRAY_CTX_INTERNAL_H
#define GRAY_CTX_INTERNAL_H

#include <map>
#include <mutex>
#include <vector>

#include "gray_internal.h"
#include "mixed_table.h"

struct Render {
	gray_render_desc desc;
	RenderParams p;
	double *d_data = nullptr;
	double *d_info = nullptr;
	unsigned long long *d_steps = nullptr;
	unsigned int *d_queue = nullptr;
	MixedRender *d_table = nullptr;       /* one-entry table for gray_run */
	unsigned long long *d_prefix = nullptr;
	size_t bytes = 0;
	bool has_state = false;
};

struct Grid {
	gray_grid_desc desc;
	bool loaded[2] = {false, false};
	float *lvl[2] = {nullptr, nullptr};
	float *spare = nullptr;         /* third level of a snapshot series    */
	float *staging = nullptr;       /* pinned host snapshot (series loads) */
	double *nodes[3] = {nullptr, nullptr, nullptr};
	float *nodes_f[3] = {nullptr, nullptr, nullptr};
	size_t bytes = 0;
	GridParams gp;
};

struct Batch {
	std::vector<int> ids;
	int spacetime = GRAY_ST_KERR;
	int n_freq = 0;
	unsigned long long total = 0;
	void *block = nullptr;          /* table | prefix | queue | steps      */
	size_t bytes = 0;
	MixedRender *d_table = nullptr;
	unsigned long long *d_prefix = nullptr;
	unsigned int *d_queue = nullptr;
	unsigned long long *d_steps = nullptr;
	std::vector<MixedRender> host_table;
	cudaGraphExec_t exec = nullptr;
	MixedLaunch graph_cfg = {0, 0, 0, 0};
	cudaStream_t graph_stream = nullptr;
	/* numerical batches: the grid parameters the graph's launches were
	 * captured with (level pointers, time box, node tables) */
	GridParams graph_gp;
};

struct Server; /* serve.cu */

struct gray_ctx {
	int device = 0;
	size_t budget = 0;
	size_t used = 0;
	std::mutex mem_mu;               /* budget accounting (server thread) */
	int sms = 0;
	cudaStream_t own = nullptr;
	cudaStream_t stream = nullptr;
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	std::map<int, Render *> renders;
	int next_id = 1;
	Grid *grid = nullptr;
	int evolve64_block = 128;
	/* default plan (GRAY_PLAN_ESTIMATE): one ray per thread, 256-thread
	 * blocks -- the shape the measuring planner picks on B200 for the
	 * analytic torus renders */
	MixedLaunch mixed = {256, 0, 0, 1};
	std::map<int, Batch *> batches;
	int next_batch = 1;
	Server *server = nullptr;
};

/* helpers of gray_api.cu shared with serve.cu */
int  gi_from_cuda(cudaError_t e);
int  gi_dalloc(gray_ctx *c, void **p, size_t bytes);
void gi_dfree(gray_ctx *c, void *p, size_t bytes);
/* the HBM budget without an allocation (memory from the server's pool) */
int  gi_reserve(gray_ctx *c, size_t bytes);
void gi_unreserve(gray_ctx *c, size_t bytes);
int  gi_grid_ready(gray_ctx *c);
Render *gi_find_render(gray_ctx *c, int id);
int  gi_icond(gray_ctx *c, Render *r);
int  gi_evolve_interval(gray_ctx *c, Render *r, double t, double target, uint64_t n_sub);
int  gi_check_grid(const gray_grid_desc *g);
int  gi_ensure_grid(gray_ctx *c, const gray_grid_desc *g);
int  gi_timed_begin(gray_ctx *c);
int  gi_timed_end(gray_ctx *c, double *ns);
void gi_serve_shutdown(gray_ctx *c); /* serve.cu: stop and free the server */

#endif /* GRAY_CTX_INTERNAL_H */
