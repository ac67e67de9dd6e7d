/*
 * The reference's numerical-spacetime program (sim-org: preamble.cl,
 * interp.cl, dyst.cl, flow.cl, rt.cl, AoS.cl, phys.cl, RK4.cl, driver.cl --
 * the source list of sim-org/build.c:85-95 with coordinates = dyst.cl),
 * compiled from the reference's own files with opencl_shim.h -- TEST
 * INFRASTRUCTURE ONLY.
 *
 * Supplied here, and nothing else: the build-time definitions
 * sim-org/build.c:100-122 prepends (one frequency: n_freq, n_data, n_info,
 * the ray counts, n_chunk, realE, nus, M_ADM), and the 102 images of the two
 * time levels, which read the interleaved [z][y][x][51] levels in place.
 * The bounding box is passed as reals, which is what the kernels declare;
 * the reference's host passes a cl_float8 (sim-org/evolve.c:55), which an
 * FP64 build would misread.  The entry point runs icond_drv and evolve_drv
 * over a list of rays, one work-item at a time, dump by dump as the host
 * loop of sim-org/gray.c:243-294 drives them on one snapshot pair.
 */
#include "opencl_shim.h"

#include <vector>

thread_local size_t gray_shim_gid[2];

namespace ref_dyst {

#define n_freq 1
#define n_data 10
#define n_info 1
static size_t w_rays_v, h_rays_v;
#define w_rays w_rays_v
#define h_rays h_rays_v
#define n_rays (w_rays_v * h_rays_v)
#define n_chunk 5
typedef real2 realE;
static real nus[1];
static real M_ADM;

#include "preamble.cl"
#include "interp.cl"
#include "dyst.cl"
#include "flow.cl"
#include "rt.cl"
#include "AoS.cl"
#include "phys.cl"
#include "RK4.cl"
#include "driver.cl"

} /* namespace ref_dyst */

using namespace ref_dyst;

struct ref_dyst_desc {
	double w_img, h_img, r_obs, i_obs, j_obs;
	int64_t w_rays, h_rays;
	double t_init, dt_dump;
	int64_t n_sub, n_dump;
	double nu, m_adm;          /* the one frequency (Hz) and M_ADM */
	double box[8];             /* {t1, xmin, ymin, zmin, t2, xmax, ymax, zmax} */
	int nx, ny, nz;
};

extern "C" int
ref_dyst_trace(const ref_dyst_desc *d, const float *lv1, const float *lv2, const int64_t *rays,
               int64_t n, double *out, double *info)
{
	w_rays_v = (size_t)d->w_rays;
	h_rays_v = (size_t)d->h_rays;
	nus[0] = d->nu;
	M_ADM = d->m_adm;
	real8 bounding_box;
	for(int i = 0; i < 8; ++i)
		bounding_box.v[i] = d->box[i];
	int4 num_points = {0, d->nx, d->ny, d->nz}; /* s1..s3 are read (interp.cl) */
	const float *lv[2] = {lv1, lv2};
	auto img = [&](int l, int c) { return image3d_t{lv[l], d->nx, d->ny, d->nz, 51, c}; };
#include "dyst_images.inc"
	std::vector<real> data((size_t)n_data * n_rays), inf((size_t)n_info * n_rays);
	for(int64_t j = 0; j < n; ++j) {
		const int64_t g = rays[j];
		if(g < 0 || (size_t)g >= n_rays)
			return -1;
		gray_shim_gid[0] = (size_t)(g / d->w_rays); /* gj: row    */
		gray_shim_gid[1] = (size_t)(g % d->w_rays); /* gi: column */
		icond_drv(data.data(), inf.data(), d->w_img, d->h_img, d->r_obs, d->i_obs, d->j_obs,
		          nullptr, SPACETIME_ARGS);
		for(int64_t i = 0; i < d->n_dump;) {
			const real t = d->t_init + (real)i * d->dt_dump;
			const real target = d->t_init + (real)(++i) * d->dt_dump;
			evolve_drv(data.data(), inf.data(), target - t, (whole)d->n_sub, nullptr,
			           SPACETIME_ARGS);
		}
		for(int s = 0; s < n_data; ++s)
			out[j * n_data + s] = data[(size_t)g * n_data + s];
		info[j] = inf[(size_t)g];
	}
	return 0;
}
