/*
 * The GRay2 lux job in C, driving libgray_cuda.
 *
 * Options: the union of the reference's run-time tables, same names,
 * aliases and defaults --
 *   sim/gray.opts:1-14      i_platform:ip i_device:id device_type:type
 *                           spacetime:st initcond:ic t_init:t0 dt_dump:dt
 *                           i_init:i0 n_dump:N rayfile:ray
 *   sim/Kerr.opts:1-2       m_bh:M a_spin:a
 *   sim/infcam.opts:2-11    w_img:w h_img:h r_obs:r i_obs:i j_obs:j
 *                           coordinates:coor n_width:W n_height:H
 *   sim-org/setup.opts:6-15 precision:p scheme:scm morder:mo:ml kflags:kf
 *                           outfile:out n_sub:n
 *   sim-org/param.opts:4-18 M_ADM:m dyst_file:data enable_fast_light:fast_light
 *                           n_electron:ne beta_crit:bc R_high:Rh R_low:Rl nu
 * plus the options of the analytic torus (flow, torus_n0, torus_kappa,
 * torus_hr), of the thermal flow (flow_te:te, flow_b:b; flow.cl:51-52 fixes
 * them at 1e12 and 0), the stop rule (term) and the launch planner (plan:pl,
 * measure or estimate).  conf() follows the lux convention:
 * 0 when the argument was consumed (sim/gray.c:37-73).
 *
 * init() replaces sim/gray.c:75-151 (device, ray buffer, initcond, planner);
 * exec() replaces the dump loop of sim-org/gray.c:243-294 with the per-dump
 * evolve the new tree leaves as a TODO (sim/gray.c:168), and writes the raw
 * dumps of sim-org/io.c:39-72 (outfile) and the HDF5 /rays files of
 * sim/gray.c:170-176 (rayfile); either is switched off by an empty name.
 *
 * spacetime=dyst is the numerical spacetime of sim-org (dyst.cl, built in
 * place of KS.cl there): the snapshots come from the HDF5 file dyst_file
 * (sim-org/gray.c:164-230, io.c:149-533) and stream through
 * gray_run_series, one snapshot pair per dump interval as
 * sim-org/gray.c:243-294 switches them.
 */
#include "gray_job.h"
#include "gray_h5.h"

#include <errno.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef enum { T_DBL, T_SIZE, T_UINT, T_STR, T_LIST, T_PREC } opt_type;

struct gray_job {
	gray_lux_job super;

	/* sim/gray.opts */
	unsigned i_platform, i_device;
	char     device_type[32];
	char     spacetime[32];
	char     initcond[32];
	double   t_init, dt_dump;
	size_t   i_init, n_dump;
	char     rayfile[256];
	/* sim/Kerr.opts */
	double   m_bh, a_spin;
	/* sim/infcam.opts */
	double   w_img, h_img, r_obs, i_obs, j_obs;
	char     coordinates[32];
	size_t   n_width, n_height;
	/* sim-org/setup.opts */
	int      precision;          /* size of real: 4 (mixed here) or 8 */
	char     scheme[16];
	char     morder[16];
	char     kflags[64];
	char     outfile[256];
	size_t   n_sub;
	/* sim-org/param.opts */
	double   M_ADM;
	char     dyst_file[256];
	size_t   enable_fast_light;
	double   n_electron, beta_crit, R_high, R_low;
	double   nu[GRAY_MAX_FREQ];
	int      n_freq;
	/* analytic torus and stop rule */
	char     flow[16];
	double   torus_n0, torus_kappa, torus_hr;
	double   flow_te, flow_b;
	char     term[16];
	char     plan[16];

	/* run time */
	gray_ctx *ctx;
	int       render;
	gray_h5_spacetime *sf;   /* spacetime=dyst: the open dyst_file */
	gray_grid_desc     grid;
	uint64_t  steps;
	double    ns;
};

#define EGO ((struct gray_job *)ego)
#define OFF(f) offsetof(struct gray_job, f)
#define SZ(f)  sizeof(((struct gray_job *)0)->f)

typedef struct {
	const char *names;   /* "name:alias:alias" */
	opt_type    type;
	size_t      off, size;
	const char *dflt;
} opt;

static const opt OPTS[] = {
	{"i_platform:ip",        T_UINT, OFF(i_platform), SZ(i_platform), "0"},
	{"i_device:id",          T_UINT, OFF(i_device), SZ(i_device), "0"},
	{"device_type:type",     T_STR,  OFF(device_type), SZ(device_type), "all"},
	{"spacetime:st",         T_STR,  OFF(spacetime), SZ(spacetime), "Kerr"},
	{"initcond:ic",          T_STR,  OFF(initcond), SZ(initcond), "infcam"},
	{"t_init:t0",            T_DBL,  OFF(t_init), SZ(t_init), "0"},
	{"dt_dump:dt",           T_DBL,  OFF(dt_dump), SZ(dt_dump), "-32"},
	{"i_init:i0",            T_SIZE, OFF(i_init), SZ(i_init), "0"},
	{"n_dump:N",             T_SIZE, OFF(n_dump), SZ(n_dump), "64"},
	{"rayfile:ray",          T_STR,  OFF(rayfile), SZ(rayfile), "ray%04d.h5"},
	{"m_bh:M",               T_DBL,  OFF(m_bh), SZ(m_bh), "4e6"},
	{"a_spin:a",             T_DBL,  OFF(a_spin), SZ(a_spin), "0"},
	{"w_img:w",              T_DBL,  OFF(w_img), SZ(w_img), "64"},
	{"h_img:h",              T_DBL,  OFF(h_img), SZ(h_img), "64"},
	{"r_obs:r",              T_DBL,  OFF(r_obs), SZ(r_obs), "1024"},
	{"i_obs:i",              T_DBL,  OFF(i_obs), SZ(i_obs), "60"},
	{"j_obs:j",              T_DBL,  OFF(j_obs), SZ(j_obs), "0"},
	{"coordinates:coor",     T_STR,  OFF(coordinates), SZ(coordinates), "pxcenter"},
	{"n_width:W:w_rays",     T_SIZE, OFF(n_width), SZ(n_width), "512"},
	{"n_height:H:h_rays",    T_SIZE, OFF(n_height), SZ(n_height), "512"},
	{"precision:p",          T_PREC, OFF(precision), SZ(precision), "4"},
	{"scheme:scm",           T_STR,  OFF(scheme), SZ(scheme), "RK4"},
	{"morder:mo:ml",         T_STR,  OFF(morder), SZ(morder), "AoS"},
	{"kflags:kf",            T_STR,  OFF(kflags), SZ(kflags), "-w"},
	{"outfile:out",          T_STR,  OFF(outfile), SZ(outfile), "%04d.raw"},
	{"n_sub:n",              T_SIZE, OFF(n_sub), SZ(n_sub), "1024"},
	{"M_ADM:m",              T_DBL,  OFF(M_ADM), SZ(M_ADM), "4.3e6"},
	{"dyst_file:data",       T_STR,  OFF(dyst_file), SZ(dyst_file), "data.h5"},
	{"enable_fast_light:fast_light", T_SIZE, OFF(enable_fast_light), SZ(enable_fast_light), "0"},
	{"n_electron:ne",        T_DBL,  OFF(n_electron), SZ(n_electron), "1e6"},
	{"beta_crit:bc",         T_DBL,  OFF(beta_crit), SZ(beta_crit), "1"},
	{"R_high:Rh",            T_DBL,  OFF(R_high), SZ(R_high), "1"},
	{"R_low:Rl",             T_DBL,  OFF(R_low), SZ(R_low), "1"},
	{"nu",                   T_LIST, OFF(nu), SZ(nu), ""},
	{"flow",                 T_STR,  OFF(flow), SZ(flow), "torus"},
	{"torus_n0",             T_DBL,  OFF(torus_n0), SZ(torus_n0), "1"},
	{"torus_kappa",          T_DBL,  OFF(torus_kappa), SZ(torus_kappa), "1"},
	{"torus_hr",             T_DBL,  OFF(torus_hr), SZ(torus_hr), "0.3"},
	{"flow_te:te",           T_DBL,  OFF(flow_te), SZ(flow_te), "1e12"},
	{"flow_b:b",             T_DBL,  OFF(flow_b), SZ(flow_b), "0"},
	{"plan:pl",              T_STR,  OFF(plan), SZ(plan), "measure"},
	{"term",                 T_STR,  OFF(term), SZ(term), "eps"},
};
#define N_OPTS (sizeof(OPTS) / sizeof(OPTS[0]))

/* name matches one of the ':'-separated names of o */
static int
matches(const opt *o, const char *name, size_t len)
{
	const char *p = o->names;
	while(*p) {
		const char *e = strchr(p, ':');
		size_t n = e ? (size_t)(e - p) : strlen(p);
		if(n == len && strncmp(p, name, len) == 0)
			return 1;
		if(!e)
			break;
		p = e + 1;
	}
	return 0;
}

/* parse a full double; the whole token must be consumed */
static int
parse_dbl(const char *s, double *v)
{
	char *rem;
	errno = 0;
	*v = strtod(s, &rem);
	return (rem == s || *rem != '\0' || errno == ERANGE) ? GRAY_EINVAL : GRAY_OK;
}

static int
parse_size(const char *s, size_t *v)
{
	char *rem;
	if(*s == '-')
		return GRAY_EINVAL;
	errno = 0;
	unsigned long long x = strtoull(s, &rem, 0);
	if(rem == s || *rem != '\0' || errno == ERANGE)
		return GRAY_EINVAL;
	*v = (size_t)x;
	return GRAY_OK;
}

/* strtoprec of setup.opts: "4"/"single"/"float" or "8"/"double"; "mixed"
 * names the FP32-bulk path, which is what the single-precision request
 * runs here. */
static int
parse_prec(const char *s, int *v)
{
	if(!strcmp(s, "4") || !strcmp(s, "single") || !strcmp(s, "float") || !strcmp(s, "mixed"))
		*v = 4;
	else if(!strcmp(s, "8") || !strcmp(s, "double"))
		*v = 8;
	else
		return GRAY_EINVAL;
	return GRAY_OK;
}

/* strtoda of param.opts:18: a comma-separated list of reals; empty or
 * "none" turns transfer off (the reference's NaN-terminated empty list). */
static int
parse_list(const char *s, double *v, int *n)
{
	int k = 0;
	char buf[512];
	if(!*s || !strcmp(s, "none")) {
		*n = 0;
		return GRAY_OK;
	}
	if(strlen(s) >= sizeof(buf))
		return GRAY_EINVAL;
	strcpy(buf, s);
	for(char *tok = strtok(buf, ","); tok; tok = strtok(NULL, ",")) {
		double x;
		if(k == GRAY_MAX_FREQ || parse_dbl(tok, &x) || !(x > 0.0))
			return GRAY_EINVAL;
		v[k++] = x;
	}
	*n = k;
	return GRAY_OK;
}

static int
set_opt(struct gray_job *j, const opt *o, const char *val)
{
	void *dst = (char *)j + o->off;
	switch(o->type) {
	case T_DBL: {
		double v;
		if(parse_dbl(val, &v))
			return GRAY_EINVAL;
		*(double *)dst = v;
		return GRAY_OK;
	}
	case T_SIZE: {
		size_t v;
		if(parse_size(val, &v))
			return GRAY_EINVAL;
		*(size_t *)dst = v;
		return GRAY_OK;
	}
	case T_UINT: {
		size_t v;
		if(parse_size(val, &v) || v > 0xffffffffu)
			return GRAY_EINVAL;
		*(unsigned *)dst = (unsigned)v;
		return GRAY_OK;
	}
	case T_STR:
		if(strlen(val) >= o->size)
			return GRAY_EINVAL;
		strcpy((char *)dst, val);
		return GRAY_OK;
	case T_LIST:
		return parse_list(val, (double *)dst, &j->n_freq);
	case T_PREC:
		return parse_prec(val, (int *)dst);
	}
	return GRAY_EINVAL;
}

/* A file-name pattern takes at most one integer conversion, the dump index
 * (sim-org/io.c formats the name with it); any other conversion would make
 * snprintf read an argument that is not there. */
static int
valid_pattern(const char *s)
{
	int conv = 0;
	for(const char *p = s; *p; ++p) {
		if(*p != '%')
			continue;
		++p; /* the character after '%' */
		if(*p == '%')
			continue; /* a literal percent sign */
		while(*p && strchr("-+ #0", *p))
			++p;
		while(*p >= '0' && *p <= '9')
			++p;
		if(*p == '.')
			for(++p; *p >= '0' && *p <= '9'; ++p)
				;
		if(!*p || !strchr("diouxX", *p) || ++conv > 1)
			return 0;
	}
	return 1;
}

static int
valid_choices(const struct gray_job *j)
{
	if(strcmp(j->spacetime, "Kerr") && strcmp(j->spacetime, "KS") && strcmp(j->spacetime, "dyst"))
		return 0; /* sim/gray.c:55-57: unknown spacetime */
	if(strcmp(j->initcond, "infcam"))
		return 0; /* sim/gray.c:67-69: unknown initial conditions */
	if(strcmp(j->scheme, "RK4"))
		return 0; /* sim-org/setup.opts:7: the only scheme shipped */
	if(strcmp(j->morder, "AoS") && strcmp(j->morder, "SoA"))
		return 0;
	if(strcmp(j->flow, "torus") && strcmp(j->flow, "none") && strcmp(j->flow, "thermal"))
		return 0;
	if(strcmp(j->term, "eps") && strcmp(j->term, "rplus"))
		return 0;
	if(strcmp(j->plan, "measure") && strcmp(j->plan, "estimate"))
		return 0;
	if(!valid_pattern(j->outfile) || !valid_pattern(j->rayfile))
		return 0;
	return 1;
}

static int
conf(gray_lux_job *ego, const char *arg)
{
	const char *eq = arg ? strchr(arg, '=') : NULL;
	if(!eq)
		return GRAY_JOB_UNKNOWN;
	for(size_t k = 0; k < N_OPTS; ++k) {
		if(!matches(&OPTS[k], arg, (size_t)(eq - arg)))
			continue;
		struct gray_job save = *EGO;
		int st = set_opt(EGO, &OPTS[k], eq + 1);
		if(st == GRAY_OK && !valid_choices(EGO))
			st = GRAY_EINVAL;
		if(st != GRAY_OK)
			*EGO = save; /* a rejected value leaves the job unchanged */
		return st;
	}
	return GRAY_JOB_UNKNOWN;
}

int
gray_job_desc(const gray_lux_job *ego, gray_render_desc *d)
{
	if(!ego || !d)
		return GRAY_EINVAL;
	const struct gray_job *j = (const struct gray_job *)ego;
	memset(d, 0, sizeof(*d));
	d->m_bh = j->m_bh;
	d->a_spin = j->a_spin;
	d->w_img = j->w_img;
	d->h_img = j->h_img;
	d->r_obs = j->r_obs;
	d->i_obs = j->i_obs;
	d->j_obs = j->j_obs;
	d->n_width = j->n_width;
	d->n_height = j->n_height;
	d->t_init = j->t_init;
	d->dt_dump = j->dt_dump;
	d->n_sub = j->n_sub;
	d->n_dump = j->n_dump;
	d->term = strcmp(j->term, "rplus") ? GRAY_TERM_EPS : GRAY_TERM_RPLUS;
	d->n_freq = j->n_freq;
	for(int i = 0; i < j->n_freq; ++i)
		d->nu[i] = j->nu[i];
	d->flow = !j->n_freq                   ? GRAY_FLOW_NONE
	          : !strcmp(j->flow, "torus")   ? GRAY_FLOW_TORUS
	          : !strcmp(j->flow, "thermal") ? GRAY_FLOW_THERMAL
	                                        : GRAY_FLOW_NONE;
	d->m_adm = j->M_ADM;
	d->flow_te = j->flow_te;
	d->flow_b = j->flow_b;
	d->torus_n0 = j->torus_n0;
	d->torus_kappa = j->torus_kappa;
	d->torus_hr = j->torus_hr;
	d->spacetime = strcmp(j->spacetime, "dyst") ? GRAY_ST_KERR : GRAY_ST_NUMERICAL;
	d->precision = j->precision == 8 ? GRAY_PREC_FP64 : GRAY_PREC_MIXED;
	return GRAY_OK;
}

int
gray_job_get(const gray_lux_job *ego, const char *name, char *buf, size_t len)
{
	if(!ego || !name || !buf || !len)
		return GRAY_EINVAL;
	const struct gray_job *j = (const struct gray_job *)ego;
	for(size_t k = 0; k < N_OPTS; ++k) {
		const opt *o = &OPTS[k];
		if(!matches(o, name, strlen(name)))
			continue;
		const void *src = (const char *)j + o->off;
		int n = 0;
		switch(o->type) {
		case T_DBL:  n = snprintf(buf, len, "%.17g", *(const double *)src); break;
		case T_SIZE: n = snprintf(buf, len, "%zu", *(const size_t *)src); break;
		case T_UINT: n = snprintf(buf, len, "%u", *(const unsigned *)src); break;
		case T_STR:  n = snprintf(buf, len, "%s", (const char *)src); break;
		case T_PREC: n = snprintf(buf, len, "%d", *(const int *)src); break;
		case T_LIST: {
			size_t used = 0;
			buf[0] = '\0';
			for(int i = 0; i < j->n_freq && used < len; ++i)
				used += (size_t)snprintf(buf + used, len - used, i ? ",%.17g" : "%.17g", j->nu[i]);
			n = (int)used;
			break;
		}
		}
		return (n < 0 || (size_t)n >= len) ? GRAY_ESIZE : GRAY_OK;
	}
	return GRAY_ENOTFOUND;
}

int
gray_job_stats(const gray_lux_job *ego, uint64_t *ray_steps, double *kernel_ns)
{
	if(!ego)
		return GRAY_EINVAL;
	if(ray_steps)
		*ray_steps = EGO->steps;
	if(kernel_ns)
		*kernel_ns = EGO->ns;
	return GRAY_OK;
}

int
gray_write_raw(const char *path, const double *data, const double *info,
               size_t n_data, size_t w, size_t h)
{
	const size_t sz = sizeof(double), n_rays = w * h, n_info = 1;
	FILE *f = fopen(path, "wb");
	if(!f)
		return GRAY_EINVAL;
	int ok = fwrite(&sz, sizeof(size_t), 1, f) == 1 &&
	         fwrite(&n_data, sizeof(size_t), 1, f) == 1 &&
	         fwrite(&w, sizeof(size_t), 1, f) == 1 &&
	         fwrite(&h, sizeof(size_t), 1, f) == 1 &&
	         fwrite(data, sz * n_data, n_rays, f) == n_rays &&
	         fwrite(info, sz * n_info, n_rays, f) == n_rays;
	return (fclose(f) == 0 && ok) ? GRAY_OK : GRAY_EINVAL;
}

int
gray_read_raw(const char *path, double *data, double *info, size_t n_data, size_t w, size_t h)
{
	size_t hdr[4];
	const size_t n_rays = w * h;
	if(!path || !data || !info)
		return GRAY_EINVAL;
	FILE *f = fopen(path, "rb");
	if(!f)
		return GRAY_ENOTFOUND;
	int st = GRAY_OK;
	if(fread(hdr, sizeof(size_t), 4, f) != 4 || hdr[0] != sizeof(double) ||
	   hdr[1] != n_data || hdr[2] != w || hdr[3] != h)
		st = GRAY_ESIZE;
	else if(fread(data, sizeof(double) * n_data, n_rays, f) != n_rays ||
	        fread(info, sizeof(double), n_rays, f) != n_rays)
		st = GRAY_ESIZE;
	fclose(f);
	return st;
}

/* The dump layout the reference writes: sim-org/io.c:52-67 writes the
 * device buffer as it is, so the element size is the run's precision
 * (4 bytes for p=4, 8 for p=8) and the order is morder (AoS or SoA). */
static size_t
dump_size(const struct gray_job *j)
{
	return j->precision == 8 ? sizeof(double) : sizeof(float);
}

static int
dump_layout(const struct gray_job *j)
{
	return strcmp(j->morder, "SoA") ? GRAY_LAYOUT_AOS : GRAY_LAYOUT_SOA;
}

/* Resume at dump i_init from the dump file a previous run wrote there
 * (the checkpoint the reference's dumps are but cannot load, io.c:37).
 * GRAY_ENOTFOUND when there is no such file: the run then starts from the
 * camera as the reference does. */
static int
resume(struct gray_job *j, size_t i)
{
	if(!j->outfile[0] || i == 0)
		return GRAY_ENOTFOUND;
	gray_render_desc d;
	gray_job_desc(&j->super, &d);
	const size_t n_rays = d.n_width * d.n_height;
	const size_t n_data = 8 + 2 * (size_t)d.n_freq;
	const size_t n = n_rays * n_data, sz = dump_size(j);
	char name[512];
	snprintf(name, sizeof(name), j->outfile, (int)i);
	FILE *f = fopen(name, "rb");
	if(!f)
		return GRAY_ENOTFOUND;
	size_t hdr[4];
	double *data = malloc(sizeof(double) * n);
	void *raw = malloc(sz * n);
	int st = (data && raw) ? GRAY_OK : GRAY_ENOMEM;
	if(!st && (fread(hdr, sizeof(size_t), 4, f) != 4 || hdr[0] != sz || hdr[1] != n_data ||
	           hdr[2] != d.n_width || hdr[3] != d.n_height || fread(raw, sz, n, f) != n))
		st = GRAY_ESIZE;
	fclose(f);
	if(!st) {
		for(size_t k = 0; k < n; ++k)
			data[k] = sz == sizeof(float) ? (double)((float *)raw)[k] : ((double *)raw)[k];
		st = gray_write_state(j->ctx, j->render, data, sizeof(double) * n, dump_layout(j));
	}
	free(raw);
	free(data);
	return st;
}

/* sim/gray.c:170-176: after interval i (>= 1) the rays, copied to the host
 * as an array {n_width, n_height, n_data} of the run's real type, go to a
 * new HDF5 file rayfile % i as the dataset /rays (never overwritten: the
 * reference opens it with H5F_ACC_EXCL) */
static int
dump_rays(struct gray_job *j, size_t i)
{
	if(!j->rayfile[0])
		return GRAY_OK;
	gray_render_desc d;
	gray_job_desc(&j->super, &d);
	const size_t n_rays = d.n_width * d.n_height;
	const size_t n_data = 8 + 2 * (size_t)d.n_freq, n = n_rays * n_data;
	double *data = malloc(sizeof(double) * n);
	double *info = malloc(sizeof(double) * n_rays);
	int st = (data && info) ? GRAY_OK : GRAY_ENOMEM;
	if(!st)
		st = gray_read_state(j->ctx, j->render, data, sizeof(double) * n, info,
		                     sizeof(double) * n_rays, GRAY_LAYOUT_AOS);
	if(!st) {
		char name[512];
		snprintf(name, sizeof(name), j->rayfile, (int)i);
		const int sz = (int)dump_size(j);
		if(sz == (int)sizeof(float)) {
			float *f = (float *)data; /* narrowed in place, front to back */
			for(size_t k = 0; k < n; ++k)
				f[k] = (float)data[k];
		}
		int h = gray_h5_write_rays(name, data, sz, d.n_width, d.n_height, n_data);
		st = h == GRAY_H5_OK ? GRAY_OK : h == GRAY_H5_EEXIST ? GRAY_ESTATE : GRAY_EINVAL;
		if(h)
			fprintf(stderr, "GRay2: %s: %s\n", name, gray_h5_strerror(h));
	}
	free(data);
	free(info);
	return st;
}

/* sim-org/io.c:39-72 dump(): header {sz, n_data, W, H}, the state, its
 * info diagnostic, in the run's element size and memory order */
static int
dump(struct gray_job *j, size_t i)
{
	if(!j->outfile[0])
		return GRAY_OK; /* dumps switched off */
	gray_render_desc d;
	gray_job_desc(&j->super, &d);
	const size_t n_rays = d.n_width * d.n_height;
	const size_t n_data = 8 + 2 * (size_t)d.n_freq;
	const size_t n = n_rays * n_data, sz = dump_size(j);
	double *data = malloc(sizeof(double) * n);
	double *info = malloc(sizeof(double) * n_rays);
	int st = (data && info) ? GRAY_OK : GRAY_ENOMEM;
	if(!st)
		st = gray_read_state(j->ctx, j->render, data, sizeof(double) * n, info,
		                     sizeof(double) * n_rays, dump_layout(j));
	if(!st) {
		char name[512];
		snprintf(name, sizeof(name), j->outfile, (int)i);
		if(sz == sizeof(double)) {
			st = gray_write_raw(name, data, info, n_data, d.n_width, d.n_height);
		} else { /* p=4: the reference's state is float, so is its dump */
			float *fd = malloc(sizeof(float) * (n + n_rays));
			FILE *f = fd ? fopen(name, "wb") : NULL;
			int ok = 0;
			if(f) {
				for(size_t k = 0; k < n; ++k)
					fd[k] = (float)data[k];
				for(size_t k = 0; k < n_rays; ++k)
					fd[n + k] = (float)info[k];
				const size_t hdr[4] = {sz, n_data, d.n_width, d.n_height};
				ok = fwrite(hdr, sizeof(size_t), 4, f) == 4 &&
				     fwrite(fd, sz, n + n_rays, f) == n + n_rays;
				ok = (fclose(f) == 0) && ok;
			}
			st = fd ? (ok ? GRAY_OK : GRAY_EINVAL) : GRAY_ENOMEM;
			free(fd);
		}
	}
	free(data);
	free(info);
	if(!st && i > 0)
		st = dump_rays(j, i);
	return st;
}

/* sim-org/gray.c:164-205 + io.c:149-275: open dyst_file, list its
 * snapshot times and read the grid; the grid keeps the reference's
 * semantics (clamp-to-edge outside the box, unclamped time extrapolation) */
static int
open_dyst(struct gray_job *j)
{
	int h = gray_h5_spacetime_open(j->dyst_file, &j->sf);
	if(h) {
		fprintf(stderr, "GRay2: %s: %s\n", j->dyst_file, gray_h5_strerror(h));
		return h == GRAY_H5_ENOTFOUND ? GRAY_ENOTFOUND : GRAY_EINVAL;
	}
	const double *times;
	uint64_t nt = gray_h5_spacetime_times(j->sf, &times);
	int n[3];
	float lo[3], hi[3];
	gray_h5_spacetime_grid(j->sf, n, lo, hi);
	memset(&j->grid, 0, sizeof(j->grid));
	j->grid.nx = n[0];
	j->grid.ny = n[1];
	j->grid.nz = n[2];
	for(int a = 0; a < 3; ++a) {
		j->grid.box[1 + a] = lo[a];
		j->grid.box[5 + a] = hi[a];
	}
	printf("GRay2: Reading spacetime from file %s: %llu snapshot(s) in [%g, %g], "
	       "grid %dx%dx%d\n", j->dyst_file, (unsigned long long)nt, times[0], times[nt - 1],
	       n[0], n[1], n[2]);
	return GRAY_OK;
}

static int
init(gray_lux_job *ego)
{
	gray_render_desc d;
	int st;
	printf("GRay2:init: spacetime:st: %s, initcond:ic: %s\n", EGO->spacetime, EGO->initcond);
	gray_job_desc(ego, &d);
	if(EGO->ctx) { /* a second init starts over */
		gray_destroy(EGO->ctx);
		EGO->ctx = NULL;
	}
	gray_h5_spacetime_close(EGO->sf);
	EGO->sf = NULL;
	/* the spacetime file first: a bad file needs no device to be refused */
	if(d.spacetime == GRAY_ST_NUMERICAL && (st = open_dyst(EGO)))
		return st;
	EGO->ctx = gray_create((int)EGO->i_device, 0, &st);
	if(!EGO->ctx)
		return st;
	st = gray_render_create(EGO->ctx, &d, &EGO->render);
	if(st)
		return st;
	/* the lux planner of sim/gray/Kerr/ocl.c:41-75: time the launch shapes
	 * on this render (a mixed one: the FP64 kernel has a single shape);
	 * exec starts from icond, so the trial launches leave no trace */
	if(d.precision == GRAY_PREC_MIXED && d.spacetime == GRAY_ST_KERR &&
	   !strcmp(EGO->plan, "measure")) {
		int batch;
		gray_launch_plan best;
		if((st = gray_batch_create(EGO->ctx, &EGO->render, 1, &batch)))
			return st;
		st = gray_plan(EGO->ctx, batch, GRAY_PLAN_MEASURE, &best);
		gray_batch_destroy(EGO->ctx, batch);
		if(st)
			return st;
		printf("GRay2:init: plan: block %d, rays/thread %d, RK4 %s\n", best.block,
		       best.rays_per_thread, best.rk4_rolled ? "looped" : "unrolled");
	}
	EGO->steps = 0;
	EGO->ns = 0.0;
	return GRAY_OK;
}

typedef struct {
	struct gray_job *j;
	const double    *times;
	size_t           i;
} series_user;

static int
series_load(void *user, uint64_t k, float *fields)
{
	series_user *u = (series_user *)user;
	return gray_h5_spacetime_load(u->j->sf, k, fields) != GRAY_H5_OK;
}

static int
series_dump(void *user, uint64_t i)
{
	series_user *u = (series_user *)user;
	struct gray_job *j = u->j;
	printf("%llu: %4.1f -> %4.1f", (unsigned long long)i,
	       j->t_init + (double)(i - 1) * j->dt_dump, j->t_init + (double)i * j->dt_dump);
	int st = dump(j, i);
	printf(st ? ": FAILED\n" : ": DONE\n");
	return st != GRAY_OK;
}

/* sim-org/gray.c:164-294 with spacetime=dyst: icond on the snapshot pair
 * bracketing t_init, dump 0, then the dump intervals with their snapshot
 * pairs streamed by gray_run_series (which repeats the icond on the same
 * pair: the state it integrates is the one dumped).  The reference has no
 * restart from a dump on this path, and neither has the job: i_init must
 * be 0. */
static int
exec_dyst(struct gray_job *j)
{
	const double *times;
	const uint64_t nt = gray_h5_spacetime_times(j->sf, &times);
	if(j->i_init)
		return GRAY_EINVAL;
	int64_t first;
	int st = gray_series_schedule(times, nt, j->t_init, j->dt_dump, 1, (int)j->enable_fast_light,
	                              &first);
	if(st)
		return st;
	const int frozen = nt == 1 || j->enable_fast_light;
	const size_t npts = (size_t)j->grid.nx * j->grid.ny * j->grid.nz;
	float *lv = malloc(sizeof(float) * npts * 51);
	if(!lv)
		return GRAY_ENOMEM;
	gray_grid_desc g = j->grid;
	g.box[0] = (float)times[first];
	g.box[4] = (float)times[frozen ? first : first + 1];
	for(int l = 0; l < 2 && !st; ++l) {
		int h = gray_h5_spacetime_load(j->sf, (uint64_t)(l && !frozen ? first + 1 : first), lv);
		st = h ? GRAY_ESOURCE : gray_load_spacetime_interleaved(j->ctx, &g, lv, l);
	}
	free(lv);
	if(!st)
		st = gray_icond(j->ctx, j->render);
	if(st)
		return st;
	printf("0:  initialize at %4.1f", j->t_init);
	if((st = dump(j, 0)))
		return st;
	printf(": DONE\n");
	series_user u = {j, times, 0};
	gray_snapshot_source src = {nt, times, &u, series_load};
	uint64_t loads = 0;
	double ns = 0.0;
	st = gray_run_series(j->ctx, j->render, &j->grid, &src, (int)j->enable_fast_light,
	                     series_dump, &ns, &loads);
	if(st)
		return st;
	j->ns += ns;
	printf("GRay2: %llu snapshot load(s)\n", (unsigned long long)loads);
	fflush(stdout);
	return gray_ray_steps(j->ctx, j->render, &j->steps);
}

/* sim-org/gray.c:243-294 */
static int
exec(gray_lux_job *ego)
{
	struct gray_job *j = EGO;
	size_t i = j->i_init;
	if(!j->ctx)
		return GRAY_ESTATE;
	if(j->sf)
		return exec_dyst(j);
	const double n_rays = (double)j->n_width * (double)j->n_height;
	int st = resume(j, i);
	if(st == GRAY_OK) {
		printf("%zu:  resumed from its dump\n", i);
	} else if(st == GRAY_ENOTFOUND) {
		if((st = gray_icond(j->ctx, j->render)))
			return st;
		printf("%zu:  initialize at %4.1f", i, j->t_init);
		if((st = dump(j, i)))
			return st;
		printf(": DONE\n");
	} else {
		return st; /* a dump is there but does not fit this run */
	}
	while(i < j->n_dump) {
		double ns;
		double t      = j->t_init + (double)i * j->dt_dump;
		double target = j->t_init + (double)(++i) * j->dt_dump;
		printf("%zu: %4.1f -> %4.1f", i, t, target);
		if((st = gray_evolve(j->ctx, j->render, t, target, j->n_sub, &ns)))
			return st;
		if((st = dump(j, i)))
			return st;
		j->ns += ns;
		printf(": DONE (%.3gns/step/ray)\n", ns / (double)j->n_sub / n_rays);
	}
	fflush(stdout);
	return gray_ray_steps(j->ctx, j->render, &j->steps);
}

gray_lux_job *
gray_job_mkmod(const void *opts)
{
	(void)opts;
	struct gray_job *j = calloc(1, sizeof(*j));
	if(!j)
		return NULL;
	for(size_t k = 0; k < N_OPTS; ++k)
		if(set_opt(j, &OPTS[k], OPTS[k].dflt) != GRAY_OK) {
			free(j);
			return NULL;
		}
	j->super.conf = conf;
	j->super.init = init;
	j->super.exec = exec;
	return &j->super;
}

void
gray_job_rmmod(gray_lux_job *ego)
{
	if(!ego)
		return;
	if(EGO->ctx)
		gray_destroy(EGO->ctx); /* frees the render as well */
	gray_h5_spacetime_close(EGO->sf);
	free(ego);
}
