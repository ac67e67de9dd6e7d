/*
 * Self-contained reader and writer of the classic HDF5 file format for
 * GRay2's spacetime files (sim-org/io.c:149-533, README.md:40-60) and ray
 * files (sim/gray.c:170-176).  See include/gray_h5.h for the subset.
 *
 * Structures follow the HDF5 file format specification (version 0/1
 * superblock, version-1 object headers, symbol-table groups, local heaps,
 * version-1 B-trees of group nodes, dataspace/datatype/fill-value/layout
 * messages).  All multi-byte fields are little-endian; offsets and lengths
 * are 8 bytes.  Every read is bounds-checked against the file size, so a
 * truncated or corrupt file gives GRAY_H5_EFORMAT, never a wild read.
 */
#define _FILE_OFFSET_BITS 64
#define _POSIX_C_SOURCE 200809L
#include "gray_h5.h"

#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/types.h>

#define UNDEF 0xffffffffffffffffull
#define NFIELD 51

static const unsigned char SIG[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

const char *
gray_h5_strerror(int s)
{
	switch(s) {
	case GRAY_H5_OK:        return "success";
	case GRAY_H5_EINVAL:    return "invalid argument";
	case GRAY_H5_ENOMEM:    return "out of memory";
	case GRAY_H5_ENOTFOUND: return "no such file, group or dataset";
	case GRAY_H5_ESIZE:     return "dataset shape or size mismatch";
	case GRAY_H5_EFORMAT:   return "not an HDF5 file, corrupt, or an unsupported HDF5 feature";
	case GRAY_H5_EIO:       return "read or write failed";
	case GRAY_H5_EEXIST:    return "file exists";
	default:                return "unknown status";
	}
}

static uint64_t
le(const unsigned char *p, int n)
{
	uint64_t v = 0;
	for(int i = n - 1; i >= 0; --i)
		v = (v << 8) | p[i];
	return v;
}

static void
put(unsigned char *p, uint64_t v, int n)
{
	for(int i = 0; i < n; ++i, v >>= 8)
		p[i] = (unsigned char)(v & 0xff);
}

/* ======================================================================= */
/* reading                                                                 */
/* ======================================================================= */

struct gray_h5 {
	FILE    *f;
	uint64_t size;  /* bytes in the file                 */
	uint64_t base;  /* base address (superblock location) */
	uint64_t root;  /* root group object header address   */
};

/* n bytes at relative address addr, inside the file */
static int
rd(gray_h5 *h, uint64_t addr, void *buf, uint64_t n)
{
	if(addr == UNDEF)
		return GRAY_H5_EFORMAT;
	uint64_t off = h->base + addr;
	if(off < addr || n > h->size || off > h->size - n)
		return GRAY_H5_EFORMAT;
	if(fseeko(h->f, (off_t)off, SEEK_SET) || fread(buf, 1, (size_t)n, h->f) != (size_t)n)
		return GRAY_H5_EIO;
	return 0;
}

int
gray_h5_open(const char *path, gray_h5 **out)
{
	if(!path || !out)
		return GRAY_H5_EINVAL;
	*out = NULL;
	gray_h5 *h = calloc(1, sizeof(*h));
	if(!h)
		return GRAY_H5_ENOMEM;
	h->f = fopen(path, "rb");
	if(!h->f) {
		free(h);
		return GRAY_H5_ENOTFOUND;
	}
	int st = GRAY_H5_EFORMAT;
	if(fseeko(h->f, 0, SEEK_END) == 0) {
		off_t sz = ftello(h->f);
		h->size = sz > 0 ? (uint64_t)sz : 0;
	}
	/* the superblock sits at 0, 512, 1024, 2048, ... (user block) */
	unsigned char sb[96];
	uint64_t at = UNDEF;
	for(uint64_t o = 0; o + sizeof(sb) <= h->size; o = o ? 2 * o : 512) {
		h->base = 0;
		if(rd(h, o, sb, 8) == 0 && !memcmp(sb, SIG, 8)) {
			at = o;
			break;
		}
	}
	if(at == UNDEF)
		goto fail;
	h->base = 0;
	if(rd(h, at, sb, sizeof(sb)))
		goto fail;
	/* version 0: offsets 13/14, root entry at 56; version 1 has 4 more
	 * bytes (indexed storage K + reserved) before the addresses */
	int ver = sb[8];
	if(ver > 1 || sb[13] != 8 || sb[14] != 8)
		goto fail; /* newer superblock or non-8-byte addresses */
	const unsigned char *a = sb + 24 + (ver == 1 ? 4 : 0);
	h->base = le(a, 8);
	if(h->base == UNDEF || h->base != at)
		h->base = at; /* the base address is the superblock's location */
	const unsigned char *root = a + 32; /* symbol table entry of the root group */
	h->root = le(root + 8, 8);
	*out = h;
	return 0;
fail:
	fclose(h->f);
	free(h);
	return st;
}

void
gray_h5_close(gray_h5 *h)
{
	if(!h)
		return;
	fclose(h->f);
	free(h);
}

/* ---- object headers ------------------------------------------------------ */

typedef struct {
	unsigned type;
	unsigned size;
	uint64_t data; /* address of the message body */
} msgref;

#define MAXMSG 64
#define MAXBLK 16

/* the messages of a version-1 object header, continuation blocks included */
static int
messages(gray_h5 *h, uint64_t oh, msgref *m, int *n)
{
	unsigned char p[16];
	int st = rd(h, oh, p, 16);
	if(st)
		return st;
	if(p[0] != 1)
		return GRAY_H5_EFORMAT; /* version-2 "OHDR" headers are not read */
	uint64_t blk[MAXBLK], len[MAXBLK];
	int nb = 1;
	blk[0] = oh + 16;
	len[0] = le(p + 8, 4);
	*n = 0;
	for(int b = 0; b < nb; ++b) {
		uint64_t at = blk[b], end = blk[b] + len[b];
		if(end < at)
			return GRAY_H5_EFORMAT;
		while(at + 8 <= end) {
			unsigned char mh[8];
			if((st = rd(h, at, mh, 8)))
				return st;
			unsigned type = (unsigned)le(mh, 2), size = (unsigned)le(mh + 2, 2);
			uint64_t data = at + 8;
			if(data + size > end)
				return GRAY_H5_EFORMAT;
			if(mh[4] & 0x02)
				return GRAY_H5_EFORMAT; /* shared messages are not read */
			if(type == 0x0010) { /* continuation: address, length */
				unsigned char c[16];
				if(size < 16 || nb == MAXBLK)
					return GRAY_H5_EFORMAT;
				if((st = rd(h, data, c, 16)))
					return st;
				blk[nb] = le(c, 8);
				len[nb] = le(c + 8, 8);
				++nb;
			} else if(type != 0) {
				if(*n == MAXMSG)
					return GRAY_H5_EFORMAT;
				m[*n].type = type;
				m[*n].size = size;
				m[*n].data = data;
				++*n;
			}
			at = data + size;
		}
	}
	return 0;
}

/* ---- groups ------------------------------------------------------------- */

typedef struct {
	char    *name;
	uint64_t oh;
} entry;

typedef struct {
	entry   *v;
	size_t   n, cap;
	char    *heap;   /* the local heap's data segment */
	uint64_t hsize;
} entries;

static void
free_entries(entries *e)
{
	for(size_t i = 0; i < e->n; ++i)
		free(e->v[i].name);
	free(e->v);
	free(e->heap);
	memset(e, 0, sizeof(*e));
}

static int
add_entry(entries *e, uint64_t name_off, uint64_t oh)
{
	if(name_off >= e->hsize || !memchr(e->heap + name_off, 0, e->hsize - name_off))
		return GRAY_H5_EFORMAT;
	if(e->n == e->cap) {
		size_t cap = e->cap ? 2 * e->cap : 16;
		entry *v = realloc(e->v, cap * sizeof(*v));
		if(!v)
			return GRAY_H5_ENOMEM;
		e->v = v;
		e->cap = cap;
	}
	char *s = strdup(e->heap + name_off);
	if(!s)
		return GRAY_H5_ENOMEM;
	e->v[e->n].name = s;
	e->v[e->n].oh = oh;
	++e->n;
	return 0;
}

/* symbol-table node: "SNOD", version 1, reserved, count, entries of 40 */
static int
snod(gray_h5 *h, uint64_t at, entries *e)
{
	unsigned char p[8];
	int st = rd(h, at, p, 8);
	if(st)
		return st;
	if(memcmp(p, "SNOD", 4) || p[4] != 1)
		return GRAY_H5_EFORMAT;
	unsigned n = (unsigned)le(p + 6, 2);
	for(unsigned i = 0; i < n; ++i) {
		unsigned char s[40];
		if((st = rd(h, at + 8 + 40ull * i, s, 40)))
			return st;
		if((st = add_entry(e, le(s, 8), le(s + 8, 8))))
			return st;
	}
	return 0;
}

/* version-1 B-tree of group nodes (type 0): keys and children alternate
 * after a 24-byte header; level 0 children are symbol-table nodes */
static int
btree(gray_h5 *h, uint64_t at, entries *e, int depth)
{
	unsigned char p[24];
	int st = rd(h, at, p, 24);
	if(st)
		return st;
	if(memcmp(p, "TREE", 4) || p[4] != 0 || depth > 16)
		return GRAY_H5_EFORMAT;
	int level = p[5];
	unsigned used = (unsigned)le(p + 6, 2);
	for(unsigned i = 0; i < used; ++i) {
		unsigned char c[8];
		if((st = rd(h, at + 24 + 16ull * i + 8, c, 8)))
			return st;
		uint64_t child = le(c, 8);
		st = level > 0 ? btree(h, child, e, depth + 1) : snod(h, child, e);
		if(st)
			return st;
	}
	return 0;
}

/* the members of the group whose object header is at oh */
static int
group_entries(gray_h5 *h, uint64_t oh, entries *e)
{
	msgref m[MAXMSG];
	int n, st;
	memset(e, 0, sizeof(*e));
	if((st = messages(h, oh, m, &n)))
		return st;
	for(int i = 0; i < n; ++i) {
		if(m[i].type != 0x0011 || m[i].size < 16)
			continue;
		unsigned char s[16], hp[32];
		if((st = rd(h, m[i].data, s, 16)))
			return st;
		uint64_t tree = le(s, 8), heap = le(s + 8, 8);
		if((st = rd(h, heap, hp, 32)))
			return st;
		if(memcmp(hp, "HEAP", 4) || hp[4] != 0)
			return GRAY_H5_EFORMAT;
		e->hsize = le(hp + 8, 8);
		if(e->hsize > h->size)
			return GRAY_H5_EFORMAT;
		e->heap = malloc(e->hsize + 1);
		if(!e->heap)
			return GRAY_H5_ENOMEM;
		if((st = rd(h, le(hp + 24, 8), e->heap, e->hsize))) {
			free_entries(e);
			return st;
		}
		e->heap[e->hsize] = 0;
		if((st = btree(h, tree, e, 0)))
			free_entries(e);
		return st;
	}
	return GRAY_H5_ENOTFOUND; /* not a group (no symbol table) */
}

/* object header address of a '/'-separated path below the root */
static int
resolve(gray_h5 *h, const char *path, uint64_t *oh)
{
	uint64_t at = h->root;
	const char *p = path;
	while(*p == '/')
		++p;
	while(*p) {
		const char *q = strchr(p, '/');
		size_t len = q ? (size_t)(q - p) : strlen(p);
		entries e;
		int st = group_entries(h, at, &e);
		if(st)
			return st;
		int found = 0;
		for(size_t i = 0; i < e.n && !found; ++i)
			if(strlen(e.v[i].name) == len && !memcmp(e.v[i].name, p, len)) {
				at = e.v[i].oh;
				found = 1;
			}
		free_entries(&e);
		if(!found)
			return GRAY_H5_ENOTFOUND;
		p += len;
		while(*p == '/')
			++p;
	}
	*oh = at;
	return 0;
}

int
gray_h5_member(gray_h5 *h, const char *group, uint64_t i, char *name, size_t name_len,
               uint64_t *n)
{
	if(!h || !group)
		return GRAY_H5_EINVAL;
	uint64_t oh;
	int st = resolve(h, group, &oh);
	if(st)
		return st;
	entries e;
	if((st = group_entries(h, oh, &e)))
		return st;
	if(n)
		*n = e.n;
	if(name) {
		if(i >= e.n)
			st = GRAY_H5_ENOTFOUND;
		else if(strlen(e.v[i].name) + 1 > name_len)
			st = GRAY_H5_ESIZE;
		else
			strcpy(name, e.v[i].name);
	}
	free_entries(&e);
	return st;
}

/* ---- datasets ------------------------------------------------------------ */

typedef struct {
	int      rank;
	uint64_t dims[8];
	uint64_t count;   /* elements                          */
	int      esize;   /* 4 or 8                            */
	int      big;     /* big-endian elements               */
	uint64_t addr;    /* raw data address (UNDEF: unwritten) */
	uint64_t bytes;   /* storage bytes                     */
} dset;

static int
dataset(gray_h5 *h, const char *path, dset *d)
{
	uint64_t oh;
	int st = resolve(h, path, &oh);
	if(st)
		return st;
	msgref m[MAXMSG];
	int n;
	if((st = messages(h, oh, m, &n)))
		return st;
	int have_space = 0, have_type = 0, have_layout = 0;
	memset(d, 0, sizeof(*d));
	d->addr = UNDEF;
	for(int i = 0; i < n; ++i) {
		unsigned char p[256];
		unsigned sz = m[i].size < sizeof(p) ? m[i].size : (unsigned)sizeof(p);
		if((st = rd(h, m[i].data, p, sz)))
			return st;
		switch(m[i].type) {
		case 0x0001: { /* dataspace, version 1 (dims at 8) or 2 (dims at 4) */
			if(sz < 4)
				return GRAY_H5_EFORMAT;
			int ver = p[0], rank = p[1];
			unsigned off = ver == 1 ? 8 : ver == 2 ? 4 : 0;
			if(!off || rank > 8 || off + 8u * rank > sz)
				return GRAY_H5_EFORMAT;
			d->rank = rank;
			d->count = 1;
			for(int k = 0; k < rank; ++k) {
				d->dims[k] = le(p + off + 8 * k, 8);
				if(d->dims[k] && d->count > UINT64_MAX / d->dims[k])
					return GRAY_H5_EFORMAT;
				d->count *= d->dims[k];
			}
			have_space = 1;
			break;
		}
		case 0x0003: { /* datatype: class 1 (IEEE float) only */
			if(sz < 8 || (p[0] & 0x0f) != 1)
				return GRAY_H5_EFORMAT;
			if(p[1] & 0x40)
				return GRAY_H5_EFORMAT; /* VAX byte order */
			d->big = p[1] & 1;
			d->esize = (int)le(p + 4, 4);
			if(d->esize != 4 && d->esize != 8)
				return GRAY_H5_EFORMAT;
			have_type = 1;
			break;
		}
		case 0x0008: { /* data layout */
			int ver = p[0];
			if(ver == 3) {
				if(p[1] == 1) { /* contiguous */
					d->addr = le(p + 2, 8);
					d->bytes = le(p + 10, 8);
				} else if(p[1] == 0) { /* compact: raw data in the message */
					d->bytes = le(p + 2, 2);
					d->addr = m[i].data + 4;
				} else {
					return GRAY_H5_EFORMAT; /* chunked */
				}
			} else if(ver == 1 || ver == 2) {
				int nd = p[1], cls = p[2];
				if(cls == 1) {
					d->addr = le(p + 8, 8);
					d->bytes = UNDEF; /* from the dataspace below */
				} else if(cls == 0) {
					unsigned off = 8 + 4u * nd;
					if(off + 4 > sz)
						return GRAY_H5_EFORMAT;
					d->bytes = le(p + off, 4);
					d->addr = m[i].data + off + 4;
				} else {
					return GRAY_H5_EFORMAT;
				}
			} else {
				return GRAY_H5_EFORMAT;
			}
			have_layout = 1;
			break;
		}
		case 0x000b: /* filter pipeline: compressed data */
			return GRAY_H5_EFORMAT;
		default:
			break;
		}
	}
	if(!have_space || !have_type || !have_layout)
		return GRAY_H5_ENOTFOUND; /* not a dataset */
	if(d->count > UINT64_MAX / (uint64_t)d->esize)
		return GRAY_H5_EFORMAT;
	if(d->bytes == UNDEF)
		d->bytes = d->count * (uint64_t)d->esize;
	if(d->addr != UNDEF && d->bytes < d->count * (uint64_t)d->esize)
		return GRAY_H5_EFORMAT;
	return 0;
}

int
gray_h5_dataset_info(gray_h5 *h, const char *path, int *rank, uint64_t dims[8], int *elem_size)
{
	if(!h || !path)
		return GRAY_H5_EINVAL;
	dset d;
	int st = dataset(h, path, &d);
	if(st)
		return st;
	if(rank)
		*rank = d.rank;
	if(dims)
		memcpy(dims, d.dims, sizeof(d.dims));
	if(elem_size)
		*elem_size = d.esize;
	return 0;
}

/* raw elements -> float or double, in chunks */
static int
read_dset(gray_h5 *h, const dset *d, int elem_size, void *out)
{
	if(d->addr == UNDEF) { /* never written: the fill value, 0 */
		memset(out, 0, (size_t)(d->count * (uint64_t)elem_size));
		return 0;
	}
	enum { CH = 1 << 16 };
	unsigned char *buf = malloc((size_t)CH * 8);
	if(!buf)
		return GRAY_H5_ENOMEM;
	int st = 0;
	for(uint64_t i = 0; i < d->count && !st; i += CH) {
		uint64_t k = d->count - i < CH ? d->count - i : CH;
		if((st = rd(h, d->addr + i * d->esize, buf, k * d->esize)))
			break;
		for(uint64_t j = 0; j < k; ++j) {
			unsigned char *e = buf + j * d->esize;
			if(d->big)
				for(int a = 0, b = d->esize - 1; a < b; ++a, --b) {
					unsigned char t = e[a];
					e[a] = e[b];
					e[b] = t;
				}
			double v;
			if(d->esize == 4) {
				float f;
				memcpy(&f, e, 4);
				v = f;
			} else {
				memcpy(&v, e, 8);
			}
			if(elem_size == 4)
				((float *)out)[i + j] = (float)v;
			else
				((double *)out)[i + j] = v;
		}
	}
	free(buf);
	return st;
}

int
gray_h5_read(gray_h5 *h, const char *path, int elem_size, void *out, uint64_t n_elems)
{
	if(!h || !path || !out || (elem_size != 4 && elem_size != 8))
		return GRAY_H5_EINVAL;
	dset d;
	int st = dataset(h, path, &d);
	if(st)
		return st;
	if(d.count != n_elems)
		return GRAY_H5_ESIZE;
	return read_dset(h, &d, elem_size, out);
}

/* ---- the spacetime file ------------------------------------------------- */

struct gray_h5_spacetime {
	gray_h5 *h;
	uint64_t n_times;
	double  *times;
	char   **names;   /* group name of each sorted time */
	int      n[3];
	float    lo[3], hi[3];
};

typedef struct {
	double t;
	char  *name;
} tname;

static int
by_time(const void *a, const void *b)
{
	double x = ((const tname *)a)->t, y = ((const tname *)b)->t;
	return x < y ? -1 : x > y;
}

/* tools/generate_data.py:49-58: x_i = sinh((A i + B)^3), B = cbrt(asinh(lo)),
 * A = (cbrt(asinh(hi)) - B) / (n - 1) */
static int
fisheye_ok(const float *x, int n)
{
	if(n < 2)
		return 0;
	const double lo = x[0], hi = x[n - 1];
	if(!(hi > lo))
		return 0;
	const double B = cbrt(asinh(lo)), A = (cbrt(asinh(hi)) - B) / (n - 1);
	for(int i = 0; i < n; ++i) {
		double want = sinh(pow(A * i + B, 3.0));
		double cell = i + 1 < n ? fabs(sinh(pow(A * (i + 1) + B, 3.0)) - want)
		                        : fabs(want - sinh(pow(A * (i - 1) + B, 3.0)));
		if(fabs((double)x[i] - want) > 1e-4 * cell + 1e-6 * fabs(want))
			return 0;
	}
	return 1;
}

void
gray_h5_spacetime_close(gray_h5_spacetime *s)
{
	if(!s)
		return;
	for(uint64_t i = 0; i < s->n_times; ++i)
		free(s->names ? s->names[i] : NULL);
	free(s->names);
	free(s->times);
	gray_h5_close(s->h);
	free(s);
}

int
gray_h5_spacetime_open(const char *path, gray_h5_spacetime **out)
{
	if(!path || !out)
		return GRAY_H5_EINVAL;
	*out = NULL;
	gray_h5_spacetime *s = calloc(1, sizeof(*s));
	if(!s)
		return GRAY_H5_ENOMEM;
	int st = gray_h5_open(path, &s->h);
	if(st) {
		free(s);
		return st;
	}
	entries e;
	if((st = group_entries(s->h, s->h->root, &e)))
		goto fail;
	/* io.c:199-213: every root member not starting with 'g' is a time */
	tname *tn = calloc(e.n ? e.n : 1, sizeof(*tn));
	if(!tn) {
		free_entries(&e);
		st = GRAY_H5_ENOMEM;
		goto fail;
	}
	uint64_t k = 0;
	for(size_t i = 0; i < e.n; ++i) {
		if(e.v[i].name[0] == 'g')
			continue;
		char *end;
		tn[k].t = strtod(e.v[i].name, &end);
		tn[k].name = e.v[i].name;
		e.v[i].name = NULL; /* moved */
		++k;
	}
	qsort(tn, k, sizeof(*tn), by_time);
	s->n_times = k;
	s->times = malloc((k ? k : 1) * sizeof(double));
	s->names = calloc(k ? k : 1, sizeof(char *));
	if(!s->times || !s->names)
		st = GRAY_H5_ENOMEM;
	for(uint64_t i = 0; i < k; ++i) {
		if(s->times)
			s->times[i] = tn[i].t;
		if(s->names)
			s->names[i] = tn[i].name;
		else
			free(tn[i].name);
	}
	free(tn);
	free_entries(&e);
	if(st)
		goto fail;
	if(k == 0) {
		st = GRAY_H5_ENOTFOUND;
		goto fail;
	}
	/* io.c:229-275: the grid coordinates and the box */
	static const char *const axis[3] = {"grid/x", "grid/y", "grid/z"};
	for(int a = 0; a < 3; ++a) {
		int rank, es;
		uint64_t dims[8];
		if((st = gray_h5_dataset_info(s->h, axis[a], &rank, dims, &es)))
			goto fail;
		if(rank != 1 || dims[0] < 2 || dims[0] > (1u << 20)) {
			st = GRAY_H5_ESIZE;
			goto fail;
		}
		float *x = malloc(dims[0] * sizeof(float));
		if(!x) {
			st = GRAY_H5_ENOMEM;
			goto fail;
		}
		st = gray_h5_read(s->h, axis[a], 4, x, dims[0]);
		if(!st && !fisheye_ok(x, (int)dims[0]))
			st = GRAY_H5_EFORMAT;
		s->n[a] = (int)dims[0];
		s->lo[a] = x[0];
		s->hi[a] = x[dims[0] - 1];
		free(x);
		if(st)
			goto fail;
	}
	*out = s;
	return 0;
fail:
	gray_h5_spacetime_close(s);
	return st;
}

uint64_t
gray_h5_spacetime_times(const gray_h5_spacetime *s, const double **times)
{
	if(!s)
		return 0;
	if(times)
		*times = s->times;
	return s->n_times;
}

void
gray_h5_spacetime_grid(const gray_h5_spacetime *s, int n[3], float lo[3], float hi[3])
{
	for(int a = 0; a < 3 && s; ++a) {
		if(n)
			n[a] = s->n[a];
		if(lo)
			lo[a] = s->lo[a];
		if(hi)
			hi[a] = s->hi[a];
	}
}

/* the 51 dataset names in io.c order (io.c:356-428) */
static void
field_name(int c, char *buf, size_t len)
{
	static const char D[4] = {'t', 'x', 'y', 'z'};
	if(c < 40) {
		int idx = c;
		for(int i = 0; i < 4; ++i)
			for(int j = 0; j < 4; ++j)
				for(int k = j; k < 4; ++k)
					if(idx-- == 0) {
						snprintf(buf, len, "Gamma_%c%c%c", D[i], D[j], D[k]);
						return;
					}
	} else if(c < 50) {
		int idx = c - 40;
		for(int j = 0; j < 4; ++j)
			for(int k = j; k < 4; ++k)
				if(idx-- == 0) {
					snprintf(buf, len, "g_%c%c", D[j], D[k]);
					return;
				}
	}
	snprintf(buf, len, "rho");
}

int
gray_h5_spacetime_load(gray_h5_spacetime *s, uint64_t k, float *fields)
{
	if(!s || !fields || k >= s->n_times)
		return GRAY_H5_EINVAL;
	const uint64_t np = (uint64_t)s->n[0] * s->n[1] * s->n[2];
	float *tmp = malloc(np * sizeof(float));
	if(!tmp)
		return GRAY_H5_ENOMEM;
	int st = 0;
	for(int c = 0; c < NFIELD && !st; ++c) {
		char nm[32], path[320];
		field_name(c, nm, sizeof(nm));
		snprintf(path, sizeof(path), "%s/%s", s->names[k], nm);
		int rank, es;
		uint64_t dims[8];
		if((st = gray_h5_dataset_info(s->h, path, &rank, dims, &es)))
			break;
		/* [nz][ny][nx]; the reference checks only the element count */
		if(rank == 3 && (dims[0] != (uint64_t)s->n[2] || dims[1] != (uint64_t)s->n[1] ||
		                 dims[2] != (uint64_t)s->n[0])) {
			st = GRAY_H5_ESIZE;
			break;
		}
		if((st = gray_h5_read(s->h, path, 4, tmp, np)))
			break;
		for(uint64_t p = 0; p < np; ++p)
			fields[p * NFIELD + c] = tmp[p];
	}
	free(tmp);
	return st;
}

int
gray_h5_spacetime_loader(void *user, uint64_t k, float *fields)
{
	return gray_h5_spacetime_load((gray_h5_spacetime *)user, k, fields);
}

/* ======================================================================= */
/* writing                                                                 */
/* ======================================================================= */

enum { LEAF_K = 4, NODE_K = 16 }; /* libhdf5's defaults */

typedef struct {
	FILE *f;
	int   err;
} W;

static uint64_t
wtell(W *w)
{
	off_t o = ftello(w->f);
	if(o < 0)
		w->err = 1;
	return o < 0 ? 0 : (uint64_t)o;
}

static void
wput(W *w, const void *p, size_t n)
{
	if(!w->err && n && fwrite(p, 1, n, w->f) != n)
		w->err = 1;
}

static void
wzero(W *w, size_t n)
{
	static const unsigned char z[64];
	while(n) {
		size_t k = n < sizeof(z) ? n : sizeof(z);
		wput(w, z, k);
		n -= k;
	}
}

static void
pad8(W *w)
{
	uint64_t at = wtell(w);
	if(at % 8)
		wzero(w, (size_t)(8 - at % 8));
}

/* one message of a version-1 object header: type, size (padded to 8),
 * flags, reserved, body */
static size_t
msg(unsigned char *p, unsigned type, unsigned flags, const unsigned char *body, size_t len)
{
	size_t padded = (len + 7) & ~(size_t)7;
	memset(p, 0, 8 + padded);
	put(p, type, 2);
	put(p + 2, padded, 2);
	p[4] = (unsigned char)flags;
	memcpy(p + 8, body, len);
	return 8 + padded;
}

static void
ohdr(W *w, unsigned nmsgs, const unsigned char *msgs, size_t len)
{
	unsigned char p[16] = {0};
	p[0] = 1; /* version */
	put(p + 2, nmsgs, 2);
	put(p + 4, 1, 4); /* reference count */
	put(p + 8, len, 4);
	wput(w, p, 16);
	wput(w, msgs, len);
}

/* a float dataset (object header, then its contiguous data); returns the
 * object header address */
static uint64_t
w_dataset(W *w, int rank, const uint64_t *dims, int esize, const void *data)
{
	unsigned char body[128], msgs[512];
	size_t n = 0;
	uint64_t count = 1;
	pad8(w);
	const uint64_t oh = wtell(w);
	/* dataspace, version 1 */
	memset(body, 0, sizeof(body));
	body[0] = 1;
	body[1] = (unsigned char)rank;
	for(int k = 0; k < rank; ++k) {
		put(body + 8 + 8 * k, dims[k], 8);
		count *= dims[k];
	}
	n += msg(msgs + n, 0x0001, 0, body, 8 + 8 * (size_t)rank);
	/* datatype, version 1, class 1: little-endian IEEE float */
	memset(body, 0, sizeof(body));
	body[0] = 0x11;
	body[1] = 0x20;                           /* mantissa msb implied */
	body[2] = esize == 4 ? 31 : 63;           /* sign bit */
	put(body + 4, (uint64_t)esize, 4);
	put(body + 8, 0, 2);                      /* bit offset */
	put(body + 10, (uint64_t)esize * 8, 2);   /* precision */
	body[12] = esize == 4 ? 23 : 52;          /* exponent location */
	body[13] = esize == 4 ? 8 : 11;           /* exponent size */
	body[14] = 0;                             /* mantissa location */
	body[15] = esize == 4 ? 23 : 52;          /* mantissa size */
	put(body + 16, esize == 4 ? 127 : 1023, 4);
	n += msg(msgs + n, 0x0003, 1, body, 20);
	/* fill value, version 2: late allocation, fill if set, none defined */
	memset(body, 0, sizeof(body));
	body[0] = 2;
	body[1] = 2;
	body[2] = 2;
	body[3] = 0;
	n += msg(msgs + n, 0x0005, 1, body, 4);
	/* layout, version 3, contiguous: the data right after this header */
	const uint64_t bytes = count * (uint64_t)esize;
	const uint64_t at = oh + 16 + n + 8 + 24;
	memset(body, 0, sizeof(body));
	body[0] = 3;
	body[1] = 1;
	put(body + 2, at, 8);
	put(body + 10, bytes, 8);
	n += msg(msgs + n, 0x0008, 0, body, 18);
	ohdr(w, 4, msgs, n);
	if(wtell(w) != at)
		w->err = 1;
	wput(w, data, (size_t)bytes);
	return oh;
}

typedef struct {
	const char *name;
	uint64_t    oh;
	int         group;      /* cache the group's B-tree and heap */
	uint64_t    tree, heap;
} child;

static int
by_name(const void *a, const void *b)
{
	return strcmp(((const child *)a)->name, ((const child *)b)->name);
}

/* a group: local heap of names, symbol-table nodes of up to 2 LEAF_K
 * entries, one level-0 B-tree node over them, and the object header with
 * the symbol-table message.  Returns the header address; *tree and *heap
 * receive the addresses a parent caches in its entry. */
static uint64_t
w_group(W *w, child *c, size_t n, uint64_t *tree, uint64_t *heap)
{
	const size_t per = 2 * LEAF_K;
	const size_t nnodes = (n + per - 1) / per;
	if(nnodes > 2 * NODE_K) { /* one B-tree node: up to 256 members */
		w->err = 1;
		return 0;
	}
	qsort(c, n, sizeof(*c), by_name);
	uint64_t *off = malloc((n ? n : 1) * sizeof(uint64_t));
	if(!off) {
		w->err = 1;
		return 0;
	}
	uint64_t seg = 8; /* offset 0: the empty name */
	for(size_t i = 0; i < n; ++i) {
		off[i] = seg;
		seg += (strlen(c[i].name) + 1 + 7) & ~(uint64_t)7;
	}
	/* local heap */
	pad8(w);
	*heap = wtell(w);
	unsigned char hp[32] = {'H', 'E', 'A', 'P', 0};
	put(hp + 8, seg, 8);
	put(hp + 16, 1, 8); /* no free block: libhdf5's on-disk sentinel (1) */
	put(hp + 24, *heap + 32, 8);
	wput(w, hp, 32);
	wzero(w, 8);
	for(size_t i = 0; i < n; ++i) {
		size_t len = strlen(c[i].name) + 1;
		wput(w, c[i].name, len);
		wzero(w, (size_t)(((len + 7) & ~(size_t)7) - len));
	}
	/* symbol-table nodes */
	uint64_t nodes[2 * NODE_K];
	for(size_t b = 0; b < nnodes; ++b) {
		pad8(w);
		nodes[b] = wtell(w);
		size_t k0 = b * per, k1 = k0 + per < n ? k0 + per : n;
		unsigned char p[8] = {'S', 'N', 'O', 'D', 1, 0};
		put(p + 6, k1 - k0, 2);
		wput(w, p, 8);
		for(size_t i = k0; i < k1; ++i) {
			unsigned char e[40] = {0};
			put(e, off[i], 8);
			put(e + 8, c[i].oh, 8);
			if(c[i].group) {
				put(e + 16, 1, 4); /* cache type 1: B-tree and heap */
				put(e + 24, c[i].tree, 8);
				put(e + 32, c[i].heap, 8);
			}
			wput(w, e, 40);
		}
		wzero(w, 40 * (per - (k1 - k0)));
	}
	/* B-tree, level 0: key0 child0 key1 ... ; key i+1 is the last name of
	 * child i */
	pad8(w);
	*tree = wtell(w);
	unsigned char t[24] = {'T', 'R', 'E', 'E', 0, 0};
	put(t + 6, nnodes, 2);
	put(t + 8, UNDEF, 8);
	put(t + 16, UNDEF, 8);
	wput(w, t, 24);
	unsigned char kv[8];
	put(kv, 0, 8);
	wput(w, kv, 8);
	for(size_t b = 0; b < nnodes; ++b) {
		size_t last = (b + 1) * per < n ? (b + 1) * per - 1 : n - 1;
		put(kv, nodes[b], 8);
		wput(w, kv, 8);
		put(kv, off[last], 8);
		wput(w, kv, 8);
	}
	wzero(w, 16 * (2 * NODE_K - nnodes));
	free(off);
	/* object header: the symbol-table message */
	pad8(w);
	uint64_t oh = wtell(w);
	unsigned char body[16], m[32];
	put(body, *tree, 8);
	put(body + 8, *heap, 8);
	size_t len = msg(m, 0x0011, 0, body, 16);
	ohdr(w, 1, m, len);
	return oh;
}

/* the version-0 superblock at offset 0 with the root group's entry */
static void
w_superblock(W *w, uint64_t root_oh, uint64_t tree, uint64_t heap, uint64_t eof)
{
	unsigned char p[96] = {0};
	memcpy(p, SIG, 8);
	/* versions: superblock, free space, root entry, reserved, shared header */
	p[13] = 8;                  /* size of offsets */
	p[14] = 8;                  /* size of lengths */
	put(p + 16, LEAF_K, 2);
	put(p + 18, NODE_K, 2);
	put(p + 24, 0, 8);          /* base address */
	put(p + 32, UNDEF, 8);      /* free-space info */
	put(p + 40, eof, 8);        /* end of file */
	put(p + 48, UNDEF, 8);      /* driver info */
	put(p + 56, 0, 8);          /* root entry: name offset */
	put(p + 64, root_oh, 8);
	put(p + 72, 1, 4);          /* cache type 1 */
	put(p + 80, tree, 8);
	put(p + 88, heap, 8);
	if(fseeko(w->f, 0, SEEK_SET))
		w->err = 1;
	wput(w, p, 96);
}

static int
finish(W *w, const char *path)
{
	int bad = w->err;
	if(fclose(w->f))
		bad = 1;
	if(bad) {
		remove(path);
		return GRAY_H5_EIO;
	}
	return 0;
}

int
gray_h5_write_spacetime(const char *path, int nx, int ny, int nz, const float *x,
                        const float *y, const float *z, uint64_t n_times,
                        const char *const *time_names, const float *const *levels)
{
	if(!path || nx < 2 || ny < 2 || nz < 2 || !x || !y || !z || !n_times || !time_names ||
	   !levels || n_times + 1 > 2 * LEAF_K * 2 * NODE_K)
		return GRAY_H5_EINVAL;
	for(uint64_t k = 0; k < n_times; ++k)
		if(!time_names[k] || !time_names[k][0] || time_names[k][0] == 'g' ||
		   strchr(time_names[k], '/') || !levels[k])
			return GRAY_H5_EINVAL;
	const uint64_t np = (uint64_t)nx * ny * nz;
	float *tmp = malloc(np * sizeof(float));
	child *top = calloc(n_times + 1, sizeof(child));
	if(!tmp || !top) {
		free(tmp);
		free(top);
		return GRAY_H5_ENOMEM;
	}
	W w = {fopen(path, "wb"), 0};
	if(!w.f) {
		free(tmp);
		free(top);
		return GRAY_H5_EIO;
	}
	wzero(&w, 96); /* the superblock, written last */
	/* grid/{x,y,z} */
	child g[3] = {{"x", 0, 0, 0, 0}, {"y", 0, 0, 0, 0}, {"z", 0, 0, 0, 0}};
	const float *ax[3] = {x, y, z};
	const uint64_t na[3] = {(uint64_t)nx, (uint64_t)ny, (uint64_t)nz};
	for(int a = 0; a < 3; ++a)
		g[a].oh = w_dataset(&w, 1, &na[a], 4, ax[a]);
	top[0].name = "grid";
	top[0].group = 1;
	top[0].oh = w_group(&w, g, 3, &top[0].tree, &top[0].heap);
	/* one group per snapshot with its 51 datasets */
	char names[NFIELD][16];
	child f[NFIELD];
	for(uint64_t k = 0; k < n_times && !w.err; ++k) {
		const uint64_t dims[3] = {(uint64_t)nz, (uint64_t)ny, (uint64_t)nx};
		for(int c = 0; c < NFIELD; ++c) {
			for(uint64_t p = 0; p < np; ++p)
				tmp[p] = levels[k][p * NFIELD + c];
			field_name(c, names[c], sizeof(names[c]));
			f[c].name = names[c];
			f[c].group = 0;
			f[c].oh = w_dataset(&w, 3, dims, 4, tmp);
		}
		top[k + 1].name = time_names[k];
		top[k + 1].group = 1;
		top[k + 1].oh = w_group(&w, f, NFIELD, &top[k + 1].tree, &top[k + 1].heap);
	}
	uint64_t tree, heap;
	uint64_t root = w_group(&w, top, n_times + 1, &tree, &heap);
	pad8(&w);
	uint64_t eof = wtell(&w);
	w_superblock(&w, root, tree, heap, eof);
	free(tmp);
	free(top);
	return finish(&w, path);
}

int
gray_h5_write_rays(const char *path, const void *data, int elem_size, uint64_t w_rays,
                   uint64_t h_rays, uint64_t n_data)
{
	if(!path || !data || (elem_size != 4 && elem_size != 8) || !w_rays || !h_rays || !n_data)
		return GRAY_H5_EINVAL;
	/* H5F_ACC_EXCL (sim/gray.c:175): never overwrite */
	W w = {fopen(path, "wbx"), 0};
	if(!w.f)
		return errno == EEXIST ? GRAY_H5_EEXIST : GRAY_H5_EIO;
	wzero(&w, 96);
	const uint64_t dims[3] = {w_rays, h_rays, n_data};
	child c = {"rays", 0, 0, 0, 0};
	c.oh = w_dataset(&w, 3, dims, elem_size, data);
	uint64_t tree, heap;
	uint64_t root = w_group(&w, &c, 1, &tree, &heap);
	pad8(&w);
	uint64_t eof = wtell(&w);
	w_superblock(&w, root, tree, heap, eof);
	return finish(&w, path);
}
