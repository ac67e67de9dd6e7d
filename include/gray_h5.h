/*
 * gray_h5 -- GRay2's HDF5 files without libhdf5.
 *
 * The reference reads its numerical spacetimes from HDF5 (sim-org/io.c:
 * 149-533, layout in README.md:40-60, written by tools/generate_data.py:
 * 132-160) and the new lux tree writes each dump's rays to an HDF5 file as
 * the dataset /rays (sim/gray.c:170-176, rayfile "ray%04d.h5",
 * sim/gray.opts:14).  No HDF5 library is available to this build, so this
 * is a self-contained reader and writer of the classic HDF5 file format
 * that libhdf5 writes by default (h5py's libver "earliest"):
 *
 *  - superblock version 0 or 1 with 8-byte offsets and lengths;
 *  - version-1 object headers (with continuation blocks);
 *  - groups as symbol tables (version-1 B-tree of symbol-table nodes and a
 *    local heap of names);
 *  - datasets of little- or big-endian IEEE float32 / float64 with
 *    contiguous or compact storage (dataspace v1/v2, datatype class 1,
 *    layout message v1-v3).
 *
 * Newer-format files (superblock v2/v3, "OHDR" headers, link messages),
 * chunked or filtered (compressed) datasets and other datatypes are refused
 * with GRAY_H5_EFORMAT rather than misread; the reference leaves compressed
 * files as a TODO as well (io.c:305-306).
 *
 * Status codes are 0 or the negative values below; nothing aborts.
 */
#ifndef GRAY_H5_H
#define GRAY_H5_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRAY_H5_OK        0
#define GRAY_H5_EINVAL   (-1)   /* bad argument                                  */
#define GRAY_H5_ENOMEM   (-2)   /* host allocation failed                        */
#define GRAY_H5_ENOTFOUND (-7)  /* no such file, group or dataset                 */
#define GRAY_H5_ESIZE    (-9)   /* dataset shape or buffer size mismatch         */
#define GRAY_H5_EFORMAT  (-20)  /* not HDF5, corrupt, or an unsupported feature   */
#define GRAY_H5_EIO      (-21)  /* read or write failed                          */
#define GRAY_H5_EEXIST   (-22)  /* file exists (exclusive create)                */

const char *gray_h5_strerror(int status);

/* ---- generic reading ------------------------------------------------- */

typedef struct gray_h5 gray_h5;

int  gray_h5_open(const char *path, gray_h5 **out);
void gray_h5_close(gray_h5 *h);

/* Member i of a group ("/" or a path such as "grid"), in stored (name)
 * order; *n receives the number of members.  name may be NULL to ask only
 * for the count. */
int gray_h5_member(gray_h5 *h, const char *group, uint64_t i, char *name, size_t name_len,
                   uint64_t *n);

/* Shape and element size (4 or 8) of a float dataset ("grid/x", "rays"). */
int gray_h5_dataset_info(gray_h5 *h, const char *path, int *rank, uint64_t dims[8],
                         int *elem_size);

/* The whole dataset converted to elem_size (4 = float, 8 = double);
 * n_elems must equal the dataset's element count (GRAY_H5_ESIZE). */
int gray_h5_read(gray_h5 *h, const char *path, int elem_size, void *out, uint64_t n_elems);

/* ---- the spacetime file of sim-org/io.c ------------------------------- */

typedef struct gray_h5_spacetime gray_h5_spacetime;

/* io.c:149-275: the snapshot times are the root groups whose names do not
 * start with 'g', parsed with strtod and sorted ascending (io.c:191-213);
 * the grid is grid/{x,y,z} (1-D, float32 in the reference's files, float64
 * accepted) and its box is their first and last values (io.c:264-273).
 * The coordinates must follow the n = 3 fisheye map between those ends
 * (tools/generate_data.py:49-58) within 1e-4 of the cell size, because the
 * interpolation assumes it (interp.cl:89-96): other spacings would be
 * misread silently, so they are refused with GRAY_H5_EFORMAT.  At least one
 * snapshot is required. */
int gray_h5_spacetime_open(const char *path, gray_h5_spacetime **out);
void gray_h5_spacetime_close(gray_h5_spacetime *s);
/* number of snapshots; *times (nullable) receives the sorted times */
uint64_t gray_h5_spacetime_times(const gray_h5_spacetime *s, const double **times);
/* grid points per axis (x, y, z) and the box (lo, hi per axis) */
void gray_h5_spacetime_grid(const gray_h5_spacetime *s, int n[3], float lo[3], float hi[3]);
/* io.c:302-533 load_snapshot: snapshot k's 51 datasets -- Gamma_{ijk}
 * (i in t,x,y,z; j <= k), g_{ij} (i <= j), rho -- each [nz][ny][nx],
 * interleaved into fields[((z ny + y) nx + x) 51 + c] (the layout
 * gray_load_spacetime_interleaved and gray_snapshot_source.load take). */
int gray_h5_spacetime_load(gray_h5_spacetime *s, uint64_t k, float *fields);
/* gray_snapshot_source.load for gray_run_series: user is the spacetime */
int gray_h5_spacetime_loader(void *user, uint64_t k, float *fields);

/* ---- writing ----------------------------------------------------------- */

/* A spacetime file in the layout above (what tools/generate_data.py:132-160
 * writes): grid/{x,y,z} float32 and, per snapshot, a group named
 * time_names[k] holding the 51 float32 datasets [nz][ny][nx] taken from
 * levels[k] (interleaved as gray_h5_spacetime_load returns them).
 * Overwrites path. */
int gray_h5_write_spacetime(const char *path, int nx, int ny, int nz, const float *x,
                            const float *y, const float *z, uint64_t n_times,
                            const char *const *time_names, const float *const *levels);

/* sim/gray.c:170-176: a new file (exclusive create, GRAY_H5_EEXIST if it
 * exists) holding the dataset /rays of shape {w, h, n_data} -- the
 * reference's host array palloc(real, n_width, n_height, 8) -- with elements
 * of elem_size bytes (4 float, 8 double: the job's precision), in ray order
 * (ray = column + row * w, the state of each ray contiguous). */
int gray_h5_write_rays(const char *path, const void *data, int elem_size, uint64_t w,
                       uint64_t h, uint64_t n_data);

#ifdef __cplusplus
}
#endif

#endif /* GRAY_H5_H */
