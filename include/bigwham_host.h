/* bigwham_host -- C ABI of BigWhamIO with the B200 backend installed.
 *
 * libbigwham_host.so contains the reference's own, unmodified host code
 * (mesh, elastic kernels, cluster tree, admissibility, ACA; compiled from its
 * sources) plus the HmatGpu adapter (bigwham_dev_b200/host/hmat_gpu.h).  These
 * entry points mirror the methods the reference's pybind11 module exposes on
 * BigWhamIOSelf (interfaces/python/py_bigwham.cc:141-260) for the matvec path,
 * so a ctypes / cgo / JNI caller can drive the whole flow without C++.
 *
 * All functions return 0 on success; on failure a non-zero status and the
 * message from bwh_last_error().
 */
#ifndef BIGWHAM_HOST_H
#define BIGWHAM_HOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bwh_io bwh_io;
struct bw_hmat;

/* BigWhamIO(coor, conn, kernel, properties, n_openMP_threads, n_GPUs, verbose,
 * homogeneous_size_pattern, useCuda = false, fixed_rank)
 * (src/io/bigwham_io.h:73-82; py_bigwham.cc:144). */
int bwh_create(const double *coor, int64_t n_coor, const int *conn, int64_t n_conn, const char *kernel,
               const double *properties, int n_properties, int n_openmp_threads, int verbose, int fixed_rank,
               bwh_io **out);

/* The rectangular BigWhamIO (src/io/bigwham_io.h:85-96; pybind11
 * BigWhamIORect): a source mesh and a different receiver mesh, kernels such
 * as "3DR0-3DR0-H"; the H-matrix has receiver rows and source columns. */
int bwh_create_rect(const double *coor_src, int64_t n_coor_src, const int *conn_src, int64_t n_conn_src,
                    const double *coor_rec, int64_t n_coor_rec, const int *conn_rec, int64_t n_conn_rec,
                    const char *kernel, const double *properties, int n_properties, int n_openmp_threads,
                    int verbose, int fixed_rank, bwh_io **out);

/* BigWhamIO::BuildHierarchicalMatrix (bigwham_io.cc:635-704), host build. */
int bwh_build(bwh_io *io, int max_leaf_size, double eta, double eps_aca);
/* BigWhamIO::BuildPattern (src/io/bigwham_io.cc:487-511): cluster tree and
 * block pattern only, no blocks; bwh_hpattern and bwh_permutation then
 * describe the pattern, for a build of the blocks on the device. */
int bwh_build_pattern(bwh_io *io, int max_leaf_size, double eta);

/* Upload the built H-matrix to `device` in the precisions of `storage`
 * (BW_FP64 | BW_FP32 | BW_BF16 [| BW_STORE_TRANSPOSE]) and install it with
 * BigWhamIO::setHmat (bigwham_io.h:206).  After this call every matvec below
 * runs on the GPU.  release_host: drop the reference's host copy of the
 * low-rank factors (the GPU keeps its own). */
int bwh_attach_gpu(bwh_io *io, int device, int storage, int release_host);

/* Precision of the reference-facing matvec calls (one of BW_FP64, BW_FP32, BW_BF16). */
int bwh_set_precision(bwh_io *io, int precision);

/* Plan parameter for the next bwh_attach_gpu (passed to bw_set_tuning; an
 * unknown key or a bad value makes bwh_attach_gpu fail). */
int bwh_set_tuning(bwh_io *io, const char *key, int64_t value);

/* BigWhamIO::MatVec(il::ArrayView) -- host arrays, original ordering.  The
 * product is written straight into y (n_rows values); the reference returns a
 * new il::Array that its bindings copy into the caller's array. */
int bwh_matvec(bwh_io *io, const double *x, double *y);
/* BigWhamIO::MatVecPerm -- host arrays, permuted ordering, written into y. */
int bwh_matvec_perm(bwh_io *io, const double *x, double *y);
/* BigWhamIO::MatVec(double*, double*) -- device pointers (matvec_raw_ptr). */
int bwh_matvec_raw_ptr(bwh_io *io, double *x, double *y);
/* BigWhamIO::GetDiagonal (original ordering). */
int bwh_diagonal(bwh_io *io, double *d);

int64_t bwh_size(const bwh_io *io, int k);
int bwh_dof(const bwh_io *io);
double bwh_compression(const bwh_io *io);
double bwh_hmat_time(const bwh_io *io);
/* GetPermutation (bigwham_io.cc): n_points int64 values. */
int bwh_permutation(const bwh_io *io, int64_t *perm);
/* GetCollocationPoints: returns the count; fills `out` when non-null. */
int64_t bwh_collocation_points(const bwh_io *io, double *out);
/* Per element of a 3D mesh with one collocation point per element, 15
 * doubles: collocation point, rotation matrix row-major (local = R global)
 * and unit normal, from the reference's element objects
 * (GetCollocationPoints / GetRotationMatrix / GetElementNormals,
 * src/io/bigwham_io.cc:985-1140).  Returns the element count; fills `out`
 * when non-null; -1 for other meshes. */
int64_t bwh_element_frames(const bwh_io *io, double *out);
/* GetHPattern: 6 doubles per block; returns the count; fills `out` when non-null. */
int64_t bwh_hpattern(const bwh_io *io, double *out);
/* Block counts of the pattern: kind 0 full rank, 1 low rank. */
int64_t bwh_n_blocks(const bwh_io *io, int kind);

/* Stored entries of the FR blocks (kind 0) or of the LR factors A and B (kind 1). */
int64_t bwh_entries(const bwh_io *io, int kind);
/* Copy the built H-matrix out (before bwh_attach_gpu, or after it when the
 * host blocks were kept, release_host = 0): fr (n_FR x 4: i0, j0,
 * iend, jend in points), lr (n_LR x 5: ..., r), the FR blocks back to back and
 * per LR block A then B (column-major), and both permutations.  This is the
 * flat form bw_add_* accept and the form of the benchmark's block cache. */
int bwh_export(const bwh_io *io, int64_t *fr, int64_t *lr, double *fr_data, double *lr_data, int64_t *perm0,
               int64_t *perm1);

/* Save the built H-matrix as a block file (bw_file_write_blocks of
 * include/bigwham_b200.h: pattern with its HPattern spots, permutations, every
 * block and the ACA error estimates), before bwh_attach_gpu or after one with
 * release_host = 0.  The content of
 * the reference's Hmat::writeToFile (src/hmat/hmatrix/hmat.cc:749-835), which
 * needs HDF5.  Load it with bw_create_from_file / HmatGpu.from_file. */
int bwh_write_to_file(const bwh_io *io, const char *path);

/* Pass-throughs to the reference's BigWhamIO, as the pybind11 module
 * exposes them (interfaces/python/py_bigwham.cc:141-260).  Array results:
 * the function returns the element count and fills `out` when it is
 * non-null (two calls: size, then data).  -1 on error (bwh_last_error). */
/* ConvertToLocal (to_global = 0) / ConvertToGlobal (1): n values, out n values. */
int bwh_convert(const bwh_io *io, int to_global, const double *in, int64_t n, double *out);
/* GetElementNormals / GetRotationMatrix (flattened per element). */
int64_t bwh_element_normals(const bwh_io *io, double *out);
int64_t bwh_rotation_matrix(const bwh_io *io, double *out);
/* GetMaxErrorACA (largest ACA error estimate over the low-rank blocks). */
double bwh_max_error_aca(const bwh_io *io);
/* GetFullBlocks (original_order != 0) / GetFullBlocksPerm: the full-rank
 * blocks' entries with their row and column; returns the entry count. */
int64_t bwh_full_blocks(const bwh_io *io, int original_order, double *val, int32_t *row, int32_t *col);
/* ComputeDisplacements (kind 0) / ComputeStresses (kind 1) at the points
 * coor_obs (n_coor values, spatial dimension per point) for the solution sol
 * (n_sol values, local element frames, original ordering): out_len values
 * (points x dof, or points x 3 / 6 stress components in 2D / 3D); returns the
 * value count.  The reference's own host code. */
int64_t bwh_compute_fields(const bwh_io *io, int kind, const double *coor_obs, int64_t n_coor, const double *sol,
                           int64_t n_sol, double *out, int64_t out_len);
/* GetStorageRequirement in bytes (entries x 8) and GetOmpThreads. */
int64_t bwh_storage_requirement(const bwh_io *io);
int bwh_omp_threads(const bwh_io *io);
/* Spatial dimension of the mesh (2 or 3). */
int bwh_spatial_dimension(const bwh_io *io);

/* The device H-matrix after bwh_attach_gpu (owned by io), for the
 * extensions of include/bigwham_b200.h (precision choice, H^T, matmat). */
struct bw_hmat *bwh_gpu_handle(bwh_io *io);

int bwh_destroy(bwh_io *io);
const char *bwh_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* BIGWHAM_HOST_H */
