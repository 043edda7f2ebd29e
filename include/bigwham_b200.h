/* bigwham_b200 -- B200 (sm_100a) H-matrix x vector backend, C ABI.
 *
 * Drop-in boundary for BigWham's H-matrix matvec.  The reference keeps
 * building the H-matrix on the host (mesh, kernel, cluster tree,
 * admissibility, ACA); its full-rank blocks and low-rank blocks are handed to
 * this library once, which re-lays them out in device memory and applies the
 * operator with hand-written CUDA kernels.
 *
 * Units: rows/columns are SCALAR indices (collocation point * dof + component),
 * i.e. the reference's HPattern entries multiplied by the dof dimension
 * (src/hmat/hmatrix/h_pattern.h:21-33).  Blocks are column-major with a
 * leading dimension, as il::Array2D stores them (il/il/container/2d/Array2D.h:840).
 *
 * Every entry point returns an int status (BW_OK == 0) and never exits the
 * process; bw_last_error() gives the message.  Calls on one handle must be
 * ordered on one CUDA stream (they share the handle's scratch vectors).
 */
#ifndef BIGWHAM_B200_H
#define BIGWHAM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bw_hmat bw_hmat;

/* status codes */
enum {
  BW_OK = 0,
  BW_ERR_ARG = 1,         /* bad argument, malformed pattern, non-finite block entry */
  BW_ERR_STATE = 2,       /* call not valid in the handle's state (e.g. matvec before finalize) */
  BW_ERR_OOM = 3,         /* device or host allocation failed, or above the configured limit */
  BW_ERR_CUDA = 4,        /* a CUDA runtime call failed */
  BW_ERR_DEVICE = 5,      /* a kernel reported an error word (e.g. a bounded wait ran out) */
  BW_ERR_UNSUPPORTED = 6, /* precision or operation not stored / not available */
  BW_ERR_IO = 7           /* a block file could not be read or written, or failed its checks */
};

/* storage / precision flags */
enum {
  BW_FP64 = 1,            /* FP64 blocks, FP64 accumulation */
  BW_FP32 = 2,            /* FP32 blocks, FP32 accumulation */
  BW_BF16 = 4,            /* BF16 blocks with a per-block FP32 scale, FP32 accumulation */
  BW_STORE_TRANSPOSE = 16,/* bw_finalize: also lay out H^T for bw_matvec(..., BW_TRANSPOSE) */
  BW_NO_FINITE_CHECK = 32,/* bw_finalize: skip the non-finite entry check */
  BW_PLAN_ONLY = 64,      /* bw_finalize: build the host plan only (no device); for inspection */
  BW_STORE_MATMAT = 128   /* bw_finalize: also store the BF16 matmat layout, so bw_matmat(..., BW_BF16)
                             runs on the tcgen05 tensor cores (64 right-hand sides per pass) */
};

/* matvec flags (OR with exactly one of BW_FP64 / BW_FP32 / BW_BF16) */
enum {
  BW_PERMUTED = 256,      /* x and y are in the clustered (permuted) ordering:
                             Hmat::matvec instead of Hmat::matvecOriginal */
  BW_TRANSPOSE = 512      /* apply H^T instead of H */
};

/* Create an empty handle.
 * dof: dofs per collocation point; n_rows, n_cols: scalar sizes (Hmat::size(0/1),
 * src/hmat/hmatrix/hmat.h:80); perm0 (n_rows/dof) and perm1 (n_cols/dof): the
 * row / column permutations (HRepresentation::permutation_0_/_1_,
 * src/hmat/hierarchical_representation.h:28-29), copied.
 * device: CUDA device ordinal, or -1 for a host-only plan (BW_PLAN_ONLY).
 * Replaces: the HmatCuda constructor's upload set-up
 * (src/hmat/hmatrix/hmat_cuda.cc:98-329). */
int bw_create(int dof, int64_t n_rows, int64_t n_cols, const int64_t *perm0, const int64_t *perm1, int device,
              bw_hmat **out);

/* Create one handle for `count` independent H-matrices with the same dof
 * ("members"); one bw_matvec then applies all of them in the same four
 * launches.  The handle is the block-diagonal H-matrix diag(H_0, ..., H_{count-1}):
 * member k's rows and columns start at the sums of the earlier members'
 * n_rows / n_cols (bw_batch_offsets), its blocks are added with bw_add_full /
 * bw_add_lowrank at those offsets, and x / y are the members' vectors back to
 * back.  perm0[k], perm1[k]: member k's own permutations, as for bw_create.
 * No reference counterpart (the reference applies one Hmat per call). */
int bw_create_batch(int dof, int count, const int64_t *n_rows, const int64_t *n_cols, const int64_t *const *perm0,
                    const int64_t *const *perm1, int device, bw_hmat **out);

/* First scalar row and column of member k of a bw_create_batch handle (a
 * bw_create handle has the one member 0 at (0, 0)). */
int bw_batch_offsets(const bw_hmat *h, int member, int64_t *row0, int64_t *col0);

/* Number of members (1 for a bw_create handle, 0 for NULL). */
int bw_batch_count(const bw_hmat *h);

/* Bound (in ns, 1 ns .. 60 s, default 2 s) of every wait inside the kernels:
 * a stage that never fills or empties, an item reduction that never completes.
 * When a wait runs out the kernel writes an error word and returns; the
 * cleanup waits (copies in flight, tensor-core work before its memory is
 * freed) keep their own 2 s bound, so no work is left outstanding.  The next
 * bw_sync on the stream reports BW_ERR_DEVICE and clears the word; the handle
 * stays usable. */
int bw_set_wait_limit(bw_hmat *h, int64_t ns);

/* Test hook for the timeout path: in the next streaming launch (phase 1 of the
 * next bw_matvec or bw_matmat), CTA 0 never stages its chunk number `index`.
 * The wait for that chunk then runs out after the wait limit, the kernel
 * reports it through the error word, and the result of that call is
 * incomplete.  Nothing is left in flight: the chunk was never copied. */
int bw_test_withhold_chunk(bw_hmat *h, int index);

/* Plan parameters, set before bw_finalize (bigwham_dev_b200/tune.py sweeps
 * them on a GPU and commits the best per workload):
 *   "items_per_cta_phase1", "items_per_cta_phase2": items per CTA share
 *       (granularity of the work queue), 1..256, default 8;
 *   "chunk_bytes": block data per chunk, 4096..32768, multiple of 16,
 *       default 32768;
 *   "mm_items_per_cta": granularity of the matmat's phase 1, default 8;
 *   "unit_bytes": the streaming queue hands out runs of consecutive items
 *       until a run's cost reaches this many bytes (0: one item at a time),
 *       0..2^30, default 0;
 *   "narrow_rows", "narrow_cols", "narrow_coop": the items of a phase
 *       after its last item of more than narrow_rows padded rows (0..64,
 *       default 64) in the queue's cost order skip the staging: they run in a
 *       second launch with direct loads, warp per item, from the last item
 *       of more than narrow_cols columns (default 512) on; narrow_coop 1
 *       (default 0) runs the items before it there as well, a CTA per item,
 *       instead of in the CTA-wide kernel.  narrow_rows 0 keeps every item
 *       in the CTA-wide kernel.
 * They move item and chunk boundaries or the kernel an item runs in, and
 * with them the order of the additions that make an output row (results
 * agree to rounding); for fixed settings results are repeatable bit for bit
 * and do not depend on the schedule (each item is reduced in a fixed order).
 * BW_ERR_ARG for an unknown key or a value out of range. */
int bw_set_tuning(bw_hmat *h, const char *key, int64_t value);

/* Register a full-rank block: rows [i0, i0+m), cols [j0, j0+n), column-major
 * with leading dimension lda >= m.  The pointer is BORROWED until bw_finalize
 * returns (no copy is made before then).
 * Replaces: the FR half of HmatCuda::copyToDevice (hmat_cuda.cc:331-1183). */
int bw_add_full(bw_hmat *h, int64_t i0, int64_t j0, int64_t m, int64_t n, const double *a, int64_t lda);

/* Register a low-rank block y[i0:i0+m] += A (B x[j0:j0+n]) with A m x r
 * (lda >= m) and B r x n (ldb >= r), both column-major, exactly as
 * bigwham::LowRank stores them (src/hmat/hmatrix/LowRank.h:18-24,
 * hmat.cc:524-526).  r may differ block to block.  Pointers are BORROWED until
 * bw_finalize returns.  Replaces: the LR half of HmatCuda::copyToDevice. */
int bw_add_lowrank(bw_hmat *h, int64_t i0, int64_t j0, int64_t m, int64_t n, int64_t r, const double *A,
                   int64_t lda, const double *B, int64_t ldb);

/* Validate the pattern (in range, no overlaps, every row/column covered),
 * build the device layout for the precisions in `flags` (BW_FP64 | BW_FP32 |
 * BW_BF16, optionally BW_STORE_TRANSPOSE, BW_NO_FINITE_CHECK, BW_PLAN_ONLY)
 * and upload it.  Synchronous.  After it returns the borrowed block pointers
 * are no longer used. */
/* Register all blocks from the flat form (as bw_file_write takes it: fr
 * n_fr x 4 and lr n_lr x 5 in points on the host, the blocks back to back in
 * fr_data / lr_data) when the block data is in DEVICE memory of the handle's
 * device, e.g. from bw_r0_assemble_fr / bw_r0_aca.  bw_finalize then computes
 * the BF16 scales, the diagonal and the packed layout on the device (the host
 * never reads the data; results equal the host path's bit for bit).  The
 * arrays are borrowed until bw_finalize.  Only on an empty handle with a
 * device; not with BW_PLAN_ONLY or BW_STORE_MATMAT. */
int bw_add_flat_device(bw_hmat *h, int64_t n_fr, const int64_t *fr, int64_t n_lr, const int64_t *lr,
                       const double *fr_data, int64_t fr_len, const double *lr_data, int64_t lr_len);

int bw_finalize(bw_hmat *h, int flags);

/* y = H x (or H^T x with BW_TRANSPOSE) on DEVICE pointers, stream-ordered on
 * `stream` (a cudaStream_t; 0 is the legacy default stream).  Original dof
 * ordering unless BW_PERMUTED.  x and y must not overlap.  Does not
 * synchronize.
 * Replaces: Hmat<double>::matvecOriginal(double*, double*) / matvec(double*,
 * double*) (src/hmat/hmatrix/hmat.h:91,95; HmatCuda overrides at
 * hmat_cuda.cc:2397-2460), reached from BigWhamIO::MatVec(double*, double*)
 * (src/io/bigwham_io.cc:935-941) and py_bigwham matvec_raw_ptr
 * (interfaces/python/py_bigwham.cc:213-222). */
int bw_matvec(bw_hmat *h, const double *x, double *y, int flags, void *stream);

/* Bytes of device memory reserved by bw_matvec_static_scratch (per device). */
#define BW_STATIC_SCRATCH_BYTES (64u << 20)

/* y = H x like bw_matvec, but the call allocates no device memory: for callers
 * that cannot let a library call cudaMalloc -- a process whose device memory
 * belongs to another allocator (a framework's caching pool, a solver that
 * reserved the card up front), or a latency-critical path where cudaMalloc /
 * cudaFree are not allowed because they can synchronize the device.  The
 * caller passes x and y; the scratch vectors live in a fixed device array of
 * BW_STATIC_SCRATCH_BYTES (64 MiB) compiled into the library, which every GPU
 * that loads the library holds until the process exits.  H-matrices needing
 * more scratch than that are rejected with BW_ERR_ARG: 8 bytes (FP64) or 4
 * (FP32, BF16) per input, per low-rank rank column and per column of every row
 * panel (the phase-2 gather array).  For the 3DR0-H square crack that is
 * 14 MB (FP64) or 7 MB (FP32, BF16) at 12,288 DoF and 40 MB or 20 MB at
 * 49,152 DoF; the 196,608-DoF matrix needs more and is rejected.
 * The first call on a device looks the array's address up (once per device).
 * With lazy module loading (the CUDA default) that first lookup can also load
 * the library's device code, which reserves the array and may synchronize the
 * device: make the first call on each device outside latency-critical code and
 * before any stream capture.  The address is kept for the life of the process;
 * after cudaDeviceReset on a device, do not call this entry point on it again.
 * Every call overwrites the
 * scratch before reading it, so nothing in it needs to start at zero, and the
 * array keeps the last call's contents.  All calls on a device share the one
 * array: calls whose kernels overlap on the GPU (several streams or several
 * handles) race on it.  No counterpart in the reference. */
int bw_matvec_static_scratch(bw_hmat *h, const double *x, double *y, int flags, void *stream);

/* Same product on HOST arrays: copies x to the device, runs bw_matvec on the
 * handle's stream, copies y back and synchronizes.  The vectors move in four
 * pieces through pinned buffers of the handle, so the host copies overlap
 * the DMA; on BW_ERR_DEVICE the contents of y are unspecified.
 * Replaces: Hmat<double>::matvecOriginal(il::ArrayView<double>) / matvec(...)
 * (hmat.cc:572-635 / :472-537), reached from BigWhamIO::MatVec(il::ArrayView)
 * (bigwham_io.cc:927-933) and MatVecPerm (bigwham_io.cc:965-980). */
int bw_matvec_host(bw_hmat *h, const double *x, double *y, int flags);

/* Y = H X for nrhs right-hand sides on DEVICE pointers; X is n_cols x nrhs
 * (column stride ldx), Y is n_rows x nrhs (column stride ldy), FP64 in and out.
 * With BW_BF16 on a handle finalized with BW_STORE_MATMAT this runs on the
 * tensor cores:
 *  - X is rounded to BF16, products accumulate in FP32;
 *  - 64 right-hand sides per pass of 3 launches.
 * Otherwise it is one bw_matvec per column.  BW_PERMUTED and BW_TRANSPOSE
 * apply as for bw_matvec.  No reference counterpart. */
int bw_matmat(bw_hmat *h, const double *X, int64_t ldx, double *Y, int64_t ldy, int nrhs, int flags,
              void *stream);

/* Diagonal of H into a HOST array of length max(n_rows, n_cols), original
 * ordering unless BW_PERMUTED.  Replaces: Hmat::diagonalOriginal / diagonal
 * (hmat.cc:240-285) and HmatCuda::setDiagonal (hmat_cuda.cc:2462-2493). */
int bw_diagonal(bw_hmat *h, double *d, int flags);

/* Wait for the handle's pending work on `stream` and read the device error
 * word; BW_ERR_DEVICE if a kernel reported one (the word is then cleared). */
int bw_sync(bw_hmat *h, void *stream);

/* Sizes and statistics.  Fills up to n values of:
 * [0] n_rows [1] n_cols [2] dof [3] n_full [4] n_lowrank [5] stored entries
 * (Hmat::nbOfEntries, hmat.cc:299-313) [6] sum of ranks [7] n row panels
 * [8] device bytes in use [9] grid CTAs [10] phase-1 chunks (FP64)
 * [11] phase-2 chunks (FP64) [12] stored precisions mask.  Returns BW_OK. */
int bw_info(const bw_hmat *h, int64_t *out, int n);

/* Algorithmic bytes of one matvec in the given precision: stored entries x
 * element size (+ the BF16 per-block scales) + 8 bytes per input and per output
 * scalar.  Fills *bytes. */
int bw_algorithmic_bytes(const bw_hmat *h, int precision, int64_t *bytes);

/* Last error message of the handle (or of the last failed bw_create when h is
 * NULL), NUL-terminated into buf. */
int bw_last_error(const bw_hmat *h, char *buf, size_t len);

/* Cap on the device bytes bw_finalize may allocate (0 = no cap).  Exceeding it
 * makes bw_finalize return BW_ERR_OOM before allocating. */
int bw_set_device_limit(bw_hmat *h, int64_t bytes);

/* Host view of the matmat plan (BW_STORE_MATMAT) for one phase:
 *  - chunks: n_chunks x 16 int32 words in the layout of bw::MmChunk
 *    (bigwham_dev_b200/csrc/bw_layout.h);
 *  - data: n_elems raw BF16 words in 8x8 tiles (BW_PLAN_ONLY handles only);
 *  - item_ptr: the chunk ranges of the items (n_item_ptr = items + 1), in the
 *    order the kernel's CTAs take them (longest first);
 *  - t8_len: rows of the low-rank product array T8.
 * Any output pointer may be NULL. */
int bw_mm_plan_export(const bw_hmat *h, int phase, int transposed, int64_t *n_chunks, int32_t *chunks,
                      int64_t *n_elems, uint16_t *data, int64_t *n_item_ptr, int32_t *item_ptr, int64_t *t8_len);

/* Host view of the built plan for one precision and phase (1: low-rank B
 * stage, 2: row panels), for inspection and testing.  Any output pointer may be
 * NULL; counts are always written.  chunks: n_chunks x 8 int32 words in the
 * layout of bw::Chunk (bigwham_dev_b200/csrc/bw_layout.h); data: n_elems values
 * converted to double, in the precision's layout (column-major items for FP64 /
 * FP32, 8x8 tiles for BF16; BF16 values divided by their block scale);
 * item_ptr: the chunk ranges of the items (n_item_ptr = items + 1 offsets), in
 * the order the kernel's CTAs take them (longest first).  data is only
 * available on a handle finalized with BW_PLAN_ONLY. */
int bw_plan_export(const bw_hmat *h, int precision, int phase, int transposed, int64_t *n_chunks,
                   int32_t *chunks, int64_t *n_elems, double *data, int64_t *n_item_ptr, int32_t *item_ptr);

/* How one phase's items divide between the two streaming kernels: items
 * [0, n_wide) of bw_plan_export's item order run in the CTA-wide kernel, the
 * rest in the unstaged kernel, [n_wide, n_coop) a CTA per item and the rest
 * warp per item (the "narrow_*" tuning keys). */
int bw_plan_split(const bw_hmat *h, int precision, int phase, int transposed, int64_t *n_wide, int64_t *n_coop);

/* Kernel launches of one bw_matvec in this precision and direction: the x
 * gather, the G2 gather and one or two per phase (CTA-wide, unstaged). */
int bw_matvec_launches(const bw_hmat *h, int precision, int transposed, int64_t *n);

/* Per-launch timing for benchmarks.  With timing enabled every bw_matvec
 * records CUDA events on its stream around its launches (x gather, phase 1,
 * G2 gather, phase 2; a phase is one launch of the CTA-wide kernel, of the
 * unstaged kernel, or of both).  bw_timing_read waits for the last recorded
 * event, writes the summed durations in milliseconds of the four steps into
 * ms[0..3] and the number of recorded matvecs, and clears the record. */
int bw_set_timing(bw_hmat *h, int enable);
int bw_timing_read(bw_hmat *h, double *ms, int64_t *n_matvecs);
/* The same record launch by launch, ms[0..5]: x gather, phase 1 CTA-wide,
 * phase 1 unstaged, G2 gather, phase 2 CTA-wide, phase 2 unstaged (0 for a
 * kernel a phase does not use).  Clears the record like bw_timing_read. */
int bw_timing_read_launches(bw_hmat *h, double *ms, int64_t *n_matvecs);

/* Algorithmic bytes of each streaming launch of one matvec: phase 1 reads the
 * low-rank B factors (+ x, + t written), phase 2 reads the full blocks and the
 * A factors (+ y written).  Stored entries only: padding is not counted. */
int bw_phase_bytes(const bw_hmat *h, int precision, int transposed, int64_t *phase1, int64_t *phase2);

/* Runs that fill the phase-2 gather array (4 int32 words each: dst, src_off,
 * cols | src << 31, scale bits), for inspection and testing. */
int bw_plan_gather(const bw_hmat *h, int precision, int transposed, int64_t *n, int32_t *runs);

/* Per-t-entry scales of the BF16 layout (scale(A) * scale(B) of the entry's
 * low-rank block; 1 elsewhere), for inspection and testing.  Phase 1 writes t
 * unscaled; the phase-2 gather runs that read t carry these products. */
int bw_plan_tscale(const bw_hmat *h, int transposed, int64_t *n, float *out);

/* ---- Block files ----------------------------------------------------------
 * A built H-matrix on disk: dof, sizes, both permutations, the HPattern
 * columns (spot, i0, j0, i_end, j_end, flag) of every block, the full-rank
 * blocks, each low-rank block's A and B, and optionally the low-rank blocks'
 * ACA error estimates, in a page-aligned binary with a checksum per section.
 * The content of the reference's Hmat<T>::writeToFile / readFromFile
 * (src/hmat/hmatrix/hmat.cc:749-935, declared hmat.h:100-101), which need
 * HDF5; here the file is mapped, so a later run uploads the blocks without
 * rebuilding the H-matrix.  Writers go through a temporary file renamed into
 * place.  Errors: BW_ERR_ARG (inconsistent arguments), BW_ERR_IO (file cannot
 * be read or written, is not a block file, is truncated, or fails a checksum);
 * bw_last_error(NULL, ...) gives the message. */

/* Write from the flat form of bwh_export: fr (n_fr x 4: i0, j0, i_end, j_end
 * in points), lr (n_lr x 5: the same + rank in scalar columns), the FR blocks
 * back to back and per LR block A then B (column-major, no padding).
 * lr_error: n_lr values or NULL.  The HPattern spot of block k is stored as k. */
int bw_file_write(const char *path, int dof, int64_t n_rows, int64_t n_cols, const int64_t *perm0,
                  const int64_t *perm1, int64_t n_fr, const int64_t *fr, const double *fr_data, int64_t n_lr,
                  const int64_t *lr, const double *lr_data, const double *lr_error);

/* Write from per-block pointers, as an Hmat holds them: fr_pattern /
 * lr_pattern are HPattern columns (n x 6, FRB_pattern / LRB_pattern of
 * h_pattern.h:21-33 with LR flag = rank in scalar columns, hmat.cc:390); block
 * k is column-major at fr[k] with leading dimension fr_ld[k] (>= its rows),
 * its factors at lr_a[k] (ld lr_a_ld[k]) and lr_b[k] (ld lr_b_ld[k]). */
int bw_file_write_blocks(const char *path, int dof, int64_t n_rows, int64_t n_cols, const int64_t *perm0,
                         const int64_t *perm1, int64_t n_fr, const int64_t *fr_pattern, const double *const *fr,
                         const int64_t *fr_ld, int64_t n_lr, const int64_t *lr_pattern, const double *const *lr_a,
                         const int64_t *lr_a_ld, const double *const *lr_b, const int64_t *lr_b_ld,
                         const double *lr_error);

/* Header of a block file (the header checksum, section bounds, pattern and
 * permutations are checked): info[0..8] = dof, n_rows, n_cols, n_fr, n_lr,
 * FR entries, LR entries, 1 if ACA error estimates are stored, file bytes. */
int bw_file_info(const char *path, int64_t info[9]);

/* Copy a block file out in the flat form of bw_file_write (array sizes from
 * bw_file_info).  fr_data / lr_data may be NULL to leave that block data in
 * the file; lr_error may be NULL (zeros are written when the file has none);
 * fr_pattern / lr_pattern (n x 6 HPattern columns) may be NULL.  verify != 0
 * also checks the block data checksums. */
int bw_file_read(const char *path, int verify, int64_t *fr, int64_t *lr, double *fr_data, double *lr_data,
                 int64_t *perm0, int64_t *perm1, double *lr_error, int64_t *fr_pattern, int64_t *lr_pattern);

/* Create a handle from a block file: bw_create with the file's sizes and
 * permutations, then every block registered as bw_add_full / bw_add_lowrank
 * would, borrowing the mapped file (no copy) until bw_finalize succeeds or the
 * handle is destroyed.  Call bw_set_tuning / bw_set_device_limit and
 * bw_finalize on it as usual.  verify != 0 checks the block data checksums
 * first (one pass over the file). */
int bw_create_from_file(const char *path, int device, int verify, bw_hmat **out);

/* ---- Device assembly (3DR0-H) ----------------------------------------------
 * Full-rank blocks of a 3DR0-H H-matrix computed on the device: the work of
 * the reference's Hmat::buildFR (src/hmat/hmatrix/hmat.cc:315-353) for the
 * rectangle hypersingular kernel
 * (src/elasticity/fullspace_iso_3d_rectangle/
 * bie_elastostatic_rectangle_0_influence.h:29-125).
 * records: n_elems x 17 doubles per element (collocation point, rotation
 * matrix row-major with local = R global, unit normal, half sides a and b
 * along the local x and y); G, nu: shear modulus and Poisson ratio; fr:
 * n_fr x 4 blocks (i0, j0, i_end, j_end) in permuted points; perm: n_points
 * values, permuted point -> element.  out (device, out_len doubles): the
 * blocks back to back, column-major, as bw_add_full / bw_file_write take
 * them.  Every index is checked on the host before the launch; returns once
 * the blocks are written (stream-ordered, then synchronized). */
int bw_r0_assemble_fr(int device, int64_t n_elems, const double *records, double G, double nu, int64_t n_fr,
                      const int64_t *fr, const int64_t *perm, int64_t n_points, double *out, int64_t out_len,
                      void *stream);

/* Low-rank blocks of a 3DR0-H H-matrix compressed on the device by block ACA
 * (3 x 3 pivots, the reference's adaptiveCrossApproximation<3>,
 * src/hmat/compression/adaptiveCrossApproximation.h:24-226), one CTA per
 * block.  records / perm / G / nu as for bw_r0_assemble_fr; lr: n_lr x 4
 * admissible blocks in permuted points; eps: the ACA tolerance.  Block k gets
 * cap_k = min(cap_blocks, rows, columns) rank blocks of storage: A_k (rows 3 x
 * cap_k 3) at factors_a + sum_{l<k} 9 rows_l cap_l and B_k (cap_k 3 x
 * columns 3) at factors_b + sum_{l<k} 9 columns_l cap_l, column-major, device
 * memory (a_len / b_len doubles available).  rank_out (host): each block's
 * scalar rank, -1 when cap_k was too small; err_out (host): the ACA error
 * estimate.  Every index is checked on the host before the launch. */
int bw_r0_aca(int device, int64_t n_elems, const double *records, double G, double nu, int64_t n_lr,
              const int64_t *lr, const int64_t *perm, int64_t n_points, double eps, int cap_blocks,
              double *factors_a, int64_t a_len, double *factors_b, int64_t b_len, int32_t *rank_out,
              double *err_out, void *stream);

/* Stresses and displacements at observation points from a solution on a
 * 2DS0 mesh (straight segments, constant displacement discontinuity, plane
 * strain): the device counterpart of BigWhamIO::ComputeStresses /
 * ComputeDisplacements (src/io/bigwham_io.cc:1166-1324) for kernel 2DS0-H.
 * All arrays are device memory.  records: n_elems x 5 (centre x, y, half
 * length, unit tangent x, y, the tangent running from the first vertex to the
 * second); dd: n_elems x 2 local DDs (shear, normal), mesh order; pts:
 * n_pts x 2; stress (n_pts x 3: s11, s22, s12) and / or disp (n_pts x 2,
 * global frame) may be null, not both.  Each point sums the elements in mesh
 * order.  Stream-ordered; returns after the launch. */
int bw_s0_fields(int device, int64_t n_elems, const double *records, const double *dd, double G, double nu,
                 int64_t n_pts, const double *pts, double *stress, double *disp, void *stream);

/* Stresses and displacements at observation points from a solution on a
 * 3DR0 mesh (rectangles, constant displacement discontinuity), global frame.
 * The reference's BigWhamIO returns zeros for this kernel family (its 3DR0
 * observation kernels are stubs); these are the sums of its element kernels
 * StressesKernelR0 / DisplacementKernelR0 in the layout of its 3D
 * observation kernels.  All arrays are device memory.  records: n_elems x 17
 * as for bw_r0_assemble_fr; dd: n_elems x 3 local DDs, mesh order; pts:
 * n_pts x 3; stress (n_pts x 6: s11, s22, s33, s12, s13, s23) and / or disp
 * (n_pts x 3) may be null, not both.  Each point sums the elements in mesh
 * order.  Stream-ordered; returns after the launch. */
int bw_r0_fields(int device, int64_t n_elems, const double *records, const double *dd, double G, double nu,
                 int64_t n_pts, const double *pts, double *stress, double *disp, void *stream);

/* Release everything. */
int bw_destroy(bw_hmat *h);

/* Library version string. */
const char *bw_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BIGWHAM_B200_H */
