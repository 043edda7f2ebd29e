// C ABI of BigWhamIO with the B200 backend installed (include/bigwham_host.h).
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "bigwham_host.h"
#include "cblas.h"
#include "hmat_gpu.h"
#include "io/bigwham_io.h"

#ifdef BIGWHAM_OPENMP
#include <omp.h>
#endif

struct bwh_io {
  std::unique_ptr<BigWhamIO> io;
  std::shared_ptr<bigwham_b200::HmatGpu> gpu;
  std::vector<std::pair<std::string, int64_t>> tuning;  // for the next bwh_attach_gpu
  std::shared_ptr<bigwham::Hmat<double>> cpu_kept;        // host blocks kept by bwh_attach_gpu(release_host = 0)
};

namespace {
std::mutex g_mu;
std::string g_err;

int fail(const std::string &m, int code = 1) {
  std::lock_guard<std::mutex> g(g_mu);
  g_err = m;
  return code;
}

template <typename F> int guarded(F &&f) {
  try {
    return f();
  } catch (const std::exception &e) {
    return fail(e.what());
  } catch (...) {
    return fail("unknown C++ exception (an il::abort / IL_EXPECT check of the reference?)");
  }
}
}  // namespace

extern "C" {

int bwh_create(const double *coor, int64_t n_coor, const int *conn, int64_t n_conn, const char *kernel,
               const double *properties, int n_properties, int n_openmp_threads, int verbose, int fixed_rank,
               bwh_io **out) {
  if (!out || !coor || !conn || !kernel || !properties) return fail("null argument");
  *out = nullptr;
  return guarded([&] {
    // the reference's matvec parallelism is over blocks: one BLAS thread
    openblas_set_num_threads(1);
    std::vector<double> c(coor, coor + n_coor);
    std::vector<int> e(conn, conn + n_conn);
    std::vector<double> p(properties, properties + n_properties);
    std::unique_ptr<bwh_io> h(new bwh_io);
    h->io.reset(new BigWhamIO(c, e, std::string(kernel), p, n_openmp_threads, 0, verbose != 0, false, false,
                              fixed_rank));
    *out = h.release();
    return 0;
  });
}

int bwh_create_rect(const double *coor_src, int64_t n_coor_src, const int *conn_src, int64_t n_conn_src,
                    const double *coor_rec, int64_t n_coor_rec, const int *conn_rec, int64_t n_conn_rec,
                    const char *kernel, const double *properties, int n_properties, int n_openmp_threads,
                    int verbose, int fixed_rank, bwh_io **out) {
  if (!out || !coor_src || !conn_src || !coor_rec || !conn_rec || !kernel || !properties)
    return fail("null argument");
  *out = nullptr;
  return guarded([&] {
    openblas_set_num_threads(1);
    std::vector<double> cs(coor_src, coor_src + n_coor_src), cr(coor_rec, coor_rec + n_coor_rec);
    std::vector<int> es(conn_src, conn_src + n_conn_src), er(conn_rec, conn_rec + n_conn_rec);
    std::vector<double> p(properties, properties + n_properties);
    std::unique_ptr<bwh_io> h(new bwh_io);
    h->io.reset(new BigWhamIO(cs, es, cr, er, std::string(kernel), p, n_openmp_threads, 0, verbose != 0, false,
                              false, fixed_rank));
    *out = h.release();
    return 0;
  });
}

int bwh_build(bwh_io *h, int leaf, double eta, double eps) {
  if (!h) return fail("null handle");
  return guarded([&] {
    h->io->BuildHierarchicalMatrix(leaf, eta, eps);
    return h->io->is_built() ? 0 : fail("BuildHierarchicalMatrix did not build");
  });
}

int bwh_build_pattern(bwh_io *h, int leaf, double eta) {
  if (!h) return fail("null handle");
  return guarded([&] {
    h->io->BuildPattern(leaf, eta);
    return 0;
  });
}

int bwh_attach_gpu(bwh_io *h, int device, int storage, int release_host) {
  if (!h) return fail("null handle");
  return guarded([&] {
    if (!h->io->is_built()) return fail("bwh_attach_gpu before bwh_build");
    auto cpu = h->io->getHmat();
    auto gpu = std::make_shared<bigwham_b200::HmatGpu>(cpu, device, storage, h->tuning);
    h->io->setHmat(gpu);
    h->gpu = gpu;
    if (release_host)
      cpu->hmatMemFree();
    else
      h->cpu_kept = cpu;
    return 0;
  });
}

int bwh_set_tuning(bwh_io *h, const char *key, int64_t value) {
  if (!h || !key) return fail("null argument");
  h->tuning.emplace_back(key, value);
  return 0;
}

int bwh_set_precision(bwh_io *h, int p) {
  if (!h || !h->gpu) return fail("no GPU H-matrix attached");
  if (p != BW_FP64 && p != BW_FP32 && p != BW_BF16) return fail("precision must be BW_FP64, BW_FP32 or BW_BF16");
  h->gpu->set_precision(p);
  return 0;
}

// The matvec entries require the GPU H-matrix: this library never applies the
// reference's CPU matvec.  BigWhamIO::MatVec / MatVecPerm return a new
// il::Array (bigwham_io.cc:927-933, 965-971) that a binding then copies into
// the caller's array; with the GPU H-matrix installed those two calls reduce
// to HmatGpu's host-array product, which writes the caller's y directly (no
// intermediate array, no second copy).
int bwh_matvec(bwh_io *h, const double *x, double *y) {
  if (!h || !x || !y) return fail("null argument");
  if (!h->gpu) return fail("no GPU H-matrix attached (bwh_attach_gpu)");
  return guarded([&] {
    h->gpu->matvecOriginalInto(x, y);
    return 0;
  });
}

int bwh_matvec_perm(bwh_io *h, const double *x, double *y) {
  if (!h || !x || !y) return fail("null argument");
  if (!h->gpu) return fail("no GPU H-matrix attached (bwh_attach_gpu)");
  return guarded([&] {
    h->gpu->matvecInto(x, y);
    return 0;
  });
}

int bwh_matvec_raw_ptr(bwh_io *h, double *x, double *y) {
  if (!h || !x || !y) return fail("null argument");
  if (!h->gpu) return fail("matvec_raw_ptr needs the GPU H-matrix (bwh_attach_gpu)");
  return guarded([&] {
    h->io->MatVec(x, y);
    return 0;
  });
}

int bwh_diagonal(bwh_io *h, double *d) {
  if (!h || !d) return fail("null argument");
  return guarded([&] {
    std::vector<double> v;
    h->io->GetDiagonal(v);
    std::memcpy(d, v.data(), sizeof(double) * v.size());
    return 0;
  });
}

int64_t bwh_size(const bwh_io *h, int k) { return h ? h->io->getHmat()->size(k) : -1; }
int bwh_dof(const bwh_io *h) { return h ? h->io->dof_dimension() : -1; }
double bwh_compression(const bwh_io *h) { return h ? h->io->GetCompressionRatio() : -1.0; }
double bwh_hmat_time(const bwh_io *h) { return h ? h->io->hmat_time() : -1.0; }

int bwh_permutation(const bwh_io *h, int64_t *perm) {
  if (!h || !perm) return fail("null argument");
  std::vector<long> p = h->io->GetPermutation();
  for (size_t i = 0; i < p.size(); i++) perm[i] = p[i];
  return 0;
}

int64_t bwh_collocation_points(const bwh_io *h, double *out) {
  if (!h) return -1;
  std::vector<double> v = h->io->GetCollocationPoints();
  if (out) std::memcpy(out, v.data(), sizeof(double) * v.size());
  return (int64_t)v.size();
}

int64_t bwh_hpattern(const bwh_io *h, double *out) {
  if (!h) return -1;
  std::vector<double> v = h->io->GetHPattern();
  if (out) std::memcpy(out, v.data(), sizeof(double) * v.size());
  return (int64_t)v.size();
}

int64_t bwh_n_blocks(const bwh_io *h, int kind) {
  if (!h) return -1;
  auto p = h->io->getHmat()->pattern();
  return kind == 0 ? p.n_FRB : p.n_LRB;
}

int64_t bwh_entries(const bwh_io *h, int kind) {
  if (!h) return -1;
  auto hm = h->io->getHmat();
  auto p = hm->pattern();
  const il::int_t dof = hm->dofDimension();
  int64_t n = 0;
  if (kind == 0) {
    for (il::int_t k = 0; k < p.n_FRB; k++)
      n += (p.FRB_pattern(3, k) - p.FRB_pattern(1, k)) * (p.FRB_pattern(4, k) - p.FRB_pattern(2, k)) * dof * dof;
  } else {
    for (il::int_t k = 0; k < p.n_LRB; k++)
      n += p.LRB_pattern(5, k) * ((p.LRB_pattern(3, k) - p.LRB_pattern(1, k)) + (p.LRB_pattern(4, k) - p.LRB_pattern(2, k))) * dof;
  }
  return n;
}

int bwh_export(const bwh_io *h, int64_t *fr, int64_t *lr, double *fr_data, double *lr_data, int64_t *perm0,
               int64_t *perm1) {
  if (!h) return fail("null handle");
  if (h->gpu && !h->cpu_kept)
    return fail("bwh_export needs the host blocks: call it before bwh_attach_gpu, or attach with release_host = 0");
  return guarded([&] {
    auto hm = h->gpu ? h->cpu_kept : h->io->getHmat();
    auto p = hm->pattern();
    auto hr = hm->get_hr();
    for (il::int_t k = 0; k < p.n_FRB; k++)
      for (int r = 0; r < 4; r++) fr[4 * k + r] = p.FRB_pattern(r + 1, k);
    for (il::int_t k = 0; k < p.n_LRB; k++)
      for (int r = 0; r < 5; r++) lr[5 * k + r] = p.LRB_pattern(r + 1, k);
    for (il::int_t i = 0; i < hr->permutation_0_.size(); i++) perm0[i] = hr->permutation_0_[i];
    for (il::int_t i = 0; i < hr->permutation_1_.size(); i++) perm1[i] = hr->permutation_1_[i];
    auto copy = [](const il::Array2D<double> &a, double *out) {
      auto v = a.view();
      for (il::int_t j = 0; j < v.size(1); j++)
        std::memcpy(out + j * v.size(0), &v(0, j), sizeof(double) * v.size(0));
      return v.size(0) * v.size(1);
    };
    int64_t o = 0;
    for (const auto &b : hm->get_full_rank_blocks()) o += copy(*b, fr_data + o);
    o = 0;
    for (const auto &b : hm->get_low_rank_blocks()) {
      o += copy(b->A, lr_data + o);
      o += copy(b->B, lr_data + o);
    }
    return 0;
  });
}

int64_t bwh_element_frames(const bwh_io *h, double *out) {
  if (!h) return fail("null handle"), -1;
  int64_t n = -1;
  const int rc = guarded([&] {
    const std::vector<double> cp = h->io->GetCollocationPoints(), rot = h->io->GetRotationMatrix(),
                              nrm = h->io->GetElementNormals();
    const size_t ne = nrm.size() / 3;
    if (h->io->spatial_dimension() != 3 || cp.size() != 3 * ne || rot.size() != 9 * ne)
      return fail("bwh_element_frames: needs a 3D mesh with one collocation point per element");
    n = (int64_t)ne;
    if (out)
      for (size_t e = 0; e < ne; e++) {
        for (int k = 0; k < 3; k++) out[15 * e + k] = cp[3 * e + k];
        for (int k = 0; k < 9; k++) out[15 * e + 3 + k] = rot[9 * e + k];
        for (int k = 0; k < 3; k++) out[15 * e + 12 + k] = nrm[3 * e + k];
      }
    return 0;
  });
  return rc == 0 ? n : -1;
}

int bwh_write_to_file(const bwh_io *h, const char *path) {
  if (!h || !path) return fail("null argument");
  if (h->gpu && !h->cpu_kept)
    return fail("bwh_write_to_file: the host blocks were released by bwh_attach_gpu (attach with release_host = 0 "
                "to keep them)");
  return guarded([&] {
    bigwham_b200::write_block_file(h->gpu ? *h->cpu_kept : *h->io->getHmat(), path);
    return 0;
  });
}

int bwh_convert(const bwh_io *h, int to_global, const double *in, int64_t n, double *out) {
  if (!h || !in || !out || n < 0) return fail("null argument");
  return guarded([&] {
    il::Array<double> v = to_global ? h->io->ConvertToGlobal(il::ArrayView<double>{in, n})
                                    : h->io->ConvertToLocal(il::ArrayView<double>{in, n});
    if (v.size() != n) return fail("bwh_convert: the mesh has a different number of values");
    std::memcpy(out, v.data(), sizeof(double) * (size_t)n);
    return 0;
  });
}

namespace {
int64_t vec_out(const std::vector<double> &v, double *out) {
  if (out) std::memcpy(out, v.data(), sizeof(double) * v.size());
  return (int64_t)v.size();
}
}  // namespace

int64_t bwh_element_normals(const bwh_io *h, double *out) {
  if (!h) return fail("null handle"), -1;
  int64_t n = -1;
  guarded([&] {
    n = vec_out(h->io->GetElementNormals(), out);
    return 0;
  });
  return n;
}

int64_t bwh_rotation_matrix(const bwh_io *h, double *out) {
  if (!h) return fail("null handle"), -1;
  int64_t n = -1;
  guarded([&] {
    n = vec_out(h->io->GetRotationMatrix(), out);
    return 0;
  });
  return n;
}

double bwh_max_error_aca(const bwh_io *h) {
  if (!h || !h->io->is_built()) return fail("bwh_max_error_aca before bwh_build"), -1.0;
  double e = -1.0;
  guarded([&] {
    e = h->io->GetMaxErrorACA();
    return 0;
  });
  return e;
}

int64_t bwh_full_blocks(const bwh_io *h, int original_order, double *val, int32_t *row, int32_t *col) {
  if (!h || !h->io->is_built()) return fail("bwh_full_blocks before bwh_build"), -1;
  int64_t n = -1;
  guarded([&] {
    std::vector<double> v;
    std::vector<int> pos;
    if (original_order)
      h->io->GetFullBlocks(v, pos);
    else
      h->io->GetFullBlocksPerm(v, pos);
    n = (int64_t)v.size();
    if (val) std::memcpy(val, v.data(), sizeof(double) * v.size());
    if (row && col)
      for (int64_t i = 0; i < n; i++) {
        row[i] = pos[2 * i];
        col[i] = pos[2 * i + 1];
      }
    return 0;
  });
  return n;
}

int64_t bwh_compute_fields(const bwh_io *h, int kind, const double *coor_obs, int64_t n_coor, const double *sol,
                           int64_t n_sol, double *out, int64_t out_len) {
  if (!h || !coor_obs || !sol || n_coor < 0 || n_sol < 0) return fail("null argument"), -1;
  int64_t n = -1;
  guarded([&] {
    const std::vector<double> c(coor_obs, coor_obs + n_coor);
    il::Array<double> v = kind == 0 ? h->io->ComputeDisplacements(c, il::ArrayView<double>{sol, n_sol})
                                    : h->io->ComputeStresses(c, il::ArrayView<double>{sol, n_sol});
    n = v.size();
    if (out) {
      if (out_len < n) return fail("bwh_compute_fields: out is too short");
      std::memcpy(out, v.data(), sizeof(double) * (size_t)n);
    }
    return 0;
  });
  return n;
}

int64_t bwh_storage_requirement(const bwh_io *h) {
  if (!h || !h->io->is_built()) return fail("bwh_storage_requirement before bwh_build"), -1;
  return (int64_t)h->io->getHmat()->nbOfEntries() * (int64_t)sizeof(double);
}

int bwh_omp_threads(const bwh_io *h) { return h ? h->io->GetOmpThreads() : -1; }

int bwh_spatial_dimension(const bwh_io *h) { return h ? h->io->spatial_dimension() : -1; }

struct bw_hmat *bwh_gpu_handle(bwh_io *h) { return (h && h->gpu) ? h->gpu->handle() : nullptr; }

int bwh_destroy(bwh_io *h) {
  delete h;
  return 0;
}

const char *bwh_last_error(void) {
  std::lock_guard<std::mutex> g(g_mu);
  return g_err.c_str();
}

}  // extern "C"
