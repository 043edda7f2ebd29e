// Oracle-side C entry points over the UNMODIFIED reference library.
//
// TEST INFRASTRUCTURE ONLY.  This file is linked, together with the reference
// sources compiled by oracle/Makefile, into oracle/_ref/libbigwham_ref.so.  Only
// the test suite, the smoke check and the CPU-baseline leg of the benchmark may
// load that library.  It exposes the reference's own construction
// (BigWhamIO ctor + BuildHierarchicalMatrix, src/io/bigwham_io.cc:41-290 and
// :635-704) and the reference's own OpenMP CPU matvec
// (BigWhamIO::MatVec -> Hmat<double>::matvecOriginal, src/io/bigwham_io.cc:927-933,
// src/hmat/hmatrix/hmat.cc:572-635) to Python through ctypes, plus read access
// to the built blocks so golden vectors can be dumped.
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cblas.h"
#include "core/bie_kernel.h"
#include "core/elastic_properties.h"
#include "elasticity/bie_elastostatic.h"
#include "elasticity/fullspace_iso_2d_segment/bie_elastostatic_segment_0_influence.h"
#include "elasticity/fullspace_iso_3d_rectangle/bie_elastostatic_rectangle_0_influence.h"
#include "elasticity/fullspace_iso_3d_rectangle/elastic_3dR0_element.h"
#include "elasticity/fullspace_iso_3d_triangle/bie_elastostatic_triangle_0_influence.h"
#include "elements/rectangle.h"
#include "elements/segment.h"
#include "elements/triangle.h"
#include "hmat/arrayFunctor/GaussianMatrix.h"
#include "hmat/cluster/cluster.h"
#include "hmat/hierarchical_representation.h"
#include "hmat/hmatrix/h_pattern.h"
#include "hmat/hmatrix/hmat.h"
#include "io/bigwham_io.h"

#ifdef BIGWHAM_OPENMP
#include <omp.h>
#endif

namespace {
struct RefHandle {
  std::unique_ptr<BigWhamIO> io;
};
RefHandle *H(void *h) { return static_cast<RefHandle *>(h); }

// The reference's Gaussian-matrix H-matrix (no mesh, no BigWhamIO): cluster
// tree, pattern and Hmat built by its own code over its GaussianMatrix
// generator (dof 1).
struct RefGauss {
  std::shared_ptr<bigwham::HRepresentation> hr;
  std::unique_ptr<bigwham::Hmat<double>> h;
};
RefGauss *GS(void *h) { return static_cast<RefGauss *>(h); }
}  // namespace

extern "C" {

// Sets the OpenMP thread count used by the reference and pins the BLAS to one
// thread, as the reference expects (the parallelism is over blocks).
int ref_set_threads(int n) {
  openblas_set_num_threads(1);
#ifdef BIGWHAM_OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// Square self-interaction BigWhamIO (src/io/bigwham_io.h:73-82); CUDA off.
void *ref_create(const double *coor, int64_t n_coor, const int *conn, int64_t n_conn, const char *kernel,
                 const double *props, int n_props, int n_threads, int verbose) {
  try {
    std::vector<double> c(coor, coor + n_coor);
    std::vector<int> e(conn, conn + n_conn);
    std::vector<double> p(props, props + n_props);
    auto *h = new RefHandle;
    h->io.reset(new BigWhamIO(c, e, std::string(kernel), p, n_threads, 0, verbose != 0, false, false, -1));
    return h;
  } catch (...) {
    return nullptr;
  }
}

// Rectangular BigWhamIO (src/io/bigwham_io.h:85-96): source mesh x receiver
// mesh, kernels such as "3DR0-3DR0-H"; CUDA off.
void *ref_create_rect(const double *coor_src, int64_t n_coor_src, const int *conn_src, int64_t n_conn_src,
                      const double *coor_rec, int64_t n_coor_rec, const int *conn_rec, int64_t n_conn_rec,
                      const char *kernel, const double *props, int n_props, int n_threads, int verbose) {
  try {
    std::vector<double> cs(coor_src, coor_src + n_coor_src), cr(coor_rec, coor_rec + n_coor_rec);
    std::vector<int> es(conn_src, conn_src + n_conn_src), er(conn_rec, conn_rec + n_conn_rec);
    std::vector<double> p(props, props + n_props);
    auto *h = new RefHandle;
    h->io.reset(new BigWhamIO(cs, es, cr, er, std::string(kernel), p, n_threads, 0, verbose != 0, false, false, -1));
    return h;
  } catch (...) {
    return nullptr;
  }
}

int ref_build(void *h, int leaf, double eta, double eps) {
  try {
    H(h)->io->BuildHierarchicalMatrix(leaf, eta, eps);
    return H(h)->io->is_built() ? 0 : 2;
  } catch (...) {
    return 1;
  }
}

int64_t ref_size(void *h, int k) { return H(h)->io->getHmat()->size(k); }
int ref_dof(void *h) { return H(h)->io->dof_dimension(); }
double ref_compression(void *h) { return H(h)->io->GetCompressionRatio(); }

int64_t ref_n_blocks(void *h, int kind) {
  auto p = H(h)->io->getHmat()->pattern();
  return kind == 0 ? p.n_FRB : p.n_LRB;
}

// FR: 4 int64 per block (i0, j0, iend, jend) in collocation-point units.
// LR: 5 int64 per block (i0, j0, iend, jend, rank in scalar columns), h_pattern.h:21-33, hmat.cc:390.
int ref_pattern(void *h, int64_t *fr, int64_t *lr) {
  auto p = H(h)->io->getHmat()->pattern();
  for (il::int_t k = 0; k < p.n_FRB; k++)
    for (int r = 0; r < 4; r++) fr[4 * k + r] = p.FRB_pattern(r + 1, k);
  for (il::int_t k = 0; k < p.n_LRB; k++)
    for (int r = 0; r < 5; r++) lr[5 * k + r] = p.LRB_pattern(r + 1, k);
  return 0;
}

int ref_permutation(void *h, int64_t *p0, int64_t *p1) {
  auto hr = H(h)->io->getHmat()->get_hr();
  for (il::int_t i = 0; i < hr->permutation_0_.size(); i++) p0[i] = hr->permutation_0_[i];
  for (il::int_t i = 0; i < hr->permutation_1_.size(); i++) p1[i] = hr->permutation_1_[i];
  return 0;
}

static void copy_colmajor(const il::Array2D<double> &a, double *out) {
  auto v = a.view();
  const il::int_t m = v.size(0), n = v.size(1);
  for (il::int_t j = 0; j < n; j++)
    for (il::int_t i = 0; i < m; i++) out[i + j * m] = v(i, j);
}

// Full-rank block k, column-major m x n (scalar units).
int ref_fr_block(void *h, int64_t k, double *out) {
  const auto &fr = H(h)->io->getHmat()->get_full_rank_blocks();
  if (k < 0 || k >= (int64_t)fr.size()) return 1;
  copy_colmajor(*fr[k], out);
  return 0;
}

// Low-rank block k: A (m x r) and B (r x n), both column-major (LowRank.h:18-24).
int ref_lr_block(void *h, int64_t k, double *A, double *B) {
  const auto &lr = H(h)->io->getHmat()->get_low_rank_blocks();
  if (k < 0 || k >= (int64_t)lr.size()) return 1;
  copy_colmajor(lr[k]->A, A);
  copy_colmajor(lr[k]->B, B);
  return 0;
}

// BigWhamIO::MatVec in the original dof ordering (bigwham_io.cc:927-933).
int ref_matvec(void *h, const double *x, double *y) {
  const int64_t n = H(h)->io->getHmat()->size(1);
  il::ArrayView<double> xv{x, n};
  il::Array<double> out = H(h)->io->MatVec(xv);
  std::memcpy(y, out.data(), sizeof(double) * out.size());
  return 0;
}

// BigWhamIO::MatVecPerm in the permuted ordering (bigwham_io.cc:965-980).
int ref_matvec_perm(void *h, const double *x, double *y) {
  const int64_t n = H(h)->io->getHmat()->size(1);
  il::ArrayView<double> xv{x, n};
  il::Array<double> out = H(h)->io->MatVecPerm(xv);
  std::memcpy(y, out.data(), sizeof(double) * out.size());
  return 0;
}

// Sub-matrix selection: BigWhamIO::hmatSelection (bigwham_io.cc:1365-1375)
// wraps the built Hmat in an HmatSelection (hmat_selection.cc); element
// indices rows / cols in the original ordering.  y = the selection's MatVec
// (matvecOriginal, hmat_selection.cc:230-258), length n_rows * dof.
// Returns 1 when the reference rejects the indices (validateIndices throws).
int ref_selection_matvec(void *h, const int *rows, int64_t n_rows, const int *cols, int64_t n_cols,
                         const double *x, double *y) {
  try {
    il::Array<int> r(n_rows), c(n_cols);
    for (int64_t i = 0; i < n_rows; i++) r[i] = rows[i];
    for (int64_t i = 0; i < n_cols; i++) c[i] = cols[i];
    BigWhamIO sel = H(h)->io->hmatSelection(r, c);
    il::ArrayView<double> xv{x, sel.getHmat()->size(1)};
    il::Array<double> out = sel.MatVec(xv);
    std::memcpy(y, out.data(), sizeof(double) * out.size());
    return 0;
  } catch (...) {
    return 1;
  }
}

// The selection's full-block entries through BigWhamIO::GetFullBlocks
// (HmatSelection::fullBlocksOriginal, hmat_selection.cc:265-375):
// val[i] = H_sel(pos[2i], pos[2i + 1]).  Returns the entry count (or -1);
// val / pos are written when cap covers it.
int64_t ref_selection_full_blocks(void *h, const int *rows, int64_t n_rows, const int *cols, int64_t n_cols,
                                  double *val, int *pos, int64_t cap) {
  try {
    il::Array<int> r(n_rows), c(n_cols);
    for (int64_t i = 0; i < n_rows; i++) r[i] = rows[i];
    for (int64_t i = 0; i < n_cols; i++) c[i] = cols[i];
    BigWhamIO sel = H(h)->io->hmatSelection(r, c);
    std::vector<double> v;
    std::vector<int> p;
    sel.GetFullBlocks(v, p);
    const int64_t n = (int64_t)v.size();
    if (val && pos && cap >= n) {
      std::memcpy(val, v.data(), sizeof(double) * n);
      std::memcpy(pos, p.data(), sizeof(int) * 2 * n);
    }
    return n;
  } catch (...) {
    return -1;
  }
}

// Gaussian-matrix H-build as the reference's own test makes it
// (src/hmat/hmatrix/_test/Hmat_test_gaussian_mat.cpp:44-71): n points on a
// line at x = i, cluster(leaf), hmatrixTreeIxI(eta), createPattern,
// GaussianMatrix(n, alpha), Hmat(M, eps, threads).  permutation_1_ is left
// unset there; it is set here to permutation_0_ (a square, self-interaction
// matrix) so that the original-order products exist.
void *ref_gaussian_create(int64_t n, double alpha, int leaf, double eta, double eps, int n_threads) {
  try {
    il::Array2D<double> points{n, 1, 0.0};
    for (il::int_t i = 0; i < n; i++) points(i, 0) = 1.0 * i;
    bigwham::Cluster cl = bigwham::cluster(leaf, il::io, points);
    const il::Tree<bigwham::SubHMatrix, 4> tree = bigwham::hmatrixTreeIxI(points, cl.partition, eta);
    auto *g = new RefGauss;
    g->hr = std::make_shared<bigwham::HRepresentation>();
    g->hr->pattern_ = bigwham::createPattern(tree);
    g->hr->permutation_0_ = cl.permutation;
    g->hr->permutation_1_ = cl.permutation;
    bigwham::GaussianMatrix<double> M{n, alpha, g->hr};
    g->h.reset(new bigwham::Hmat<double>(M, eps, n_threads, false));
    return g;
  } catch (...) {
    return nullptr;
  }
}

// sizes[4] = (FR blocks, LR blocks, FR entries, LR entries A then B).
int ref_gaussian_sizes(void *h, int64_t *sizes) {
  auto p = GS(h)->h->pattern();
  sizes[0] = p.n_FRB;
  sizes[1] = p.n_LRB;
  sizes[2] = sizes[3] = 0;
  for (const auto &b : GS(h)->h->get_full_rank_blocks()) sizes[2] += b->size(0) * b->size(1);
  for (const auto &b : GS(h)->h->get_low_rank_blocks()) sizes[3] += b->A.size(0) * b->A.size(1) + b->B.size(0) * b->B.size(1);
  return 0;
}

// The flat form: fr n_FR x 4, lr n_LR x 5 (rank in scalar columns), blocks
// column-major back to back (LR: A then B), the permutation.
int ref_gaussian_export(void *h, int64_t *fr, int64_t *lr, double *fr_data, double *lr_data, int64_t *perm) {
  auto *g = GS(h);
  auto p = g->h->pattern();
  for (il::int_t k = 0; k < p.n_FRB; k++)
    for (int r = 0; r < 4; r++) fr[4 * k + r] = p.FRB_pattern(r + 1, k);
  for (il::int_t k = 0; k < p.n_LRB; k++)
    for (int r = 0; r < 5; r++) lr[5 * k + r] = p.LRB_pattern(r + 1, k);
  int64_t o = 0;
  for (const auto &b : g->h->get_full_rank_blocks()) {
    copy_colmajor(*b, fr_data + o);
    o += b->size(0) * b->size(1);
  }
  o = 0;
  for (const auto &b : g->h->get_low_rank_blocks()) {
    copy_colmajor(b->A, lr_data + o);
    o += b->A.size(0) * b->A.size(1);
    copy_colmajor(b->B, lr_data + o);
    o += b->B.size(0) * b->B.size(1);
  }
  for (il::int_t i = 0; i < g->hr->permutation_0_.size(); i++) perm[i] = g->hr->permutation_0_[i];
  return 0;
}

// Hmat::matvec (permuted ordering, hmat.cc:472-537) and Hmat::diagonal
// (permuted ordering, hmat.cc:240-255).
int ref_gaussian_matvec_perm(void *h, const double *x, double *y) {
  const int64_t n = GS(h)->h->size(1);
  il::ArrayView<double> xv{x, n};
  il::Array<double> out = GS(h)->h->matvec(xv);
  std::memcpy(y, out.data(), sizeof(double) * out.size());
  return 0;
}

int ref_gaussian_diagonal(void *h, double *d) {
  std::vector<double> v = GS(h)->h->diagonal();
  std::memcpy(d, v.data(), sizeof(double) * v.size());
  return 0;
}

void ref_gaussian_destroy(void *h) { delete GS(h); }

// BigWhamIO::GetDiagonal, original ordering (bigwham_io.cc:909-916).
int ref_diagonal(void *h, double *d) {
  std::vector<double> v;
  H(h)->io->GetDiagonal(v);
  std::memcpy(d, v.data(), sizeof(double) * v.size());
  return 0;
}

// Rows of the DENSE FP64 operator (no H-matrix approximation) for the given
// collocation points, in the original ordering: out is (npts * dof) x
// (n_points * dof), row-major; row q*dof + a, column j*dof + b holds the
// influence of source point j's component b on receiver point points[q]'s
// component a.  The kernel is built as BigWhamIO builds it for the same
// kernel string (src/io/bigwham_io.cc:130-290) and evaluated entry by entry as
// the reference's BieMatrixGenerator::set does (src/hmat/bie_matrix_generator.h:
// 96-147), over the handle's own mesh.  Kernels: 2DS0-H, 3DR0-H, 3DT0-H.
int ref_dense_rows(void *h, const char *kernel, const double *props, const int64_t *points, int64_t npts,
                   double *out) {
  try {
    const std::shared_ptr<bigwham::Mesh> mesh = H(h)->io->GetSourceMeshPtr();
    bigwham::ElasticProperties elas(props[0], props[1]);
    std::shared_ptr<bigwham::BieKernel<double>> ker;
    const std::string k(kernel);
    if (k == "2DS0-H")
      ker = std::make_shared<bigwham::BieElastostatic<bigwham::Segment<0>, bigwham::Segment<0>,
                                                      bigwham::ElasticKernelType::H>>(elas, 2);
    else if (k == "3DR0-H")
      ker = std::make_shared<bigwham::BieElastostatic<bigwham::Rectangle<0>, bigwham::Rectangle<0>,
                                                      bigwham::ElasticKernelType::H>>(elas, 3);
    else if (k == "3DT0-H")
      ker = std::make_shared<bigwham::BieElastostatic<bigwham::Triangle<0>, bigwham::Triangle<0>,
                                                      bigwham::ElasticKernelType::H>>(elas, 3);
    else
      return 1;
    const int dof = (int)ker->dof_dimension();
    const int64_t np = mesh->num_collocation_points();
    const int64_t ncols = np * dof;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < npts; q++) {
      const int64_t i = points[q];
      if (i < 0 || i >= np) {
#pragma omp atomic write
        bad = 1;
        continue;
      }
      const auto re = mesh->GetElement(mesh->GetElementId(i));
      const il::int_t ir = mesh->GetElementCollocationId(i);
      for (int64_t j = 0; j < np; j++) {
        const auto se = mesh->GetElement(mesh->GetElementId(j));
        const std::vector<double> st = ker->influence(*se, mesh->GetElementCollocationId(j), *re, ir);
        for (int b = 0; b < dof; b++)
          for (int a = 0; a < dof; a++) out[(q * dof + a) * ncols + j * dof + b] = st[b * dof + a];
      }
    }
    return bad ? 2 : 0;
  } catch (...) {
    return 3;
  }
}

// Collocation points, flattened row-major (n_points x spatial_dim).
int64_t ref_collocation_points(void *h, double *out) {
  std::vector<double> v = H(h)->io->GetCollocationPoints();
  if (out) std::memcpy(out, v.data(), sizeof(double) * v.size());
  return (int64_t)v.size();
}

void ref_destroy(void *h) { delete H(h); }

// Per element of the handle's (source) mesh, 15 values: collocation point
// (3), rotation matrix row-major (9; local = R global, BoundaryElement::
// ConvertToLocal) and unit normal (3), as the reference's elements hold them
// (BigWhamIO::GetCollocationPoints / GetRotationMatrix / GetElementNormals,
// src/io/bigwham_io.cc:985-1140).  One collocation point per element only.
int ref_element_frames(void *h, double *out) {
  try {
    BigWhamIO &io = *H(h)->io;
    const std::vector<double> cp = io.GetCollocationPoints(), rot = io.GetRotationMatrix(),
                              nrm = io.GetElementNormals();
    const size_t ne = nrm.size() / 3;
    if (cp.size() != 3 * ne || rot.size() != 9 * ne) return 1;
    for (size_t e = 0; e < ne; e++) {
      for (int k = 0; k < 3; k++) out[15 * e + k] = cp[3 * e + k];
      for (int k = 0; k < 9; k++) out[15 * e + 3 + k] = rot[9 * e + k];
      for (int k = 0; k < 3; k++) out[15 * e + 12 + k] = nrm[3 * e + k];
    }
    return 0;
  } catch (...) {
    return 3;
  }
}

// The reference's rectangular (3DR0) point kernels, for checking a
// restatement of them: stresses at (x, y, z) in the local frame of a
// [-a, a] x [-b, b] rectangle at z = 0 carrying unit displacement
// discontinuities (StressesKernelR0, elastic_3dR0_element.h), out[6 * dd + c]
// with c = xx, yy, zz, xy, xz, yz; displacements (DisplacementKernelR0),
// out[3 * i + j] = entry (i, j) of the reference's 3 x 3 array.
int ref_r0_stress(double x, double y, double z, double a, double b, double G, double nu, double *out) {
  try {
    il::StaticArray2D<double, 3, 6> s = bigwham::StressesKernelR0(x, y, z, a, b, G, nu);
    for (int i = 0; i < 3; i++)
      for (int c = 0; c < 6; c++) out[6 * i + c] = s(i, c);
    return 0;
  } catch (...) {
    return 3;
  }
}

int ref_r0_displacement(double x, double y, double z, double a, double b, double nu, double *out) {
  try {
    il::Array2D<double> u = bigwham::DisplacementKernelR0(x, y, z, a, b, nu);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) out[3 * i + j] = u(i, j);
    return 0;
  } catch (...) {
    return 3;
  }
}

}  // extern "C"
