// HmatGpu implementation (see hmat_gpu.h).
#include "hmat_gpu.h"

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

namespace bigwham_b200 {

void HmatGpu::check(int status, const char *what) const {
  if (status == BW_OK) return;
  char buf[512];
  bw_last_error(h_, buf, sizeof buf);
  throw std::runtime_error(std::string("bigwham_b200: ") + what + " failed (" + std::to_string(status) + "): " + buf);
}

HmatGpu::HmatGpu(const std::shared_ptr<bigwham::Hmat<double>> &cpu, int device, int storage,
                 const std::vector<std::pair<std::string, int64_t>> &tuning) {
  if (!cpu || !cpu->isBuilt()) throw std::runtime_error("bigwham_b200: HmatGpu needs a built Hmat");
  // Base-class state read through the public getters (hmat.h:108-121).
  hr_ = cpu->get_hr();
  dof_dimension_ = cpu->get_dof_dimension();
  size_ = cpu->get_size();
  n_openMP_threads_ = cpu->get_n_openMP_threads();
  verbose_ = cpu->get_verbose();
  fixed_rank_ = cpu->get_fixed_rank();
  full_rank_blocks_ = cpu->get_full_rank_blocks();  // shared storage, kept for fullBlocksOriginal
  // LowRank shells that keep only the ACA error estimate (GetHPattern /
  // GetMaxErrorACA read it, bigwham_io.cc:707-784); A and B live on the GPU.
  const auto &lrs = cpu->get_low_rank_blocks();
  low_rank_blocks_.resize(lrs.size());
  for (size_t k = 0; k < lrs.size(); k++) {
    low_rank_blocks_[k] = std::make_unique<bigwham::LowRank<double>>();
    low_rank_blocks_[k]->error_on_approximation = lrs[k]->error_on_approximation;
  }

  const il::int_t dof = dof_dimension_;
  std::vector<int64_t> p0(hr_->permutation_0_.size()), p1(hr_->permutation_1_.size());
  for (size_t i = 0; i < p0.size(); i++) p0[i] = hr_->permutation_0_[(il::int_t)i];
  for (size_t i = 0; i < p1.size(); i++) p1[i] = hr_->permutation_1_[(il::int_t)i];
  int st = bw_create((int)dof, size_[0], size_[1], p0.data(), p1.data(), device, &h_);
  if (st != BW_OK) {
    char buf[512];
    bw_last_error(nullptr, buf, sizeof buf);
    throw std::runtime_error(std::string("bigwham_b200: bw_create failed: ") + buf);
  }
  try {
    for (const auto &kv : tuning) check(bw_set_tuning(h_, kv.first.c_str(), kv.second), "bw_set_tuning");
    const bigwham::HPattern &pat = hr_->pattern_;
    // FR blocks (hmat.cc:315-353 builds them; pattern rows 1..4 in points)
    for (il::int_t k = 0; k < pat.n_FRB; k++) {
      const il::Array2D<double> &a = *full_rank_blocks_[(size_t)k];
      check(bw_add_full(h_, pat.FRB_pattern(1, k) * dof, pat.FRB_pattern(2, k) * dof, a.size(0), a.size(1),
                        a.data(), a.capacity(0)),
            "bw_add_full");
      entries_ += a.size(0) * a.size(1);
    }
    // LR blocks: y += A (B x) with A m x r, B r x n (hmat.cc:510-527)
    for (il::int_t k = 0; k < pat.n_LRB; k++) {
      const bigwham::LowRank<double> &lr = *lrs[(size_t)k];
      check(bw_add_lowrank(h_, pat.LRB_pattern(1, k) * dof, pat.LRB_pattern(2, k) * dof, lr.A.size(0), lr.B.size(1),
                           lr.A.size(1), lr.A.data(), std::max<il::int_t>(1, lr.A.capacity(0)), lr.B.data(),
                           std::max<il::int_t>(1, lr.B.capacity(0))),
            "bw_add_lowrank");
      entries_ += lr.A.size(0) * lr.A.size(1) + lr.B.size(0) * lr.B.size(1);
    }
    check(bw_finalize(h_, storage), "bw_finalize");
  } catch (...) {
    bw_destroy(h_);
    h_ = nullptr;
    throw;
  }
  if (storage & BW_FP64)
    precision_ = BW_FP64;
  else if (storage & BW_FP32)
    precision_ = BW_FP32;
  else
    precision_ = BW_BF16;
  isBuilt_FR_ = isBuilt_LR_ = isBuilt_ = true;
}

HmatGpu::HmatGpu(const std::string &filename, int device, int storage,
                 const std::vector<std::pair<std::string, int64_t>> &tuning) {
  const char *path = filename.c_str();
  int64_t info[9];
  check(bw_file_info(path, info), "bw_file_info");
  const il::int_t dof = info[0], nfr = info[3], nlr = info[4];
  dof_dimension_ = dof;
  size_[0] = info[1];
  size_[1] = info[2];
  // Host side: pattern, permutations, FR blocks and ACA estimates (the LR
  // factors are left in the file; they only live on the GPU).
  std::vector<int64_t> fr(4 * nfr), lr(5 * nlr), frp(6 * nfr), lrp(6 * nlr), p0(info[1] / dof), p1(info[2] / dof);
  std::vector<double> frd(info[5]), err(nlr);
  check(bw_file_read(path, 0, fr.data(), lr.data(), frd.data(), nullptr, p0.data(), p1.data(), err.data(),
                     frp.data(), lrp.data()),
        "bw_file_read");
  hr_ = std::make_shared<bigwham::HRepresentation>();
  hr_->is_square_ = size_[0] == size_[1];
  bigwham::HPattern &pat = hr_->pattern_;
  pat.n_FRB = nfr;
  pat.n_LRB = nlr;
  pat.n_B = nfr + nlr;
  pat.FRB_pattern = il::Array2D<il::int_t>(6, nfr);
  pat.LRB_pattern = il::Array2D<il::int_t>(6, nlr);
  for (il::int_t k = 0; k < nfr; k++)
    for (int r = 0; r < 6; r++) pat.FRB_pattern(r, k) = frp[6 * k + r];
  for (il::int_t k = 0; k < nlr; k++)
    for (int r = 0; r < 6; r++) pat.LRB_pattern(r, k) = lrp[6 * k + r];
  hr_->permutation_0_ = il::Array<il::int_t>((il::int_t)p0.size());
  hr_->permutation_1_ = il::Array<il::int_t>((il::int_t)p1.size());
  for (size_t i = 0; i < p0.size(); i++) hr_->permutation_0_[(il::int_t)i] = p0[i];
  for (size_t i = 0; i < p1.size(); i++) hr_->permutation_1_[(il::int_t)i] = p1[i];
  full_rank_blocks_.resize((size_t)nfr);
  int64_t o = 0;
  for (il::int_t k = 0; k < nfr; k++) {
    const il::int_t m = (frp[6 * k + 3] - frp[6 * k + 1]) * dof, n = (frp[6 * k + 4] - frp[6 * k + 2]) * dof;
    auto a = std::make_shared<il::Array2D<double>>(m, n);
    for (il::int_t j = 0; j < n; j++)
      std::memcpy(a->Data() + j * a->capacity(0), frd.data() + o + j * m, sizeof(double) * (size_t)m);
    o += m * n;
    full_rank_blocks_[(size_t)k] = a;
  }
  low_rank_blocks_.resize((size_t)nlr);
  for (il::int_t k = 0; k < nlr; k++) {
    low_rank_blocks_[(size_t)k] = std::make_unique<bigwham::LowRank<double>>();
    low_rank_blocks_[(size_t)k]->error_on_approximation = err[(size_t)k];
  }
  entries_ = info[5] + info[6];
  // Device side: blocks registered from the mapped file, then laid out.
  check(bw_create_from_file(path, device, 1, &h_), "bw_create_from_file");
  try {
    for (const auto &kv : tuning) check(bw_set_tuning(h_, kv.first.c_str(), kv.second), "bw_set_tuning");
    check(bw_finalize(h_, storage), "bw_finalize");
  } catch (...) {
    bw_destroy(h_);
    h_ = nullptr;
    throw;
  }
  precision_ = (storage & BW_FP64) ? BW_FP64 : (storage & BW_FP32) ? BW_FP32 : BW_BF16;
  isBuilt_FR_ = isBuilt_LR_ = isBuilt_ = true;
}

void write_block_file(const bigwham::Hmat<double> &hm, const std::string &filename) {
  if (!hm.isBuilt()) throw std::runtime_error("bigwham_b200: write_block_file needs a built Hmat");
  auto hr = hm.get_hr();
  const bigwham::HPattern &p = hr->pattern_;
  const auto &frs = hm.get_full_rank_blocks();
  const auto &lrs = hm.get_low_rank_blocks();
  const il::int_t dof = hm.get_dof_dimension();
  if ((il::int_t)frs.size() != p.n_FRB || (il::int_t)lrs.size() != p.n_LRB)
    throw std::runtime_error("bigwham_b200: write_block_file: the Hmat holds no host blocks (an HmatGpu?)");
  std::vector<int64_t> frp(6 * p.n_FRB), lrp(6 * p.n_LRB), fld(p.n_FRB), ald(p.n_LRB), bld(p.n_LRB);
  std::vector<const double *> fb(p.n_FRB), ab(p.n_LRB), bb(p.n_LRB);
  std::vector<double> err(p.n_LRB);
  for (il::int_t k = 0; k < p.n_FRB; k++) {
    for (int r = 0; r < 6; r++) frp[6 * k + r] = p.FRB_pattern(r, k);
    const il::Array2D<double> &a = *frs[(size_t)k];
    if (a.size(0) != (p.FRB_pattern(3, k) - p.FRB_pattern(1, k)) * dof ||
        a.size(1) != (p.FRB_pattern(4, k) - p.FRB_pattern(2, k)) * dof)
      throw std::runtime_error("bigwham_b200: FR block " + std::to_string(k) + " disagrees with its pattern");
    fb[k] = a.data();
    fld[k] = std::max<il::int_t>(1, a.capacity(0));
  }
  for (il::int_t k = 0; k < p.n_LRB; k++) {
    for (int r = 0; r < 6; r++) lrp[6 * k + r] = p.LRB_pattern(r, k);
    if (!lrs[(size_t)k]) throw std::runtime_error("bigwham_b200: missing LR block " + std::to_string(k));
    const bigwham::LowRank<double> &lr = *lrs[(size_t)k];
    const il::int_t rank = lr.A.size(1);
    if (rank != p.LRB_pattern(5, k) || lr.B.size(0) != rank ||
        lr.A.size(0) != (p.LRB_pattern(3, k) - p.LRB_pattern(1, k)) * dof ||
        lr.B.size(1) != (p.LRB_pattern(4, k) - p.LRB_pattern(2, k)) * dof)
      throw std::runtime_error("bigwham_b200: LR block " + std::to_string(k) + " disagrees with its pattern");
    ab[k] = lr.A.data();
    ald[k] = std::max<il::int_t>(1, lr.A.capacity(0));
    bb[k] = lr.B.data();
    bld[k] = std::max<il::int_t>(1, lr.B.capacity(0));
    err[k] = lr.error_on_approximation;
  }
  std::vector<int64_t> p0(hr->permutation_0_.size()), p1(hr->permutation_1_.size());
  for (size_t i = 0; i < p0.size(); i++) p0[i] = hr->permutation_0_[(il::int_t)i];
  for (size_t i = 0; i < p1.size(); i++) p1[i] = hr->permutation_1_[(il::int_t)i];
  const auto size = hm.get_size();
  const int st = bw_file_write_blocks(filename.c_str(), (int)dof, size[0], size[1], p0.data(), p1.data(), p.n_FRB,
                                      frp.data(), fb.data(), fld.data(), p.n_LRB, lrp.data(), ab.data(), ald.data(),
                                      bb.data(), bld.data(), err.data());
  if (st != BW_OK) {
    char buf[512];
    bw_last_error(nullptr, buf, sizeof buf);
    throw std::runtime_error(std::string("bigwham_b200: write_block_file: ") + buf);
  }
}

HmatGpu::~HmatGpu() { bw_destroy(h_); }

void HmatGpu::matvec(double *x, double *y) {
  check(bw_matvec(h_, x, y, precision_ | BW_PERMUTED, nullptr), "bw_matvec");
  check(bw_sync(h_, nullptr), "bw_sync");
}

void HmatGpu::matvecOriginal(double *x, double *y) {
  check(bw_matvec(h_, x, y, precision_, nullptr), "bw_matvec");
  check(bw_sync(h_, nullptr), "bw_sync");
}

il::Array<double> HmatGpu::matvec(il::ArrayView<double> x) {
  if (x.size() != size_[1]) throw std::runtime_error("bigwham_b200: x has the wrong size");
  il::Array<double> y(size_[0]);
  check(bw_matvec_host(h_, x.data(), y.Data(), precision_ | BW_PERMUTED), "bw_matvec_host");
  return y;
}

il::Array<double> HmatGpu::matvecOriginal(il::ArrayView<double> x) {
  if (x.size() != size_[1]) throw std::runtime_error("bigwham_b200: x has the wrong size");
  il::Array<double> y(size_[0]);
  check(bw_matvec_host(h_, x.data(), y.Data(), precision_), "bw_matvec_host");
  return y;
}

void HmatGpu::matvecInto(const double *x, double *y) {
  check(bw_matvec_host(h_, x, y, precision_ | BW_PERMUTED), "bw_matvec_host");
}

void HmatGpu::matvecOriginalInto(const double *x, double *y) {
  check(bw_matvec_host(h_, x, y, precision_), "bw_matvec_host");
}

std::vector<double> HmatGpu::diagonal() {
  std::vector<double> d((size_t)std::max(size_[0], size_[1]));
  check(bw_diagonal(h_, d.data(), BW_PERMUTED), "bw_diagonal");
  return d;
}

std::vector<double> HmatGpu::diagonalOriginal() {
  std::vector<double> d((size_t)std::max(size_[0], size_[1]));
  check(bw_diagonal(h_, d.data(), 0), "bw_diagonal");
  return d;
}

il::int_t HmatGpu::nbOfEntries() { return entries_; }

}  // namespace bigwham_b200
