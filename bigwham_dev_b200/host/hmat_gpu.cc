// HmatGpu implementation (see hmat_gpu.h).
#include "hmat_gpu.h"

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
