// HmatGpu: the B200 backend behind the reference's own Hmat interface.
//
// A BigWham user builds the H-matrix as usual (BigWhamIO ctor +
// BuildHierarchicalMatrix, src/io/bigwham_io.cc:41-290, :635-704), then
//
//   auto gpu = std::make_shared<bigwham_b200::HmatGpu>(io.getHmat(), 0, BW_FP64);
//   io.setHmat(gpu);                                  // src/io/bigwham_io.h:206
//
// after which every matvec entry of BigWhamIO (MatVec host and device-pointer
// overloads, MatVecVoid, MatVecPerm: bigwham_io.cc:919-980) and the pybind11
// matvec_raw_ptr (interfaces/python/py_bigwham.cc:213-222) run on the GPU.
// The overridden virtuals are the ones Hmat declares for this purpose
// (src/hmat/hmatrix/hmat.h:76-95).  The upload reads the built blocks through
// the public getters (hmat.h:108-121); nothing in the reference is edited.
#pragma once

#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "bigwham_b200.h"
#include "hmat/hmatrix/hmat.h"

namespace bigwham_b200 {

class HmatGpu : public bigwham::Hmat<double> {
 public:
  // storage: BW_FP64 | BW_FP32 | BW_BF16 (+ BW_STORE_TRANSPOSE).  Throws
  // std::runtime_error when the upload fails.
  // tuning: plan parameters passed to bw_set_tuning before bw_finalize.
  HmatGpu(const std::shared_ptr<bigwham::Hmat<double>> &cpu, int device, int storage,
          const std::vector<std::pair<std::string, int64_t>> &tuning = {});
  // From a block file written by write_block_file (or bw_file_write): the
  // counterpart of the reference's Hmat(filename) constructor
  // (src/hmat/hmatrix/hmat.cc:64-74, readFromFile :837-935), without HDF5.
  // The device blocks are uploaded straight from the mapped file (checksums
  // verified); the pattern, permutations, FR blocks (for fullBlocksOriginal)
  // and ACA error estimates are restored on the host.
  HmatGpu(const std::string &filename, int device, int storage,
          const std::vector<std::pair<std::string, int64_t>> &tuning = {});
  ~HmatGpu() override;
  HmatGpu(const HmatGpu &) = delete;
  HmatGpu &operator=(const HmatGpu &) = delete;

  // Device pointers, permuted / original ordering; return once y is complete
  // (the reference's HmatCuda synchronizes the device inside these calls).
  void matvec(double *x, double *y) override;
  void matvecOriginal(double *x, double *y) override;
  // Host arrays (BigWhamIO::MatVec(ArrayView), MatVecPerm, MatVecVoid).
  il::Array<double> matvec(il::ArrayView<double> x) override;
  il::Array<double> matvecOriginal(il::ArrayView<double> x) override;
  // The same products into a caller's host array y of size(0) values.
  void matvecInto(const double *x, double *y);
  void matvecOriginalInto(const double *x, double *y);

  std::vector<double> diagonal() override;
  std::vector<double> diagonalOriginal() override;
  il::int_t nbOfEntries() override;

  // Precision used by the overrides above (BW_FP64 by default).
  void set_precision(int bw_precision) { precision_ = bw_precision; }
  int precision() const { return precision_; }
  bw_hmat *handle() const { return h_; }

 private:
  void check(int status, const char *what) const;
  bw_hmat *h_ = nullptr;
  int precision_ = BW_FP64;
  il::int_t entries_ = 0;
};

// Save a built Hmat as a block file: the content of the reference's
// Hmat::writeToFile (src/hmat/hmatrix/hmat.cc:749-835), without HDF5
// (bw_file_write_blocks; the file is written whole or not at all).  Works
// for a CPU Hmat before it is replaced by an HmatGpu.  Throws
// std::runtime_error on failure.
void write_block_file(const bigwham::Hmat<double> &hmat, const std::string &filename);

}  // namespace bigwham_b200
