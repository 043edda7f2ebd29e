// Block files: a built H-matrix on disk, in a form the backend maps and
// uploads without the host rebuild.
//
// Content is what the reference's Hmat<T>::writeToFile stores in HDF5
// (src/hmat/hmatrix/hmat.cc:749-835, read back by readFromFile :837-935 and
// the Hmat(filename) constructor :64-74), i.e. dof, matrix sizes, the
// HPattern columns of both block kinds, both permutations, every full-rank
// block and every low-rank block's A and B, plus the low-rank blocks' ACA
// error estimates.  The reference needs HDF5 for it; this format is a flat,
// page-aligned binary that is read by mmap, so registering the blocks copies
// nothing and the upload streams straight from the page cache.
//
// Layout (little-endian):
//   [0, 256)    FileHeader
//   sections    each starting at a multiple of 4096 bytes, zero padding between:
//     perm0       int64 [n_rows / dof]        permutation_0_ (rows)
//     perm1       int64 [n_cols / dof]        permutation_1_ (cols)
//     fr_pattern  int64 [n_fr][6]             HPattern column per FR block:
//     lr_pattern  int64 [n_lr][6]               spot, i0, j0, i_end, j_end, flag
//                                               (points; flag 0 for FR, the
//                                               rank in scalar columns for LR)
//     lr_error    double [n_lr]               LowRank::error_on_approximation
//                                               (bytes 0 when not stored)
//     fr_data     double [fr_entries]         FR blocks back to back, column-major
//     lr_data     double [lr_entries]         per LR block: A (m x r) then B (r x n),
//                                               column-major
// Each section carries a 64-bit checksum of its bytes, and the header one of
// its own; readers check the header always and the sections on request.
#pragma once

#include <cstdint>
#include <memory>
#include <string>

namespace bw {

constexpr uint32_t kFileVersion = 1;
constexpr int64_t kFileAlign = 4096;
constexpr int64_t kHashBlockWords = 1 << 17;  // 1 MiB of 8-byte words per checksum block

enum FileSection { kSecPerm0 = 0, kSecPerm1, kSecFrPattern, kSecLrPattern, kSecLrError, kSecFrData, kSecLrData, kNumSections };

struct FileSectionRec {
  int64_t offset;
  int64_t bytes;
  uint64_t hash;
};

struct FileHeader {
  char magic[8];  // "BWBLOCKS"
  uint32_t version;
  uint32_t header_bytes;  // sizeof(FileHeader)
  int64_t dof, n_rows, n_cols;
  int64_t n_fr, n_lr;
  int64_t fr_entries, lr_entries;
  int64_t flags;  // bit 0: lr_error stored
  FileSectionRec sec[kNumSections];
  uint64_t header_hash;  // checksum of every byte before this field
};
static_assert(sizeof(FileHeader) == 256, "FileHeader is 256 bytes on disk");

constexpr int64_t kFileHasLrError = 1;

// What write_block_file stores: pattern columns in HPattern order and, per
// block, a column-major pointer with its leading dimension (>= rows).
struct FileBlocks {
  int dof = 1;
  int64_t n_rows = 0, n_cols = 0;
  const int64_t *perm0 = nullptr, *perm1 = nullptr;
  int64_t n_fr = 0;
  const int64_t *fr_pattern = nullptr;  // n_fr x 6
  const double *const *fr = nullptr;
  const int64_t *fr_ld = nullptr;
  int64_t n_lr = 0;
  const int64_t *lr_pattern = nullptr;  // n_lr x 6
  const double *const *lr_a = nullptr;
  const int64_t *lr_a_ld = nullptr;
  const double *const *lr_b = nullptr;
  const int64_t *lr_b_ld = nullptr;
  const double *lr_error = nullptr;  // n_lr values or null
};

// Checks the pattern against the sizes (std::invalid_argument), then writes
// `path` through a temporary file renamed into place, so a reader never sees
// a partial file (std::runtime_error on I/O failure).
void write_block_file(const std::string &path, const FileBlocks &b);

// Checksum of a section: 8-byte words in blocks of kHashBlockWords, the
// blocks hashed in parallel and folded in order.
uint64_t section_hash(const void *data, int64_t bytes);

// A mapped block file.  open() checks the magic, version, header checksum,
// section bounds and sizes, and the pattern (blocks inside the matrix, entry
// counts equal to the data sections); with verify it also checks every
// section's checksum.  Errors: std::runtime_error naming the file
// (unreadable, not a block file, truncated, inconsistent or failing a
// checksum).
class BlockFile {
 public:
  static std::shared_ptr<BlockFile> open(const std::string &path, bool verify);
  ~BlockFile();
  BlockFile(const BlockFile &) = delete;
  BlockFile &operator=(const BlockFile &) = delete;

  const FileHeader &header() const { return *reinterpret_cast<const FileHeader *>(base_); }
  const void *section(FileSection s) const {
    return static_cast<const unsigned char *>(base_) + header().sec[s].offset;
  }
  const int64_t *perm0() const { return static_cast<const int64_t *>(section(kSecPerm0)); }
  const int64_t *perm1() const { return static_cast<const int64_t *>(section(kSecPerm1)); }
  const int64_t *fr_pattern() const { return static_cast<const int64_t *>(section(kSecFrPattern)); }
  const int64_t *lr_pattern() const { return static_cast<const int64_t *>(section(kSecLrPattern)); }
  const double *lr_error() const {
    return (header().flags & kFileHasLrError) ? static_cast<const double *>(section(kSecLrError)) : nullptr;
  }
  const double *fr_data() const { return static_cast<const double *>(section(kSecFrData)); }
  const double *lr_data() const { return static_cast<const double *>(section(kSecLrData)); }
  int64_t file_bytes() const { return static_cast<int64_t>(size_); }

 private:
  BlockFile() = default;
  void validate(const std::string &path, bool verify) const;
  void *base_ = nullptr;
  size_t size_ = 0;
};

}  // namespace bw
