// Block files: writer, checksum and mapped reader (format in bw_file.h).
#include "bw_file.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>

namespace bw {
namespace {

constexpr char kMagic[8] = {'B', 'W', 'B', 'L', 'O', 'C', 'K', 'S'};
constexpr uint64_t kSeed = 0x42574C4F434B5331ull;  // "BWLOCKS1"
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;
constexpr int64_t kMaxSide = int64_t(1) << 31;  // the backend indexes rows and columns with 32-bit ints
const char *const kSectionName[kNumSections] = {"perm0", "perm1", "fr_pattern", "lr_pattern",
                                                "lr_error", "fr_data", "lr_data"};

// splitmix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): the output function as a 64-bit mixer.
inline uint64_t mix64(uint64_t x) {
  x += kGolden;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

inline uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

// One checksum block: four independent lanes (word i goes to lane i mod 4),
// each a multiply-rotate chain, mixed together at the end with the count.
struct BlockState {
  uint64_t s[4];
  int64_t n = 0;
  explicit BlockState(int64_t block) {
    for (int i = 0; i < 4; i++) s[i] = mix64(kSeed + 4 * static_cast<uint64_t>(block) + i);
  }
  void add(uint64_t w) {
    uint64_t &l = s[n & 3];
    l = rotl(l ^ (w * kGolden), 31) * 0xBF58476D1CE4E5B9ull;
    n++;
  }
  void add4(const uint64_t *w) {  // n is a multiple of 4
    for (int i = 0; i < 4; i++) s[i] = rotl(s[i] ^ (w[i] * kGolden), 31) * 0xBF58476D1CE4E5B9ull;
    n += 4;
  }
  uint64_t fin() const {
    uint64_t h = mix64(static_cast<uint64_t>(n));
    for (int i = 0; i < 4; i++) h = mix64(h ^ s[i]);
    return h;
  }
};

inline uint64_t fold(uint64_t acc, uint64_t block_hash) { return mix64(acc ^ block_hash); }
inline uint64_t finish(uint64_t acc, int64_t bytes) { return mix64(acc ^ static_cast<uint64_t>(bytes)); }

uint64_t load_word(const unsigned char *p) {
  uint64_t w;
  std::memcpy(&w, p, 8);
  return w;
}

// Streaming form of section_hash for the writer (same blocks, same order).
class StreamHash {
 public:
  void add(const void *data, size_t bytes) {
    const unsigned char *p = static_cast<const unsigned char *>(data);
    for (size_t i = 0; i < bytes; i += 8) {
      st_.add(load_word(p + i));
      if (st_.n == kHashBlockWords) {
        acc_ = fold(acc_, st_.fin());
        st_ = BlockState(++block_);
      }
    }
    bytes_ += static_cast<int64_t>(bytes);
  }
  uint64_t value() const {
    uint64_t a = acc_;
    if (st_.n > 0) a = fold(a, st_.fin());
    return finish(a, bytes_);
  }

 private:
  BlockState st_{0};
  int64_t block_ = 0, bytes_ = 0;
  uint64_t acc_ = kSeed;
};

// Blocks inside the matrix, FR flags 0, LR ranks >= 0; returns the stored
// entries the pattern implies (FR m n, LR r (m + n)).
int64_t pattern_entries(const char *kind, const int64_t *pat, int64_t count, int64_t rows_pts, int64_t cols_pts,
                        int64_t dof, bool lowrank) {
  int64_t e = 0;
  for (int64_t k = 0; k < count; k++) {
    const int64_t *c = pat + 6 * k;
    const int64_t i0 = c[1], j0 = c[2], i1 = c[3], j1 = c[4], flag = c[5];
    if (!(0 <= i0 && i0 < i1 && i1 <= rows_pts && 0 <= j0 && j0 < j1 && j1 <= cols_pts))
      throw std::invalid_argument(std::string(kind) + " block " + std::to_string(k) + " lies outside the matrix");
    const int64_t m = (i1 - i0) * dof, n = (j1 - j0) * dof;  // each < 2^31
    int64_t term;
    if (!lowrank) {
      if (flag != 0) throw std::invalid_argument("FR block " + std::to_string(k) + " has a non-zero pattern flag");
      term = m * n;
    } else {
      if (flag < 0 || flag > kMaxSide / 2)
        throw std::invalid_argument("LR block " + std::to_string(k) + " has a negative or oversized rank");
      term = flag * (m + n);
    }
    if (term > std::numeric_limits<int64_t>::max() - e)
      throw std::invalid_argument(std::string(kind) + " entry count overflows");
    e += term;
  }
  return e;
}

void check_sizes(int64_t dof, int64_t n_rows, int64_t n_cols) {
  if (dof < 1 || dof > 64) throw std::invalid_argument("dof must be in [1, 64]");
  if (n_rows < 0 || n_cols < 0 || n_rows >= kMaxSide || n_cols >= kMaxSide || n_rows % dof || n_cols % dof)
    throw std::invalid_argument("matrix sizes must be non-negative multiples of dof below 2^31");
}

void check_perm(const char *name, const int64_t *p, int64_t n) {
  for (int64_t i = 0; i < n; i++)
    if (p[i] < 0 || p[i] >= n)
      throw std::invalid_argument(std::string(name) + " holds a value outside [0, " + std::to_string(n) + ")");
}

class Writer {
 public:
  explicit Writer(const std::string &tmp) : tmp_(tmp) {
    f_ = std::fopen(tmp.c_str(), "wb");
    if (!f_) fail("cannot create");
    std::setvbuf(f_, nullptr, _IOFBF, 8 << 20);
  }
  ~Writer() {
    if (f_) {
      std::fclose(f_);
      std::remove(tmp_.c_str());
    }
  }
  void put(const void *p, size_t bytes, StreamHash *h) {
    if (bytes && std::fwrite(p, 1, bytes, f_) != bytes) fail("write failed on");
    if (h) h->add(p, bytes);
    pos_ += static_cast<int64_t>(bytes);
  }
  void pad() {
    static const unsigned char zeros[kFileAlign] = {};
    const int64_t r = pos_ % kFileAlign;
    if (r) put(zeros, static_cast<size_t>(kFileAlign - r), nullptr);
  }
  int64_t pos() const { return pos_; }
  void commit(const FileHeader &hdr, const std::string &path) {
    if (std::fseek(f_, 0, SEEK_SET) != 0) fail("seek failed on");
    if (std::fwrite(&hdr, 1, sizeof hdr, f_) != sizeof hdr) fail("write failed on");
    if (std::fflush(f_) != 0 || fsync(fileno(f_)) != 0) fail("flush failed on");
    const int rc = std::fclose(f_);
    f_ = nullptr;
    if (rc != 0) {
      std::remove(tmp_.c_str());
      fail("close failed on");
    }
    if (std::rename(tmp_.c_str(), path.c_str()) != 0) {
      const int e = errno;
      std::remove(tmp_.c_str());
      throw std::runtime_error("cannot rename " + tmp_ + " to " + path + ": " + std::strerror(e));
    }
  }

 private:
  [[noreturn]] void fail(const char *what) {
    throw std::runtime_error(std::string(what) + " " + tmp_ + ": " + std::strerror(errno));
  }
  std::FILE *f_ = nullptr;
  std::string tmp_;
  int64_t pos_ = 0;
};

}  // namespace

uint64_t section_hash(const void *data, int64_t bytes) {
  if (bytes < 0 || bytes % 8) throw std::invalid_argument("section sizes are multiples of 8 bytes");
  const unsigned char *p = static_cast<const unsigned char *>(data);
  const int64_t words = bytes / 8;
  const int64_t nb = (words + kHashBlockWords - 1) / kHashBlockWords;
  std::vector<uint64_t> bh(static_cast<size_t>(nb));
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nb; b++) {
    const int64_t w0 = b * kHashBlockWords, w1 = std::min(words, w0 + kHashBlockWords);
    BlockState st(b);
    int64_t w = w0;
    uint64_t q[4];
    for (; w + 4 <= w1; w += 4) {
      std::memcpy(q, p + 8 * w, 32);
      st.add4(q);
    }
    for (; w < w1; w++) st.add(load_word(p + 8 * w));
    bh[static_cast<size_t>(b)] = st.fin();
  }
  uint64_t acc = kSeed;
  for (int64_t b = 0; b < nb; b++) acc = fold(acc, bh[static_cast<size_t>(b)]);
  return finish(acc, bytes);
}

void write_block_file(const std::string &path, const FileBlocks &b) {
  check_sizes(b.dof, b.n_rows, b.n_cols);
  const int64_t rp = b.n_rows / b.dof, cp = b.n_cols / b.dof;
  if (b.n_fr < 0 || b.n_lr < 0) throw std::invalid_argument("negative block count");
  if ((rp && !b.perm0) || (cp && !b.perm1)) throw std::invalid_argument("null permutation");
  if (b.n_fr && (!b.fr_pattern || !b.fr || !b.fr_ld)) throw std::invalid_argument("null FR pattern or block list");
  if (b.n_lr && (!b.lr_pattern || !b.lr_a || !b.lr_a_ld || !b.lr_b || !b.lr_b_ld))
    throw std::invalid_argument("null LR pattern or factor list");
  check_perm("perm0", b.perm0, rp);
  check_perm("perm1", b.perm1, cp);
  const int64_t fr_entries = pattern_entries("FR", b.fr_pattern, b.n_fr, rp, cp, b.dof, false);
  const int64_t lr_entries = pattern_entries("LR", b.lr_pattern, b.n_lr, rp, cp, b.dof, true);
  for (int64_t k = 0; k < b.n_fr; k++) {
    const int64_t m = (b.fr_pattern[6 * k + 3] - b.fr_pattern[6 * k + 1]) * b.dof;
    if (!b.fr[k] || b.fr_ld[k] < m) throw std::invalid_argument("FR block " + std::to_string(k) + ": null or ld < rows");
  }
  for (int64_t k = 0; k < b.n_lr; k++) {
    const int64_t m = (b.lr_pattern[6 * k + 3] - b.lr_pattern[6 * k + 1]) * b.dof, r = b.lr_pattern[6 * k + 5];
    if (r > 0 && (!b.lr_a[k] || !b.lr_b[k] || b.lr_a_ld[k] < m || b.lr_b_ld[k] < r))
      throw std::invalid_argument("LR block " + std::to_string(k) + ": null factor or ld < rows");
  }

  FileHeader hdr;
  std::memset(&hdr, 0, sizeof hdr);
  std::memcpy(hdr.magic, kMagic, 8);
  hdr.version = kFileVersion;
  hdr.header_bytes = sizeof(FileHeader);
  hdr.dof = b.dof;
  hdr.n_rows = b.n_rows;
  hdr.n_cols = b.n_cols;
  hdr.n_fr = b.n_fr;
  hdr.n_lr = b.n_lr;
  hdr.fr_entries = fr_entries;
  hdr.lr_entries = lr_entries;
  hdr.flags = b.lr_error ? kFileHasLrError : 0;

  Writer w(path + ".tmp." + std::to_string(static_cast<long long>(getpid())));
  w.put(&hdr, sizeof hdr, nullptr);  // placeholder, rewritten by commit
  auto section = [&](FileSection s, auto &&emit) {
    w.pad();
    StreamHash h;
    hdr.sec[s].offset = w.pos();
    emit(h);
    hdr.sec[s].bytes = w.pos() - hdr.sec[s].offset;
    hdr.sec[s].hash = h.value();
  };
  section(kSecPerm0, [&](StreamHash &h) { w.put(b.perm0, 8 * rp, &h); });
  section(kSecPerm1, [&](StreamHash &h) { w.put(b.perm1, 8 * cp, &h); });
  section(kSecFrPattern, [&](StreamHash &h) { w.put(b.fr_pattern, 48 * b.n_fr, &h); });
  section(kSecLrPattern, [&](StreamHash &h) { w.put(b.lr_pattern, 48 * b.n_lr, &h); });
  section(kSecLrError, [&](StreamHash &h) {
    if (b.lr_error) w.put(b.lr_error, 8 * b.n_lr, &h);
  });
  // column-major m x n with leading dimension ld, written without the padding rows
  auto matrix = [&](StreamHash &h, const double *a, int64_t m, int64_t n, int64_t ld) {
    if (ld == m) {
      w.put(a, 8 * m * n, &h);
    } else {
      for (int64_t j = 0; j < n; j++) w.put(a + j * ld, 8 * m, &h);
    }
  };
  section(kSecFrData, [&](StreamHash &h) {
    for (int64_t k = 0; k < b.n_fr; k++) {
      const int64_t *c = b.fr_pattern + 6 * k;
      matrix(h, b.fr[k], (c[3] - c[1]) * b.dof, (c[4] - c[2]) * b.dof, b.fr_ld[k]);
    }
  });
  section(kSecLrData, [&](StreamHash &h) {
    for (int64_t k = 0; k < b.n_lr; k++) {
      const int64_t *c = b.lr_pattern + 6 * k;
      const int64_t m = (c[3] - c[1]) * b.dof, n = (c[4] - c[2]) * b.dof, r = c[5];
      if (r == 0) continue;
      matrix(h, b.lr_a[k], m, r, b.lr_a_ld[k]);
      matrix(h, b.lr_b[k], r, n, b.lr_b_ld[k]);
    }
  });
  hdr.header_hash = section_hash(&hdr, offsetof(FileHeader, header_hash));
  w.commit(hdr, path);
}

BlockFile::~BlockFile() {
  if (base_) munmap(base_, size_);
}

std::shared_ptr<BlockFile> BlockFile::open(const std::string &path, bool verify) {
  const int fd = ::open(path.c_str(), O_RDONLY | O_CLOEXEC);
  if (fd < 0) throw std::runtime_error("cannot open " + path + ": " + std::strerror(errno));
  struct stat st;
  if (fstat(fd, &st) != 0) {
    const int e = errno;
    ::close(fd);
    throw std::runtime_error("cannot stat " + path + ": " + std::strerror(e));
  }
  if (st.st_size < static_cast<off_t>(sizeof(FileHeader))) {
    ::close(fd);
    throw std::runtime_error(path + " is not a block file (shorter than its header)");
  }
  void *p = mmap(nullptr, static_cast<size_t>(st.st_size), PROT_READ, MAP_SHARED, fd, 0);
  const int e = errno;
  ::close(fd);
  if (p == MAP_FAILED) throw std::runtime_error("cannot map " + path + ": " + std::strerror(e));
  std::shared_ptr<BlockFile> f(new BlockFile);
  f->base_ = p;
  f->size_ = static_cast<size_t>(st.st_size);

  try {
    f->validate(path, verify);
  } catch (const std::invalid_argument &e) {
    throw std::runtime_error(path + ": " + e.what());
  }
  return f;
}

void BlockFile::validate(const std::string &path, bool verify) const {
  const BlockFile *f = this;
  const FileHeader &h = f->header();
  auto corrupt = [&](const std::string &why) { return std::runtime_error(path + ": " + why); };
  if (std::memcmp(h.magic, kMagic, 8) != 0) throw corrupt("not a block file (bad magic)");
  if (h.version != kFileVersion) throw corrupt("unsupported block file version " + std::to_string(h.version));
  if (h.header_bytes != sizeof(FileHeader)) throw corrupt("bad header size");
  if (h.header_hash != section_hash(&h, offsetof(FileHeader, header_hash))) throw corrupt("header checksum mismatch");
  check_sizes(h.dof, h.n_rows, h.n_cols);
  const int64_t size = f->file_bytes();
  if (h.n_fr < 0 || h.n_lr < 0 || h.n_fr > size / 48 || h.n_lr > size / 48 || h.fr_entries < 0 ||
      h.lr_entries < 0 || h.fr_entries > size / 8 || h.lr_entries > size / 8 || (h.flags & ~kFileHasLrError))
    throw corrupt("header counts out of range");
  const int64_t rp = h.n_rows / h.dof, cp = h.n_cols / h.dof;
  const int64_t want[kNumSections] = {8 * rp, 8 * cp, 48 * h.n_fr, 48 * h.n_lr,
                                      (h.flags & kFileHasLrError) ? 8 * h.n_lr : 0, 8 * h.fr_entries,
                                      8 * h.lr_entries};
  int64_t end = sizeof(FileHeader);
  for (int s = 0; s < kNumSections; s++) {
    const FileSectionRec &r = h.sec[s];
    if (r.bytes != want[s]) throw corrupt(std::string("section ") + kSectionName[s] + " has the wrong size");
    if (r.offset < end || r.offset % kFileAlign || r.offset > size || r.bytes > size - r.offset)
      throw corrupt(std::string("section ") + kSectionName[s] + " lies outside the file (truncated?)");
    end = r.offset + r.bytes;
  }
  // the pattern and permutations are small: always checked
  for (int s : {kSecPerm0, kSecPerm1, kSecFrPattern, kSecLrPattern})
    if (section_hash(f->section(static_cast<FileSection>(s)), h.sec[s].bytes) != h.sec[s].hash)
      throw corrupt(std::string("checksum mismatch in section ") + kSectionName[s]);
  check_perm("perm0", f->perm0(), rp);
  check_perm("perm1", f->perm1(), cp);
  if (pattern_entries("FR", f->fr_pattern(), h.n_fr, rp, cp, h.dof, false) != h.fr_entries ||
      pattern_entries("LR", f->lr_pattern(), h.n_lr, rp, cp, h.dof, true) != h.lr_entries)
    throw corrupt("entry counts disagree with the pattern");
  if (verify)
    for (int s : {kSecLrError, kSecFrData, kSecLrData})
      if (section_hash(f->section(static_cast<FileSection>(s)), h.sec[s].bytes) != h.sec[s].hash)
        throw corrupt(std::string("checksum mismatch in section ") + kSectionName[s]);
}

}  // namespace bw
