// C++ check of the block-file API of the host adapter (bigwham_dev_b200/host),
// run by tests/test_blockfile_cpu.py on CPU:
//
//   1. build a 3DR0-H square crack with the reference's BigWhamIO;
//   2. bigwham_b200::write_block_file(*io.getHmat(), path);
//   3. HmatGpu(path, -1, BW_PLAN_ONLY | BW_FP64): the file constructor;
//   4. its Hmat state (sizes, dof, both HPatterns with their spots, both
//      permutations, every FR block, the ACA error estimates, entry count)
//      must equal the built Hmat's bitwise;
//   5. installed with BigWhamIO::setHmat, GetHPattern, GetMaxErrorACA,
//      GetFullBlocks and GetDiagonal must return what they did before.
// Prints "ok" and exits 0, or names the first mismatch and exits 1.
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "hmat_gpu.h"
#include "io/bigwham_io.h"

namespace {

int fails = 0;

void expect(bool ok, const std::string &what) {
  if (!ok && fails++ == 0) std::printf("mismatch: %s\n", what.c_str());
}

template <typename A, typename B> bool same_2d(const A &a, const B &b) {
  if (a.size(0) != b.size(0) || a.size(1) != b.size(1)) return false;
  for (il::int_t j = 0; j < a.size(1); j++)
    for (il::int_t i = 0; i < a.size(0); i++)
      if (a(i, j) != b(i, j)) return false;
  return true;
}

template <typename A> bool same_1d(const A &a, const A &b) {
  if (a.size() != b.size()) return false;
  for (il::int_t i = 0; i < a.size(); i++)
    if (a[i] != b[i]) return false;
  return true;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    std::printf("usage: %s <block file path>\n", argv[0]);
    return 2;
  }
  const std::string path = argv[1];
  // n x n rectangles on [-1, 1]^2, z = 0, nodes i + j (n + 1)
  const int n = 10;
  std::vector<double> coor;
  for (int j = 0; j <= n; j++)
    for (int i = 0; i <= n; i++) {
      coor.push_back(-1.0 + 2.0 * i / n);
      coor.push_back(-1.0 + 2.0 * j / n);
      coor.push_back(0.0);
    }
  std::vector<int> conn;
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      const int a = i + j * (n + 1);
      conn.insert(conn.end(), {a, a + 1, a + 1 + (n + 1), a + (n + 1)});
    }
  BigWhamIO io(coor, conn, "3DR0-H", {1.0, 0.25}, 2, 0, false, false, false);
  io.BuildHierarchicalMatrix(16, 3.0, 1e-5);
  const auto cpu = io.getHmat();
  const std::vector<double> pattern0 = io.GetHPattern();
  const double maxerr0 = io.GetMaxErrorACA();
  std::vector<double> fv0, d0;
  std::vector<int> fp0;
  io.GetFullBlocks(fv0, fp0);
  io.GetDiagonal(d0);

  bigwham_b200::write_block_file(*cpu, path);
  auto gpu = std::make_shared<bigwham_b200::HmatGpu>(path, -1, BW_PLAN_ONLY | BW_FP64);

  expect(gpu->isBuilt(), "isBuilt");
  expect(gpu->get_size()[0] == cpu->get_size()[0] && gpu->get_size()[1] == cpu->get_size()[1], "size");
  expect(gpu->get_dof_dimension() == cpu->get_dof_dimension(), "dof");
  const auto &pc = cpu->get_hr()->pattern_, &pg = gpu->get_hr()->pattern_;
  expect(pg.n_FRB == pc.n_FRB && pg.n_LRB == pc.n_LRB && pg.n_B == pc.n_B, "block counts");
  expect(same_2d(pg.FRB_pattern, pc.FRB_pattern), "FRB_pattern");
  expect(same_2d(pg.LRB_pattern, pc.LRB_pattern), "LRB_pattern");
  expect(same_1d(gpu->get_hr()->permutation_0_, cpu->get_hr()->permutation_0_), "permutation_0_");
  expect(same_1d(gpu->get_hr()->permutation_1_, cpu->get_hr()->permutation_1_), "permutation_1_");
  const auto &fg = gpu->get_full_rank_blocks(), &fc = cpu->get_full_rank_blocks();
  expect(fg.size() == fc.size(), "FR block count");
  for (size_t k = 0; k < fg.size() && k < fc.size(); k++) expect(same_2d(*fg[k], *fc[k]), "FR block " + std::to_string(k));
  const auto &lg = gpu->get_low_rank_blocks(), &lc = cpu->get_low_rank_blocks();
  expect(lg.size() == lc.size(), "LR block count");
  for (size_t k = 0; k < lg.size() && k < lc.size(); k++)
    expect(lg[k]->error_on_approximation == lc[k]->error_on_approximation, "ACA error " + std::to_string(k));
  expect(gpu->nbOfEntries() == cpu->nbOfEntries(), "nbOfEntries");

  io.setHmat(gpu);
  expect(io.GetHPattern() == pattern0, "GetHPattern");
  expect(io.GetMaxErrorACA() == maxerr0, "GetMaxErrorACA");
  std::vector<double> fv1, d1;
  std::vector<int> fp1;
  io.GetFullBlocks(fv1, fp1);
  expect(fv1 == fv0 && fp1 == fp0, "GetFullBlocks");
  io.GetDiagonal(d1);
  expect(d1 == d0, "GetDiagonal");
  if (fails) return 1;
  std::printf("ok %lld FR %lld LR\n", (long long)pc.n_FRB, (long long)pc.n_LRB);
  return 0;
}
