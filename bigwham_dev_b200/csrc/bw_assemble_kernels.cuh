// Device assembly of the full-rank blocks of a 3DR0-H H-matrix.
//
// The reference builds every full-rank block on the host, entry by entry
// (Hmat::buildFR, src/hmat/hmatrix/hmat.cc:315-353, through
// BieMatrixGenerator::set, src/hmat/bie_matrix_generator.h:94-142).  Here
// each CTA takes 16 x 16 point pairs of one block (a tile); a thread
// evaluates one pair's 3 x 3 entry with bw::r0::h_entry_into_block, the
// function the host tests check against the reference, and writes it into
// the block's column-major storage.  The bytes written are the FR data
// (8 B per entry); the work is FP64 transcendental math (four corners, each
// a few sqrt / log / atan), so the kernel is compute-bound.
#pragma once

#include "bw_r0.h"

namespace bw {

constexpr int kAsmTile = 16;  // points per tile side: 256 pairs per CTA

struct AsmBlock {
  long long off;  // first entry of the block in the output
  int i0, j0;     // first row / column point (permuted numbering)
  int mp, np;     // rows / columns in points
};

struct AsmTile {
  int block, ti, tj, pad;  // block, first row / column point inside it
};

__global__ void __launch_bounds__(kAsmTile *kAsmTile) r0_fr_assemble_kernel(
    const double *__restrict__ records, const int *__restrict__ perm, const AsmBlock *__restrict__ blocks,
    const AsmTile *__restrict__ tiles, long long n_tiles, double G, double nu, double *__restrict__ out) {
  for (long long t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const AsmTile tl = tiles[t];
    const AsmBlock bk = blocks[tl.block];
    const int ii = tl.ti + (int)(threadIdx.x % kAsmTile), jj = tl.tj + (int)(threadIdx.x / kAsmTile);
    if (ii < bk.mp && jj < bk.np)
      r0::h_entry_into_block(records + r0::kFrameDoubles * perm[bk.j0 + jj],
                             records + r0::kFrameDoubles * perm[bk.i0 + ii], G, nu, out + bk.off, 3LL * bk.mp,
                             3LL * ii, 3LL * jj);
  }
}

}  // namespace bw
