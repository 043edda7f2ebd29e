// Packing the streaming layout from flat block arrays, for host and device
// code: the element copy of one PackRun (bw_layout.h), equal bit for bit to
// the host fill (fill_items): FP64 copied, FP32 rounded, BF16 multiplied by
// the block's inverse scale in double, rounded to FP32, then to BF16 with
// round-to-nearest-even (the bit operation of bw::to_bf16).
#pragma once

#include <cstdint>
#include <cstring>

#include "bw_layout.h"

#ifdef __CUDACC__
#define BW_PK __host__ __device__ __forceinline__
#else
#define BW_PK inline
#endif

namespace bw {
namespace pack {

BW_PK uint16_t bf16_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return static_cast<uint16_t>((u >> 16) | 0x40u);
  u += 0x7fffu + ((u >> 16) & 1u);
  return static_cast<uint16_t>(u >> 16);
}

// Element (i, c) of run r (0 <= i < r.n, 0 <= c < r.ncols) into dst, the
// phase's data array of precision PREC (0 FP64, 1 FP32, 2 BF16).
template <int PREC>
BW_PK void element(void *dst, const PackRun &r, const double *fr, const double *lr, int64_t i, int64_t c) {
  const double *base = (r.array == 0 ? fr : lr) + r.src_off;
  const int64_t si = r.src_r0 + i, sc = r.src_c0 + c;
  const double v = r.trans ? base[si * r.ld + sc] : base[si + sc * r.ld];
  const int64_t row = r.dst_r0 + i, col = r.dst_c0 + c;
  if (PREC == 0) {
    static_cast<double *>(dst)[r.item_off + col * r.hpad + row] = v;
  } else if (PREC == 1) {
    static_cast<float *>(dst)[r.item_off + col * r.hpad + row] = static_cast<float>(v);
  } else {
    const int64_t e = r.item_off + (col >> 3) * (8 * (int64_t)r.hpad) + (row >> 3) * 64 + (col & 7) * 8 + (row & 7);
    static_cast<uint16_t *>(dst)[e] = bf16_bits(static_cast<float>(v * r.inv));
  }
}

// Every run, sequentially (host reference of the device packer).
template <int PREC>
inline void runs_host(void *dst, const PackRun *runs, int64_t n_runs, const double *fr, const double *lr) {
  for (int64_t k = 0; k < n_runs; k++)
    for (int64_t c = 0; c < runs[k].ncols; c++)
      for (int64_t i = 0; i < runs[k].n; i++) element<PREC>(dst, runs[k], fr, lr, i, c);
}

}  // namespace pack
}  // namespace bw
