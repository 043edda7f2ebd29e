// Device code of the H-matmat Y = H X (up to 64 right-hand sides per pass) on
// the 5th-generation tensor cores (tcgen05, sm_100a).
//
// One persistent kernel per phase, one CTA per SM.  The CTAs take items
// (longest first) from a queue in device memory, one atomicAdd per item; an
// item's result does not depend on the CTA that computes it.  Four roles:
//  * warp 0, producer: takes items from the queue and, for every chunk,
//    issues two or more bulk copies (cp.async.bulk) into a ring of kMmStages
//    shared-memory stages, counted in bytes on the stage's `full` mbarrier:
//      - the chunk's block data (8x8 BF16 tiles);
//      - its runs of operand rows (8x8 BF16 tiles of X or T8, 64 columns).
//    It announces each item (rows, output offset) to the epilogue in a small
//    ring in shared memory, and ends with a kEnd descriptor and an end entry
//    in that ring.
//  * warps 1 and 2, MMA issuers: warp 1 allocates 512 TMEM columns (two
//    accumulator buffers x two issuers x two m-tiles x 64 columns).  One
//    thread per issuer issues tcgen05.mma.cta_group::1.kind::f16, M = 128,
//    N = 64, K = 16.
//      - The K-steps of an item alternate between the issuers (split-K into
//        two accumulators): one thread issues an MMA at most every ~80
//        cycles, two keep the N = 64 tensor pipe fed.
//      - A and B are read from shared memory through MN-major, no-swizzle
//        descriptors.
//      - Each issuer releases a chunk's stage with tcgen05.commit on its
//        `empty` barrier (two arrivals), and at an item's last chunk signals
//        `accfull` (two arrivals).
//  * warps 3-6, epilogue: each reads its 32-lane quarter of both issuers'
//    finished accumulators with tcgen05.ld and adds them.  It then writes T8
//    (BF16 tiles, phase 1) or y (FP64, caller's ordering through the row
//    permutation, phase 2), and hands the buffer back on `accempty`.
// Items alternate between the two accumulator buffers, so the epilogue of one
// item overlaps the MMAs of the next.  Every wait is bounded; on a timeout the
// kernel records an error word, lets copies and MMAs in flight finish, frees
// its TMEM and returns.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "bw_kernels.cuh"
#include "bw_layout.h"

namespace bw {

constexpr int kMmStages = 4;
constexpr int kMmSlack = 2048;      // an M = 128 read of a chunk of fewer rows reaches up to 2 KB past it
constexpr int kMmStageSize = kMmStageBytes + kMmSlack;
constexpr int kMmThreads = 224;     // producer, 2 MMA issuers, 4 epilogue warps
constexpr int kMmTmemCols = 512;    // 2 buffers x 2 issuers x 2 m-tiles x 64 columns
constexpr int kMmRing = 16;         // item announcements in flight (the producer runs at most ~6 items ahead)
constexpr int kMmBarBytes = (2 * kMmStages + 4 + 2) * 8 + 16;
constexpr int kMmSmem =
    kMmStages * kMmStageSize + kMmStages * (int)sizeof(MmChunk) + kMmRing * 16 + kMmBarBytes;
static_assert(kMmSmem <= 232448, "shared memory above the 227 KB per-CTA limit");
static_assert(kMmHMax <= 2 * 128, "an item's rows must fit 2 m-tiles of 128");

constexpr int kErrMmTimeout = 0x201;
constexpr int kErrMmBadChunk = 0x202;

struct MmArgs {
  const uint16_t *data;       // BF16 tiles of the phase
  const MmChunk *chunks;      // item by item
  const int32_t *item_ptr;    // chunk ranges of the items, longest first (n_items + 1)
  int n_items;
  int *queue;                 // [next item, CTAs done]: zero at launch, reset to zero by the last CTA
  const uint16_t *xt;         // operand 0: X in 8x8 tiles, kMmRhs columns
  uint16_t *t8;               // operand 1 (phase 2) / output (phase 1): T8 in 8x8 tiles
  double *y;                  // phase-2 output, column-major, leading dimension ldy
  long long ldy;
  const int32_t *perm_out;    // phase 2: point permutation of the output, or null
  int dof;
  int nrhs;                   // columns of y to write (<= kMmRhs)
  int phase;                  // 1 or 2
  int *err;
  long long spin_limit;       // bound of every wait, in nanoseconds
  int withhold;               // test hook: CTA 0 never stages its chunk of this index (-1: none)
};

// ----------------------------------------------------------------------------- tcgen05 helpers
// Shared-memory matrix descriptor: start address, leading (K-direction) and
// stride (MN-direction) byte offsets of 8x8 core matrices, version 1,
// no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// MN-major, N and M encoded as N/8 and M/16.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(m >> 4) << 24);
}
// One MMA from descriptors given as 32-bit halves.  Consecutive K-steps only
// move the start address, which lives in the low word, so the issue loop
// advances two 32-bit registers per MMA.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint32_t a_lo, uint32_t a_hi, uint32_t b_lo, uint32_t b_hi,
                                          uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t.reg .b64 da, db;\n\t"
      "setp.ne.b32 p, %7, 0;\n\t"
      "mov.b64 da, {%1, %2};\n\tmov.b64 db, {%3, %4};\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], da, db, %5, p;\n\t}\n" ::"r"(d_tmem),
      "r"(a_lo), "r"(a_hi), "r"(b_lo), "r"(b_hi), "r"(idesc), "r"(0), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

// Bounded wait that also gives up when another role has aborted.
__device__ __forceinline__ bool mm_wait(uint64_t *bar, uint32_t parity, long long limit_ns, volatile int *abort) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  unsigned n = 0;
  while (!mbar_try_wait(bar, parity)) {
    if ((++n & 63u) == 0) {
      if (*abort) return false;
      if (global_ns() - t0 > static_cast<unsigned long long>(limit_ns)) return false;
    }
  }
  return true;
}

// Item announcement, producer -> epilogue: written field by field, seq last.
struct MmItemInfo {
  int rows;      // rows to write; -1: no more items
  int out_off;
  int hpad;
  int seq;       // 1 + the item's place in this CTA's sequence
};

__global__ void __launch_bounds__(kMmThreads, 1) mm_stream_kernel(MmArgs a) {
  extern __shared__ __align__(128) unsigned char mm_smem[];
  unsigned char *smem = mm_smem;
  MmChunk *sdesc = reinterpret_cast<MmChunk *>(smem + kMmStages * kMmStageSize);
  volatile MmItemInfo *ring = reinterpret_cast<volatile MmItemInfo *>(sdesc + kMmStages);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + kMmStages * kMmStageSize + kMmStages * sizeof(MmChunk) +
                                                kMmRing * sizeof(MmItemInfo));
  uint64_t *empty = full + kMmStages;
  uint64_t *accfull = empty + kMmStages;   // [2]
  uint64_t *accempty = accfull + 2;        // [2]
  uint64_t *drained = accempty + 2;        // [2] per issuer: MMA completion before TMEM is freed
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drained + 2);
  volatile int *abort = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kMmStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 2);     // one commit per MMA issuer
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accfull[b], 2);   // one commit per MMA issuer
      mbar_init(&accempty[b], 4);  // one arrival per epilogue warp
    }
    mbar_init(&drained[0], 1);
    mbar_init(&drained[1], 1);
    for (int r = 0; r < kMmRing; r++) ring[r].seq = 0;
    *abort = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kMmTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------------------------ producer
    const unsigned char *gdata = reinterpret_cast<const unsigned char *>(a.data);
    const unsigned char *gx = reinterpret_cast<const unsigned char *>(a.xt);
    const unsigned char *gt = reinterpret_cast<const unsigned char *>(a.t8);
    int issued = 0;  // chunks staged by this CTA (stage = issued % kMmStages)
    int nitems = 0;  // items announced
    bool ok = true;
    ItemQueue iq;
    iq.init(a.item_ptr, a.n_items, a.queue, lane);
    // batches of up to 32 chunks of one item; lane k holds chunk k's
    // descriptor, and the next batch's descriptors load during this one
    auto load = [&](int from, int to, uint32_t (&dw)[kMmChunkWords]) {
      if (from + lane < to) {
        const uint4 *p = reinterpret_cast<const uint4 *>(a.chunks + from + lane);
#pragma unroll
        for (int q = 0; q < kMmChunkWords / 4; q++) {
          const uint4 v = __ldg(p + q);
          dw[4 * q] = v.x;
          dw[4 * q + 1] = v.y;
          dw[4 * q + 2] = v.z;
          dw[4 * q + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int q = 0; q < kMmChunkWords; q++) dw[q] = 0;
      }
    };
    int bb = iq.cb;
    uint32_t dw[kMmChunkWords];
    load(bb, iq.ce, dw);
    while (iq.valid() && ok) {
      const int be = min(bb + 32, iq.ce);
      const bool same = be < iq.ce;
      uint32_t ndw[kMmChunkWords];
      load(same ? be : iq.ncb, same ? iq.ce : iq.nce, ndw);
      if (bb == iq.cb) {
        // a new item: announce it to the epilogue (lane 0 holds its first chunk)
        if (lane == 0) {
          volatile MmItemInfo &e = ring[nitems % kMmRing];
          e.rows = static_cast<int>(dw[4]);
          e.out_off = static_cast<int>(dw[5]);
          e.hpad = static_cast<int>(dw[3]);
          __threadfence_block();
          e.seq = nitems + 1;
        }
        nitems++;
      }
      {
        const int nb = be - bb;
        for (int k = 0; k < nb; k++) {
          const int s = issued % kMmStages;
          const uint32_t use = static_cast<uint32_t>(issued / kMmStages);
          // lane k holds chunk k's descriptor and issues it; the others wait
          bool waited = true;
          if (lane == k) {
            waited = mm_wait(&empty[s], (use & 1u) ^ 1u, a.spin_limit, abort);
            if (!waited) {
              set_error(a.err, kErrMmTimeout);
              *abort = 1;
            }
          }
          if (!__shfl_sync(0xffffffffu, waited ? 1 : 0, k)) {
            ok = false;
            break;
          }
          const uint32_t(&w)[kMmChunkWords] = dw;
          // test hook: a withheld chunk is never staged, so its wait runs out
          const bool held = blockIdx.x == 0 && issued == a.withhold;
          if (lane == k && !held) {
            MmChunk *sd = sdesc + s;
            uint4 *sdw = reinterpret_cast<uint4 *>(sd);
#pragma unroll
            for (int q = 0; q < kMmChunkWords / 4; q++)
              sdw[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
            const long long data_off = static_cast<long long>((static_cast<unsigned long long>(w[1]) << 32) | w[0]);
            const int kc = static_cast<int>(w[2]), hpad = static_cast<int>(w[3]);
            const int nr = static_cast<int>((w[6] >> 8) & 0xffu);
            uint32_t run_rows = 0;
#pragma unroll
            for (int r = 0; r < kMmMaxRuns; r++)
              if (r < nr) run_rows += w[8 + 2 * r + 1];
            const uint32_t dbytes = static_cast<uint32_t>(kc) * static_cast<uint32_t>(hpad) * 2u;
            const uint32_t bbytes = static_cast<uint32_t>(kc) * (2u * kMmRhs);
            const bool good = kc > 0 && kc <= kMmMaxCols && (kc & 15) == 0 && hpad > 0 && hpad <= kMmHMax &&
                              (hpad & 7) == 0 && nr > 0 && nr <= kMmMaxRuns &&
                              run_rows == static_cast<uint32_t>(kc) &&
                              dbytes + bbytes <= static_cast<uint32_t>(kMmStageBytes);
            unsigned char *st = smem + s * kMmStageSize;
            if (good) {
              mbar_arrive_expect_tx(&full[s], dbytes + bbytes);
              // operand rows first (stage offset 0), block data after them
              uint32_t dst = 0;
#pragma unroll
              for (int r = 0; r < kMmMaxRuns; r++) {
                if (r < nr) {
                  const uint32_t src = w[8 + 2 * r], rows = w[8 + 2 * r + 1];
                  const unsigned char *base = (src >> 31) ? gt : gx;
                  bulk_g2s(st + dst, base + static_cast<unsigned long long>(src & 0x7fffffffu) * (2u * kMmRhs),
                           rows * (2u * kMmRhs), &full[s]);
                  dst += rows * (2u * kMmRhs);
                }
              }
              // block data: read once per launch, evict first (the operand
              // rows, re-read by many chunks, keep the normal policy)
              bulk_g2s_hint(st + bbytes, gdata + static_cast<unsigned long long>(data_off) * 2ull, dbytes, &full[s],
                            l2_evict_first_policy());
            } else {
              set_error(a.err, kErrMmBadChunk);
              sd->kc = 0;  // the MMA issuers skip the chunk
              sd->flags &= ~kEnd;
              mbar_arrive(&full[s]);
            }
          }
          __syncwarp();
          issued++;
        }
      }
      if (same) {
        bb = be;
      } else {
        iq.advance(lane);
        bb = iq.cb;
      }
#pragma unroll
      for (int q = 0; q < kMmChunkWords; q++) dw[q] = ndw[q];
    }
    if (ok) {
      // end of work: the issuers get a kEnd descriptor, the epilogue an end entry
      const int s = issued % kMmStages;
      const uint32_t use = static_cast<uint32_t>(issued / kMmStages);
      if (mm_wait(&empty[s], (use & 1u) ^ 1u, a.spin_limit, abort)) {
        if (lane == 0) {
          sdesc[s].kc = 0;
          sdesc[s].flags = kEnd;
          mbar_arrive(&full[s]);
          volatile MmItemInfo &e = ring[nitems % kMmRing];
          e.rows = -1;
          __threadfence_block();
          e.seq = nitems + 1;
        }
      } else {
        if (lane == 0) {
          set_error(a.err, kErrMmTimeout);
          *abort = 1;
        }
        ok = false;
      }
    }
    if (!ok) {
      // let the copies in flight land before the CTA can exit
      for (int i = max(0, issued - kMmStages); i < issued; i++) {
        if (blockIdx.x == 0 && i == a.withhold) continue;  // nothing in flight for it
        const int s = i % kMmStages;
        mbar_wait(&full[s], static_cast<uint32_t>(i / kMmStages) & 1u, kDrainLimitNs);
      }
    }
    // This CTA takes no more items.  The last CTA to get here returns the
    // queue to zero for the next launch (every other CTA is done with it).
    if (lane == 0) {
      __threadfence();
      if (atomicAdd(&a.queue[1], 1) == static_cast<int>(gridDim.x) - 1) {
        a.queue[0] = 0;
        a.queue[1] = 0;
        __threadfence();
      }
    }
  } else if (warp < 3) {
    // ------------------------------------------------------------------ MMA issuers
    const uint32_t q = static_cast<uint32_t>(warp - 1);  // takes the item's K-steps of parity q
    const uint32_t idesc = umma_idesc_bf16(128, kMmRhs);
    uint32_t items = 0;
    int kg = 0;            // K-steps of the current item before this chunk
    bool started = false;  // this issuer's accumulator of the current item holds a product
    bool ok = true;
    for (int i = 0;; i++) {
      const int s = i % kMmStages;
      const uint32_t use = static_cast<uint32_t>(i / kMmStages);
      if (!mm_wait(&full[s], use & 1u, a.spin_limit, abort)) {
        ok = false;
        break;
      }
      const MmChunk &d = sdesc[s];
      const int kc = d.kc, hpad = d.hpad;
      const uint32_t flags = d.flags;
      if (flags & kEnd) break;
      const uint32_t buf = items & 1u;
      if (flags & kFirst) {
        if (!mm_wait(&accempty[buf], ((items >> 1) & 1u) ^ 1u, a.spin_limit, abort)) {
          ok = false;
          break;
        }
        kg = 0;
        started = false;
      }
      tc_fence_after();
      const int nks = kc >> 4;
      const int ks0 = (static_cast<int>(q) - kg) & 1;  // first K-step of this chunk with the issuer's parity
      if (lane == 0 && kc > 0 && ks0 < nks) {
        // descriptors of K-step ks0; each of this issuer's K-steps moves A by
        // 4 * lbo_a bytes and B by 4 * lbo_b bytes (two K-steps), i.e. the
        // start-address field by that / 16
        const int nM = (hpad + 127) >> 7;
        const uint32_t sb = smem_u32(smem + s * kMmStageSize);
        const uint32_t sa = sb + static_cast<uint32_t>(kc) * (2u * kMmRhs);
        const uint32_t lbo_a = 16u * static_cast<uint32_t>(hpad), lbo_b = 16u * kMmRhs;
        const uint64_t a0 = umma_desc(sa + static_cast<uint32_t>(ks0) * 2u * lbo_a, lbo_a, 128u);
        const uint64_t b0 = umma_desc(sb + static_cast<uint32_t>(ks0) * 2u * lbo_b, lbo_b, 128u);
        const uint32_t a_hi = static_cast<uint32_t>(a0 >> 32), b_hi = static_cast<uint32_t>(b0 >> 32);
        const uint32_t a_step = (4u * lbo_a) >> 4, b_step = (4u * lbo_b) >> 4;
        const uint32_t acc0 = started ? 1u : 0u;
        for (int mt = 0; mt < nM; mt++) {
          const uint32_t dt = tmem + buf * 256u + q * 128u + static_cast<uint32_t>(mt) * kMmRhs;
          uint32_t a_lo = static_cast<uint32_t>(a0) + static_cast<uint32_t>(mt) * (2048u >> 4);
          uint32_t b_lo = static_cast<uint32_t>(b0);
          umma_bf16(dt, a_lo, a_hi, b_lo, b_hi, idesc, acc0);
#pragma unroll 4
          for (int ks = ks0 + 2; ks < nks; ks += 2) {
            a_lo += a_step;
            b_lo += b_step;
            umma_bf16(dt, a_lo, a_hi, b_lo, b_hi, idesc, 1u);
          }
        }
      }
      if (ks0 < nks) started = true;
      kg += nks;
      __syncwarp();
      if (lane == 0) {
        umma_commit(&empty[s]);
        if (flags & kLast) umma_commit(&accfull[buf]);
      }
      __syncwarp();
      if (flags & kLast) items++;
    }
    if (!ok && lane == 0) {
      set_error(a.err, kErrMmTimeout);
      *abort = 1;
    }
    // every MMA issued so far completes before the TMEM is freed
    if (lane == 0) umma_commit(&drained[q]);
    __syncwarp();
    mbar_wait(&drained[q], 0u, kDrainLimitNs);
  } else {
    // ------------------------------------------------------------------ epilogue
    const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
    for (uint32_t items = 0;; items++) {
      // the item's announcement (bounded wait on the ring entry)
      volatile MmItemInfo &e = ring[items % kMmRing];
      bool seen = e.seq == static_cast<int>(items + 1);
      if (!seen) {
        const unsigned long long t0 = global_ns();
        unsigned n = 0;
        while (!(seen = e.seq == static_cast<int>(items + 1))) {
          if ((++n & 63u) == 0 && (*abort || global_ns() - t0 > static_cast<unsigned long long>(a.spin_limit)))
            break;
        }
      }
      if (!seen) {
        if (lane == 0) {
          set_error(a.err, kErrMmTimeout);
          *abort = 1;
        }
        break;
      }
      __threadfence_block();
      const int irows = e.rows, ioff = e.out_off, ihpad = e.hpad;
      if (irows < 0) break;  // no more items
      const uint32_t buf = items & 1u;
      if (!mm_wait(&accfull[buf], (items >> 1) & 1u, a.spin_limit, abort)) {
        if (lane == 0) {
          set_error(a.err, kErrMmTimeout);
          *abort = 1;
        }
        break;
      }
      tc_fence_after();
      const int nM = (ihpad + 127) >> 7;
      for (int mt = 0; mt < nM; mt++) {
        const int row = mt * 128 + quarter * 32 + lane;
        const bool live = row < irows;
        long long dst = 0;
        if (live && a.phase == 2) {
          const int orow = ioff + row;
          dst = a.perm_out ? static_cast<long long>(a.dof) * a.perm_out[orow / a.dof] + (orow % a.dof) : orow;
        }
#pragma unroll 1
        for (int c0 = 0; c0 < kMmRhs; c0 += 16) {
          float v[16], v2[16];
          const uint32_t ta = tmem + (static_cast<uint32_t>(quarter * 32) << 16) + buf * 256u +
                              static_cast<uint32_t>(mt) * kMmRhs + static_cast<uint32_t>(c0);
          tmem_ld16(ta, v);
          tmem_ld16(ta + 128u, v2);  // the second issuer's accumulator
          if (!live) continue;
#pragma unroll
          for (int k2 = 0; k2 < 16; k2++) v[k2] += v2[k2];
          if (a.phase == 1) {
            const long long r8 = static_cast<long long>(ioff) + row;
#pragma unroll
            for (int g = 0; g < 2; g++) {
              uint4 pk;
              pk.x = pack_bf16x2(v[8 * g + 0], v[8 * g + 1]);
              pk.y = pack_bf16x2(v[8 * g + 2], v[8 * g + 3]);
              pk.z = pack_bf16x2(v[8 * g + 4], v[8 * g + 5]);
              pk.w = pack_bf16x2(v[8 * g + 6], v[8 * g + 7]);
              const long long e8 = (r8 >> 3) * (8 * kMmRhs) + ((c0 >> 3) + g) * 64 + (r8 & 7) * 8;
              *reinterpret_cast<uint4 *>(a.t8 + e8) = pk;
            }
          } else {
#pragma unroll
            for (int k2 = 0; k2 < 16; k2++)
              if (c0 + k2 < a.nrhs) a.y[static_cast<long long>(c0 + k2) * a.ldy + dst] = static_cast<double>(v[k2]);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&accempty[buf]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMmTmemCols));
  }
}

// X (FP64, column-major with leading dimension ldx, caller's ordering) ->
// Xt: BF16 8x8 tiles of kMmRhs columns in the permuted row order,
// Xt(i, j) at (i/8)*8*kMmRhs + (j/8)*64 + (i%8)*8 + j%8, for rows i < n_pad
// (rows >= n and columns >= nrhs are zero).  One block per 64 rows, staged
// through shared memory so that both the reads (along rows, per column) and
// the 16-byte tile writes are coalesced.
__global__ void __launch_bounds__(256) gather_xt_kernel(const double *__restrict__ x, long long ldx, int nrhs,
                                                        uint16_t *__restrict__ xt, const int32_t *__restrict__ perm,
                                                        int dof, int n, int n_pad) {
  __shared__ float tile[64][kMmRhs + 1];
  const int i0 = blockIdx.x * 64;
  for (int e = threadIdx.x; e < 64 * kMmRhs; e += blockDim.x) {
    const int j = e >> 6, r = e & 63;
    const int i = i0 + r;
    float v = 0.f;
    if (i < n && j < nrhs) {
      const int src = perm ? dof * perm[i / dof] + (i % dof) : i;
      v = static_cast<float>(x[static_cast<long long>(j) * ldx + src]);
    }
    tile[r][j] = v;
  }
  __syncthreads();
  // 64 rows x 8 groups of 8 columns = 512 16-byte words: word q of the block
  // is row-group q / 64, column group (q / 8) % 8, row (q % 8)
  for (int q = threadIdx.x; q < 512; q += blockDim.x) {
    const int r = (q >> 6) * 8 + (q & 7), g = (q >> 3) & 7;
    const int i = i0 + r;
    if (i >= n_pad) continue;
    uint4 pk;
    pk.x = pack_bf16x2(tile[r][8 * g + 0], tile[r][8 * g + 1]);
    pk.y = pack_bf16x2(tile[r][8 * g + 2], tile[r][8 * g + 3]);
    pk.z = pack_bf16x2(tile[r][8 * g + 4], tile[r][8 * g + 5]);
    pk.w = pack_bf16x2(tile[r][8 * g + 6], tile[r][8 * g + 7]);
    *reinterpret_cast<uint4 *>(xt + static_cast<long long>(i >> 3) * (8 * kMmRhs) + g * 64 + (i & 7) * 8) = pk;
  }
}

}  // namespace bw
