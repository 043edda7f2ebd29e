// Device code of the streamed H-matrix matvec (sm_100a).
//
// One persistent kernel per phase (see bw_layout.h).  The CTAs take items
// (longest first) from a queue in device memory, one atomicAdd per item, so a
// CTA that finishes early takes more work; an item's result does not depend on
// the CTA that computes it.  Warp 0 is the producer: for every chunk it
// stages the block data and the chunk's contiguous run of vector values with
// two TMA bulk copies (cp.async.bulk of the 16-byte aligned windows around
// them) into a ring of kStages shared-memory stages; one mbarrier per stage
// counts the bytes, one more per stage returns it to the producer.
// Warps 1..8 are consumers and own the item's output rows:
//  * FP64 / FP32: each thread owns 2 (FP64) or 4 (FP32) adjacent rows and a
//    contiguous range of the chunk's columns and accumulates with FMAs;
//  * BF16: tensor cores.  The chunk is stored in 8x8 tiles, so ldmatrix.trans
//    loads 16x16 A fragments from 128-byte contiguous shared memory; the
//    vector is the B operand (column 0: its BF16 rounding, column 1: the BF16
//    rounding of the remainder, so the product keeps ~16 bits of the FP32
//    vector), mma.m16n8k16 accumulates in FP32 registers across the item.
// At the item's last chunk the partial sums are reduced in shared memory and
// written once (t for phase 1, y for phase 2, with the row permutation applied
// on the fly).  Every wait is a bounded mbarrier try_wait loop; on timeout the
// kernel records an error word and returns.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "bw_layout.h"

namespace bw {

constexpr int kStages = 6;

// Bound of the waits that only let work already issued finish (bulk copies
// in flight, MMAs before TMEM is freed) after an error: independent of the
// caller's wait limit, so that no CTA exits with work outstanding.
constexpr long long kDrainLimitNs = 2000000000LL;

// error words
constexpr int kErrTimeoutEmpty = 0x101;
constexpr int kErrTimeoutFull = 0x102;
constexpr int kErrTimeoutReduce = 0x103;
constexpr int kErrBadChunk = 0x104;

struct StreamArgs {
  const void *data;           // element array of the phase (storage type)
  const Chunk *chunks;        // item by item
  const int32_t *item_ptr;    // chunk ranges of the items, longest first (n_items + 1)
  int n_items;
  int n_coop;                 // warp-per-item kernel: units [0, n_coop) run CTA-cooperatively
  int *queue;                 // [next item, CTAs done(, next CTA-cooperative unit)]: zero at launch, reset
                              // to zero by the last CTA
  const void *gsrc;           // vector values: gathered x (phase 1) or G2 (phase 2), compute type
  void *t_out;                // phase-1 output (compute type; BF16: unscaled, G2 applies the block scales)
  double *y_out;              // phase-2 output
  const int32_t *perm_out;    // phase 2: point permutation of the output, or null
  int dof;
  int phase;                  // 1 or 2
  int *err;
  long long spin_limit;       // bound of every wait, in nanoseconds
  int withhold;               // test hook: CTA 0 never stages its chunk of this index (-1: none)
};

// ----------------------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// TMA bulk copy global -> shared (this CTA), completion counted on `bar` in bytes.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// L2 policy for data read exactly once per launch (the block data): evict
// first, so that the streamed gigabytes do not push the small arrays every
// chunk touches (vectors, permutations, descriptors, queue ranges) out of L2.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// bulk_g2s with an L2 cache policy.
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}
// Programmatic dependent launch: a kernel launched right after this one with
// the programmatic-serialization attribute may start once every CTA of this
// one has issued launch_dependents (or exited); wait blocks until the grids
// this one depends on have completed and their writes are visible.  Both are
// no-ops without such a launch.
__device__ __forceinline__ void pdl_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait: false when `limit_ns` nanoseconds passed without the phase completing.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  unsigned n = 0;
  while (!mbar_try_wait(bar, parity)) {
    if ((++n & 63u) == 0 && global_ns() - t0 > static_cast<unsigned long long>(limit_ns)) return false;
  }
  return true;
}
__device__ __forceinline__ void set_error(int *err, int code) { atomicCAS(err, 0, code); }

// Four 8x8 b16 matrices from shared memory, transposed into mma A-fragment order.
__device__ __forceinline__ void ldmatrix_x4_trans(uint32_t addr, uint32_t &a0, uint32_t &a1, uint32_t &a2,
                                                  uint32_t &a3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3)
               : "r"(addr));
}
// D(16x8, f32) += A(16x16, bf16, row) * B(16x8, bf16, col)
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

// ----------------------------------------------------------------------------- storage traits
struct Bf16 {};  // storage tag: 16-bit brain float, 8x8-tiled items

template <typename S> struct Store;
// kWarps: consumer warps per CTA (the BF16 path is latency-bound and gets
// more warps; the FMA paths already stream at the HBM roofline with 8).
// kRed: partial sums per reduction buffer, Q * hpad <= kRows * consumers
// (FMA paths) or kparts * hpad <= 16 * 128 (tensor path).
template <> struct Store<double> {
  using G = double;   // compute / gather type
  static constexpr int kEsize = 8;
  static constexpr int kRows = 2;  // rows per consumer thread
  static constexpr int kWarps = 8;
  static constexpr int kRed = 2 * 32 * kWarps;
};
template <> struct Store<float> {
  using G = float;
  static constexpr int kEsize = 4;
  static constexpr int kRows = 4;
  static constexpr int kWarps = 8;
  static constexpr int kRed = 4 * 32 * kWarps;
};
template <> struct Store<Bf16> {
  using G = float;
  static constexpr int kEsize = 2;
  static constexpr int kRows = 0;  // tensor-core path
  static constexpr int kWarps = 16;
  static constexpr int kRed = 2048;
};
template <typename S> __host__ __device__ constexpr int consumers_of() { return 32 * Store<S>::kWarps; }
template <typename S> __host__ __device__ constexpr int threads_of() { return 32 + consumers_of<S>(); }

// Adds the partial sums of R adjacent rows over columns [c0, c1) of a
// column-major chunk to o; the vector value of column c is g[c].
template <typename S, int R>
__device__ __forceinline__ void chunk_dot(const unsigned char *base, const typename Store<S>::G *g, int hv, int rv,
                                          int c0, int c1, typename Store<S>::G (&o)[R]);

template <>
__device__ __forceinline__ void chunk_dot<double, 2>(const unsigned char *base, const double *g, int hv, int rv,
                                                     int c0, int c1, double (&o)[2]) {
  const double2 *d = reinterpret_cast<const double2 *>(base) + rv;
  double a0 = 0, a1 = 0, b0 = 0, b1 = 0;
  int c = c0;
#pragma unroll 1
  for (; c + 4 <= c1; c += 4) {
    const double2 w0 = d[(c + 0) * hv], w1 = d[(c + 1) * hv], w2 = d[(c + 2) * hv], w3 = d[(c + 3) * hv];
    const double g0 = g[c], g1 = g[c + 1], g2 = g[c + 2], g3 = g[c + 3];
    a0 = fma(w0.x, g0, a0);
    a1 = fma(w0.y, g0, a1);
    b0 = fma(w1.x, g1, b0);
    b1 = fma(w1.y, g1, b1);
    a0 = fma(w2.x, g2, a0);
    a1 = fma(w2.y, g2, a1);
    b0 = fma(w3.x, g3, b0);
    b1 = fma(w3.y, g3, b1);
  }
  for (; c < c1; c++) {
    const double2 w = d[c * hv];
    a0 = fma(w.x, g[c], a0);
    a1 = fma(w.y, g[c], a1);
  }
  o[0] += a0 + b0;
  o[1] += a1 + b1;
}

template <>
__device__ __forceinline__ void chunk_dot<float, 4>(const unsigned char *base, const float *g, int hv, int rv,
                                                    int c0, int c1, float (&o)[4]) {
  const float4 *d = reinterpret_cast<const float4 *>(base) + rv;
  float a0 = 0, a1 = 0, a2 = 0, a3 = 0, b0 = 0, b1 = 0, b2 = 0, b3 = 0;
  int c = c0;
#pragma unroll 1
  for (; c + 4 <= c1; c += 4) {
    const float4 w0 = d[(c + 0) * hv], w1 = d[(c + 1) * hv], w2 = d[(c + 2) * hv], w3 = d[(c + 3) * hv];
    const float g0 = g[c], g1 = g[c + 1], g2 = g[c + 2], g3 = g[c + 3];
    a0 = fmaf(w0.x, g0, a0);
    a1 = fmaf(w0.y, g0, a1);
    a2 = fmaf(w0.z, g0, a2);
    a3 = fmaf(w0.w, g0, a3);
    b0 = fmaf(w1.x, g1, b0);
    b1 = fmaf(w1.y, g1, b1);
    b2 = fmaf(w1.z, g1, b2);
    b3 = fmaf(w1.w, g1, b3);
    a0 = fmaf(w2.x, g2, a0);
    a1 = fmaf(w2.y, g2, a1);
    a2 = fmaf(w2.z, g2, a2);
    a3 = fmaf(w2.w, g2, a3);
    b0 = fmaf(w3.x, g3, b0);
    b1 = fmaf(w3.y, g3, b1);
    b2 = fmaf(w3.z, g3, b2);
    b3 = fmaf(w3.w, g3, b3);
  }
  for (; c < c1; c++) {
    const float4 w = d[c * hv];
    a0 = fmaf(w.x, g[c], a0);
    a1 = fmaf(w.y, g[c], a1);
    a2 = fmaf(w.z, g[c], a2);
    a3 = fmaf(w.w, g[c], a3);
  }
  o[0] += a0 + b0;
  o[1] += a1 + b1;
  o[2] += a2 + b2;
  o[3] += a3 + b3;
}

// ----------------------------------------------------------------------------- shared memory
template <typename S> struct SmemLayout {
  using G = typename Store<S>::G;
  static constexpr int kDataBytes = kStageBytes + 32;
  // vector window: the chunk's run of values with up to 15 bytes of slack each side
  static constexpr int kGBytes = kMaxCols * (int)sizeof(G) + 32;
  static constexpr int kStageSize = kDataBytes + kGBytes + (int)sizeof(Chunk);
  static constexpr int kRedPer = Store<S>::kRed;
  static_assert(kHMax <= 2 * consumers_of<S>(), "each consumer thread writes at most two output rows of an item");
  static constexpr int kRedBytes = 2 * kRedPer * (int)sizeof(G);
  static constexpr int kBarBytes = (2 * kStages + 1) * 8;
  static constexpr int kTotal = kStages * kStageSize + kRedBytes + kBarBytes;
  static_assert(kStageSize % 16 == 0, "stage must keep 16-byte alignment");
  static_assert(kTotal <= 232448, "shared memory above the 227 KB per-CTA limit");
};

struct DescRegs {
  uint32_t w[kChunkWords];
};

template <int N> struct IntC {
  static constexpr int value = N;
};

// The producer warp's view of the work queue, pipelined so that no latency
// lands on an item boundary:
//  * `cur` is the item being staged, its chunk range [cb, ce) already loaded;
//  * `nxt` is the next item, its range [ncb, nce) loading during `cur`;
//  * lane 0 holds `pend`, the result of the atomicAdd for the item after
//    that, issued one item earlier.
// An index >= n_items means the queue is empty; no atomic is issued after
// that, so the CTA touches queue[0] at most n_taken + 3 times.
struct ItemQueue {
  const int32_t *item_ptr;
  int n_items;
  int *queue;
  int cur, cb, ce;
  int nxt, ncb, nce;
  int pend;  // lane 0 only

  __device__ __forceinline__ void load_range(int it, int &b, int &e) const {
    b = 0;
    e = 0;
    if (it < n_items) {
      b = item_ptr[it];
      e = item_ptr[it + 1];
    }
  }
  __device__ __forceinline__ void init(const int32_t *ptr, int n, int *q, int lane) {
    item_ptr = ptr;
    n_items = n;
    queue = q;
    int i0 = 0, i1 = 0;
    pend = n;
    if (lane == 0) {
      i0 = atomicAdd(&queue[0], 1);
      i1 = i0 < n ? atomicAdd(&queue[0], 1) : n;
      pend = i1 < n ? atomicAdd(&queue[0], 1) : n;
    }
    cur = __shfl_sync(0xffffffffu, i0, 0);
    nxt = __shfl_sync(0xffffffffu, i1, 0);
    load_range(cur, cb, ce);
    load_range(nxt, ncb, nce);
  }
  __device__ __forceinline__ bool valid() const { return cur < n_items; }
  __device__ __forceinline__ void advance(int lane) {
    cur = nxt;
    cb = ncb;
    ce = nce;
    nxt = __shfl_sync(0xffffffffu, pend, 0);
    load_range(nxt, ncb, nce);
    if (lane == 0) pend = nxt < n_items ? atomicAdd(&queue[0], 1) : n_items;
  }
};

__device__ __forceinline__ void load_desc(const Chunk *chunks, int idx, int end, DescRegs &r) {
  if (idx < end) {
    const uint4 *p = reinterpret_cast<const uint4 *>(chunks + idx);
#pragma unroll
    for (int k = 0; k < kChunkWords / 4; k++) {
      const uint4 v = __ldg(p + k);
      r.w[4 * k + 0] = v.x;
      r.w[4 * k + 1] = v.y;
      r.w[4 * k + 2] = v.z;
      r.w[4 * k + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kChunkWords; k++) r.w[k] = 0;
  }
}

template <typename S>
__global__ void __launch_bounds__(threads_of<S>(), 1) stream_panels_kernel(StreamArgs a) {
  using G = typename Store<S>::G;
  using L = SmemLayout<S>;
  constexpr int es = Store<S>::kEsize;
  constexpr bool kTensor = Store<S>::kRows == 0;
  constexpr int kConsumerWarps = Store<S>::kWarps;
  constexpr int kConsumers = consumers_of<S>();
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *stage0 = smem;
  G *red = reinterpret_cast<G *>(smem + kStages * L::kStageSize);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + kStages * L::kStageSize + L::kRedBytes);
  uint64_t *empty = full + kStages;
  uint64_t *redbar = empty + kStages;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 1);                  // lane-0 arrive.expect_tx; the two bulk copies complete the tx
      mbar_init(&empty[s], kConsumerWarps);    // one arrival per consumer warp
    }
    mbar_init(redbar, kConsumerWarps);
    fence_barrier_init();
  }
  __syncthreads();
  // Every CTA is resident and holds its shared memory: a phase's unstaged
  // launch (independent items, its own queue) may start filling the SMs this
  // launch leaves free, and the SMs it frees as its CTAs run out of items.
  pdl_launch_dependents();

  if (warp == 0) {
    // ------------------------------------------------------------------ producer
    const unsigned char *gdata = static_cast<const unsigned char *>(a.data);
    const unsigned char *gvec = static_cast<const unsigned char *>(a.gsrc);
    const uint64_t stream_policy = l2_evict_first_policy();
    bool ok = true;
    int issued = 0;  // chunks staged so far by this CTA (stage = issued % kStages)
    ItemQueue iq;
    iq.init(a.item_ptr, a.n_items, a.queue, lane);
    // batches of up to 32 chunks of one item; lane k holds chunk k's
    // descriptor, and the next batch's descriptors load during this one
    int bb = iq.cb;
    DescRegs cur_d;
    load_desc(a.chunks, bb + lane, iq.ce, cur_d);
    while (iq.valid() && ok) {
      const int be = min(bb + 32, iq.ce);
      const bool same = be < iq.ce;
      DescRegs nxt_d;
      load_desc(a.chunks, (same ? be : iq.ncb) + lane, same ? iq.ce : iq.nce, nxt_d);
      {
        const int nb = be - bb;
        for (int k = 0; k < nb; k++) {
          const int s = issued % kStages;
          const uint32_t use = static_cast<uint32_t>(issued / kStages);
          if (!mbar_wait(&empty[s], (use & 1u) ^ 1u, a.spin_limit)) {
            if (lane == 0) set_error(a.err, kErrTimeoutEmpty);
            ok = false;
            break;
          }
          uint32_t w[kChunkWords];
#pragma unroll
          for (int q = 0; q < kChunkWords; q++) w[q] = __shfl_sync(0xffffffffu, cur_d.w[q], k);
          // test hook: a withheld chunk is never staged, so its wait runs out
          const bool held = blockIdx.x == 0 && issued == a.withhold;
          if (lane == 0 && !held) {
            const long long data_off = static_cast<long long>((static_cast<unsigned long long>(w[1]) << 32) | w[0]);
            const int ncols = static_cast<int>(w[2]);
            const int hpad = static_cast<int>(w[3]);
            const int g_off = static_cast<int>(w[7]);
            unsigned char *st = stage0 + s * L::kStageSize;
            uint4 *dd = reinterpret_cast<uint4 *>(st + L::kDataBytes + L::kGBytes);
#pragma unroll
            for (int q = 0; q < kChunkWords / 4; q++)
              dd[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
            const unsigned long long cols = kTensor ? (static_cast<unsigned long long>(ncols) + 7ull) & ~7ull
                                                    : static_cast<unsigned long long>(ncols);
            const unsigned long long bytes = cols * hpad * es;
            if (ncols > 0 && ncols <= kMaxCols && bytes <= static_cast<unsigned long long>(kStageBytes)) {
              const unsigned long long src = reinterpret_cast<unsigned long long>(gdata) +
                                             static_cast<unsigned long long>(data_off) * es;
              const unsigned long long lo = src & ~15ull, hi = (src + bytes + 15ull) & ~15ull;
              const unsigned long long gs = reinterpret_cast<unsigned long long>(gvec) +
                                            static_cast<unsigned long long>(g_off) * sizeof(G);
              const unsigned long long glo = gs & ~15ull, ghi = (gs + ncols * sizeof(G) + 15ull) & ~15ull;
              mbar_arrive_expect_tx(&full[s], static_cast<uint32_t>((hi - lo) + (ghi - glo)));
              // evict-first helps the BF16 launches (measured A/B at 196,608 DoF:
              // -2 to -4%) and slows the FP32 / FP64 row panels (+1 to +3%)
              if constexpr (kTensor)
                bulk_g2s_hint(st, reinterpret_cast<const void *>(lo), static_cast<uint32_t>(hi - lo), &full[s],
                              stream_policy);
              else
                bulk_g2s(st, reinterpret_cast<const void *>(lo), static_cast<uint32_t>(hi - lo), &full[s]);
              bulk_g2s(st + L::kDataBytes, reinterpret_cast<const void *>(glo), static_cast<uint32_t>(ghi - glo),
                       &full[s]);
            } else {
              if (ncols > 0) set_error(a.err, kErrBadChunk);
              mbar_arrive(&full[s]);
            }
          }
          issued++;
        }
      }
      if (same) {
        bb = be;
      } else {
        iq.advance(lane);
        bb = iq.cb;
      }
      cur_d = nxt_d;
    }
    if (ok) {
      // end of work: a descriptor with kEnd alone, no data
      const int s = issued % kStages;
      const uint32_t use = static_cast<uint32_t>(issued / kStages);
      if (mbar_wait(&empty[s], (use & 1u) ^ 1u, a.spin_limit)) {
        if (lane == 0) {
          uint4 *dd = reinterpret_cast<uint4 *>(stage0 + s * L::kStageSize + L::kDataBytes + L::kGBytes);
          dd[0] = make_uint4(0, 0, 0, 0);
          dd[1] = make_uint4(0, 0, kEnd, 0);
          mbar_arrive(&full[s]);
        }
      } else {
        if (lane == 0) set_error(a.err, kErrTimeoutEmpty);
        ok = false;
      }
    }
    if (!ok) {
      // let the copies already in flight land before the CTA can exit
      for (int i = max(0, issued - kStages); i < issued; i++) {
        if (blockIdx.x == 0 && i == a.withhold) continue;  // nothing in flight for it
        const int s = i % kStages;
        mbar_wait(&full[s], static_cast<uint32_t>(i / kStages) & 1u, kDrainLimitNs);
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
    return;
  }

  // -------------------------------------------------------------------- consumers
  const int ct = threadIdx.x - 32;
  const int cw = warp - 1;
  uint32_t items = 0;
  long long pre_dst[2] = {0, 0};
  // FMA path state
  constexpr int R = kTensor ? 1 : Store<S>::kRows;
  int hv = 1, Q = 1, rv = 0, cq = 0;
  bool active = false;
  G acc[R];
#pragma unroll
  for (int r = 0; r < R; r++) acc[r] = 0;
  // tensor path state
  int nMt = 1, kparts = 1, mg = 0, kp = 0;
  int rot = 0;  // rotation of the K-step deal: chunk index within the item, mod kparts
  bool wact = false;
  float tacc[kTensor ? 8 : 1][4];
#pragma unroll
  for (int j = 0; j < (kTensor ? 8 : 1); j++)
#pragma unroll
    for (int q = 0; q < 4; q++) tacc[j][q] = 0.f;

  for (int i = 0;; i++) {
    const int s = i % kStages;
    const uint32_t use = static_cast<uint32_t>(i / kStages);
    if (!mbar_wait(&full[s], use & 1u, a.spin_limit)) {
      if (lane == 0) set_error(a.err, kErrTimeoutFull);
      return;
    }
    const unsigned char *st = stage0 + s * L::kStageSize;
    const Chunk &d = *reinterpret_cast<const Chunk *>(st + L::kDataBytes + L::kGBytes);
    if (d.flags & kEnd) return;  // the producer has no more items for this CTA
    // the vector window starts at the 16-byte boundary below gsrc + g_off
    const G *gs = reinterpret_cast<const G *>(
        st + L::kDataBytes +
        ((reinterpret_cast<unsigned long long>(a.gsrc) + static_cast<unsigned long long>(d.g_off) * sizeof(G)) &
         15ull));
    const uint32_t flags = d.flags;
    const int ncols = d.ncols;
    const int hpad = d.hpad;
    const int rows = d.rows, out_off = d.out_off;
    if (flags & kFirst) {
      // Phase 2: the permuted y index of the item's rows, loaded now so the
      // latency is hidden behind the item's chunks.
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int r = ct + q * kConsumers;
        pre_dst[q] = out_off + r;
        if (r < rows && a.phase == 2 && a.perm_out) {
          const int row = out_off + r;
          pre_dst[q] = static_cast<long long>(a.dof) * a.perm_out[row / a.dof] + (row % a.dof);
        }
      }
    }
    if constexpr (!kTensor) {
      if (flags & kFirst) {
        hv = hpad / R;
        Q = kConsumers / hv;
        rv = ct % hv;
        cq = ct / hv;
        active = cq < Q;
#pragma unroll
        for (int r = 0; r < R; r++) acc[r] = 0;
      }
      if (active && ncols > 0 && ncols <= kMaxCols) {
        const int c0 = (cq * ncols) / Q, c1 = ((cq + 1) * ncols) / Q;
        const int soff = static_cast<int>((static_cast<unsigned long long>(d.data_off) * es) & 15ull);
        chunk_dot<S, R>(st + soff, gs, hv, rv, c0, c1, acc);
      }
    } else {
      if (flags & kFirst) {
        nMt = (hpad + 15) >> 4;
        const int mgroups = (nMt + 7) >> 3;
        kparts = kConsumerWarps / mgroups;
        mg = cw / kparts;
        kp = cw % kparts;
        wact = mg < mgroups;
        rot = 0;
#pragma unroll
        for (int j = 0; j < 8; j++)
#pragma unroll
          for (int q = 0; q < 4; q++) tacc[j][q] = 0.f;
      }
      if (wact && ncols > 0 && ncols <= kMaxCols) {
        const int grp = lane >> 2, tq = lane & 3;
        const int nks = (ncols + 15) >> 4;
        // ldmatrix.x4.trans: lane l addresses row (l & 7) of 8x8 matrix l >> 3;
        // matrix bit 0 = second 8-row group, bit 1 = second 8-column group.
        // Byte offset of (column group kg, row group rg, row r) in the tiled
        // chunk: 2 * (kg * 8 * hpad + rg * 64 + r * 8).
        const int mat = lane >> 3;
        const uint32_t kstep_bytes = 32u * static_cast<uint32_t>(hpad);  // 16 columns
        const uint32_t lane_base = smem_u32(st) + 2u * static_cast<uint32_t>((mat >> 1) * 8 * hpad +
                                                                              (mat & 1) * 64 + (lane & 7) * 8);
        const uint32_t back_k = (mat & 2) ? 16u * static_cast<uint32_t>(hpad) : 0u;  // to group 2ks if absent
        const uint32_t back_m = (mat & 1) ? 128u : 0u;                               // to group 2mt if absent
        // K-steps are dealt round-robin, rotated every chunk so the warps
        // share the remainder evenly over the item's chunks (the rotation
        // depends only on the chunk's place in its item: results do not
        // depend on the schedule).
        int ks = kp - rot;
        if (ks < 0) ks += kparts;
        // the m-tile holding only 8 rows (hpad = 16k + 8), or -1
        const int half_mt = (hpad & 15) ? (hpad >> 4) : -1;
        // K-steps for kNJ active m-tiles of this warp: the tile count is a
        // compile-time constant, so accumulators stay in registers and no
        // slot is predicated off; full K-steps skip the bounds checks.
        auto ksteps = [&](auto nj) {
          constexpr int kNJ = decltype(nj)::value;
          for (; ks < nks; ks += kparts) {
            const bool full = 16 * ks + 16 <= ncols;
            // B fragment: lanes 0-3 hold the BF16-rounded vector (column 0),
            // lanes 4-7 the BF16-rounded remainder (column 1), others zero;
            // the vector arrives as pack_hilo words.
            uint32_t b0 = 0, b1 = 0;
            if (grp < 2) {
              const uint32_t *gw = reinterpret_cast<const uint32_t *>(gs);
              const int c = 16 * ks + 2 * tq;
              uint32_t w0, w1, w2, w3;
              if (full) {
                w0 = gw[c];
                w1 = gw[c + 1];
                w2 = gw[c + 8];
                w3 = gw[c + 9];
              } else {
                w0 = c < ncols ? gw[c] : 0u;
                w1 = c + 1 < ncols ? gw[c + 1] : 0u;
                w2 = c + 8 < ncols ? gw[c + 8] : 0u;
                w3 = c + 9 < ncols ? gw[c + 9] : 0u;
              }
              const uint32_t sel = grp == 0 ? 0x5410u : 0x7632u;  // low halves (hi) or high halves (lo)
              b0 = __byte_perm(w0, w1, sel);
              b1 = __byte_perm(w2, w3, sel);
            }
            const bool k2 = full || 16 * ks + 8 < ncols;  // second 8-column group present
            const uint32_t kaddr = lane_base + static_cast<uint32_t>(ks) * kstep_bytes - (k2 ? 0u : back_k);
#pragma unroll
            for (int j = 0; j < kNJ; j++) {
              const int mt = mg * 8 + j;
              const bool m2 = mt != half_mt;  // second 8-row group present
              uint32_t a0, a1, a2, a3;
              ldmatrix_x4_trans(kaddr + 256u * static_cast<uint32_t>(mt) - (m2 ? 0u : back_m), a0, a1, a2, a3);
              if (!m2) {
                a1 = 0;
                a3 = 0;
              }
              if (!k2) {
                a2 = 0;
                a3 = 0;
              }
              mma_bf16_16816(tacc[j], a0, a1, a2, a3, b0, b1);
            }
          }
        };
        switch (min(8, nMt - mg * 8)) {
          case 1: ksteps(IntC<1>{}); break;
          case 2: ksteps(IntC<2>{}); break;
          case 3: ksteps(IntC<3>{}); break;
          case 4: ksteps(IntC<4>{}); break;
          case 5: ksteps(IntC<5>{}); break;
          case 6: ksteps(IntC<6>{}); break;
          case 7: ksteps(IntC<7>{}); break;
          default: ksteps(IntC<8>{}); break;
        }
      }
    }
    if constexpr (kTensor) rot = rot + 1 == kparts ? 0 : rot + 1;
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (flags & kLast) {
      G *rb = red + (items & 1u) * L::kRedPer;
      int nred;
      if constexpr (!kTensor) {
        if (active) {
#pragma unroll
          for (int r = 0; r < R; r++) rb[cq * hpad + R * rv + r] = acc[r];
        }
        nred = Q;
      } else {
        if (wact && (lane & 3) == 0) {
          const int g8 = lane >> 2;
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const int mt = mg * 8 + j;
            if (mt < nMt) {
              const int row = mt * 16 + g8;
              if (row < hpad) rb[kp * hpad + row] = tacc[j][0] + tacc[j][1];
              if (row + 8 < hpad) rb[kp * hpad + row + 8] = tacc[j][2] + tacc[j][3];
            }
          }
        }
        nred = kparts;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(redbar);
      if (!mbar_wait(redbar, items & 1u, a.spin_limit)) {
        if (lane == 0) set_error(a.err, kErrTimeoutReduce);
        return;
      }
#pragma unroll
      for (int q2 = 0; q2 < 2; q2++) {
        const int r = ct + q2 * kConsumers;
        if (r < rows) {
          G sum = 0;
          for (int q = 0; q < nred; q++) sum += rb[q * hpad + r];
          if (a.phase == 1)
            static_cast<G *>(a.t_out)[out_off + r] = sum;
          else
            a.y_out[pre_dst[q2]] = static_cast<double>(sum);
        }
      }
      items++;
    }
  }
}

// ----------------------------------------------------------------------------- narrow phases
// Items of at most kNarrowRows padded rows (the row panels and B stacks of
// 2DS0-H matrices, 8 to 64 rows) run without staging: ordinary 16-byte loads
// straight from global memory, every row of the item in registers.  The
// CTA-wide kernel above spends a fixed ~1.3 us per chunk on such items (every
// consumer warp takes part in every chunk's barrier round trip and in every
// item's shared-memory reduction, measured with per-chunk clock stamps on the
// 48 x 2DS0 batch).  Two modes, one launch:
//   * CTA-cooperative (queue units [0, n_coop), long units of few rows; only
//     with the narrow_coop tuning, by default those stay in the CTA-wide
//     kernel): the CTA's 16 warps take the unit's chunks round robin, and the
//     warps' rows of each item are added in shared memory, in warp order;
//   * warp per unit (the rest): a warp takes a unit from the queue and writes
//     its outputs itself; nothing is shared between warps.
// After a CTA-wide launch of the same phase it runs as that launch's
// programmatic dependent (pdl_launch_dependents / pdl_wait).
// A warp walks a chunk in rounds: each lane issues all of a round's loads
// (the ones past the chunk's columns predicated off) before it uses any, so
// short chunks keep as many bytes in flight as long ones.  The chunk
// descriptors, the data layout and the vector sources are the ones the
// CTA-wide kernel reads, and an item's arithmetic does not depend on the warp
// or CTA that takes it.
constexpr int kNarrowRows = 64;
constexpr int kNarrowWarps = 16;  // per CTA; two CTAs per SM

// x value of a packed (hi, lo) BF16 word (pack_hilo): hi + lo, exact in FP32.
__device__ __forceinline__ float unpack_hilo(uint32_t w) {
  return __uint_as_float(w << 16) + __uint_as_float(w & 0xffff0000u);
}

// Lanes of a column-major FP64 / FP32 item: R = 16 / es adjacent rows of one
// column slot each; lpc lanes cover the padded rows (a power of two), 32 /
// lpc column slots side by side.
__device__ __forceinline__ int narrow_lpc(int hpad, int R) {
  int lpc = 1;
  while (lpc * R < hpad) lpc <<= 1;
  return lpc;
}

// One chunk of a column-major FP64 / FP32 item: lane (slot, r0) takes columns
// slot, slot + cpp, ... in rounds of kAhead.
template <typename S, int R>
__device__ __forceinline__ void narrow_fma_chunk(const unsigned char *base, const typename Store<S>::G *g, int hpad,
                                                 int ncols, int lpc, int lane, typename Store<S>::G (&acc)[R]) {
  using G = typename Store<S>::G;
  using V = typename std::conditional<sizeof(G) == 8, double2, float4>::type;
  constexpr int kAhead = sizeof(G) == 8 ? 4 : 6;  // 16-byte loads in flight per lane
  const int r0 = (lane % lpc) * R, cpp = 32 / lpc;
  if (r0 >= hpad) return;
  const G *d = reinterpret_cast<const G *>(base) + r0;
#pragma unroll 1
  for (int c = lane / lpc; c < ncols; c += kAhead * cpp) {
    V v[kAhead];
    G x[kAhead];
#pragma unroll
    for (int q = 0; q < kAhead; q++) {
      const int cq = c + q * cpp;
      if (cq < ncols) {
        v[q] = __ldg(reinterpret_cast<const V *>(d + static_cast<long long>(cq) * hpad));
        x[q] = __ldg(g + cq);
      } else {
        v[q] = V{};
        x[q] = 0;
      }
    }
#pragma unroll
    for (int q = 0; q < kAhead; q++) {
      const G *e = reinterpret_cast<const G *>(&v[q]);
#pragma unroll
      for (int k = 0; k < R; k++) acc[k] = fma(e[k], x[q], acc[k]);
    }
  }
}

// Lanes of an 8x8-tiled BF16 item with nrg = hpad / 8 row groups: lane
// (c8, rl, cs) = (lane % 8, (lane / 8) % rgl, lane / (8 rgl)) takes column c8
// of its column groups and the row groups rl (and rl + 4 when nrg > 4); rgl =
// the row-group lanes (nrg rounded up to a power of two, at most 4), and
// 4 / rgl column groups run side by side.  A 16-byte load is 8 rows of one
// column (one tile column).
__device__ __forceinline__ int narrow_rgl(int hpad) {
  const int nrg = hpad >> 3;
  return nrg <= 1 ? 1 : nrg <= 2 ? 2 : 4;
}

// One chunk of an 8x8-tiled BF16 item: lane (c8, rl, cs) takes column groups
// cs, cs + gpw, ... in rounds of kAhead.  Items of at most 4 row groups load
// one tile column per lane and column group (four column groups a round),
// items of 5 to 8 row groups two (two a round).
template <bool kTwo>
__device__ __forceinline__ void narrow_bf16_chunk_t(const uint16_t *base, const uint32_t *g, int hpad, int ncols,
                                                    int lane, float (&acc)[2][8]) {
  constexpr int kAhead = kTwo ? 2 : 4;
  const int nrg = hpad >> 3, rgl = narrow_rgl(hpad), gpw = 4 / rgl;
  const int c8 = lane & 7, rl = (lane >> 3) & (rgl - 1), cs = (lane >> 3) / rgl;
  const int ncg = (ncols + 7) >> 3;
  const bool one = rl < nrg;               // no row group 3 when nrg = 3
  const bool two = kTwo && rl + 4 < nrg;  // a second row group
  const uint16_t *lb = base + c8 * 8 + rl * 64;
#pragma unroll 1
  for (int cg = cs; cg < ncg; cg += kAhead * gpw) {
    float x[kAhead];
    uint4 w[kAhead][kTwo ? 2 : 1];
#pragma unroll
    for (int q = 0; q < kAhead; q++) {
      const int cq = cg + q * gpw, c = 8 * cq + c8;
      const bool in = cq < ncg && c < ncols;  // the tile's padding columns are not read
      const uint16_t *col = lb + static_cast<long long>(cq) * 8 * hpad;
      x[q] = in ? unpack_hilo(__ldg(g + c)) : 0.f;
      w[q][0] = in && one ? __ldg(reinterpret_cast<const uint4 *>(col)) : make_uint4(0, 0, 0, 0);
      if constexpr (kTwo) w[q][1] = in && two ? __ldg(reinterpret_cast<const uint4 *>(col + 256)) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int q = 0; q < kAhead; q++)
#pragma unroll
      for (int j = 0; j < (kTwo ? 2 : 1); j++) {
        const uint32_t ww[4] = {w[q][j].x, w[q][j].y, w[q][j].z, w[q][j].w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
          acc[j][2 * k] = fmaf(__uint_as_float(ww[k] << 16), x[q], acc[j][2 * k]);
          acc[j][2 * k + 1] = fmaf(__uint_as_float(ww[k] & 0xffff0000u), x[q], acc[j][2 * k + 1]);
        }
      }
  }
}

// Sum of a lane's BF16 row partials over the column lanes; lane (c8, rl, cs =
// 0) then holds rows (rl + 4 j) * 8 + c8 in v[j].
__device__ __forceinline__ void narrow_bf16_rows(float (&acc)[2][8], int hpad, int lane, float (&v)[2]) {
  const int rgl = narrow_rgl(hpad), c8 = lane & 7;
#pragma unroll
  for (int j = 0; j < 2; j++)
#pragma unroll
    for (int k = 0; k < 8; k++) {
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) acc[j][k] += __shfl_xor_sync(0xffffffffu, acc[j][k], o);
      for (int o = 8 * rgl; o < 32; o <<= 1) acc[j][k] += __shfl_xor_sync(0xffffffffu, acc[j][k], o);
    }
#pragma unroll
  for (int j = 0; j < 2; j++) {
    v[j] = acc[j][0];
#pragma unroll
    for (int k = 1; k < 8; k++)
      if (c8 == k) v[j] = acc[j][k];
  }
}

template <typename G>
__device__ __forceinline__ void narrow_store(const StreamArgs &a, int out_off, int r, G v) {
  if (a.phase == 1) {
    static_cast<G *>(a.t_out)[out_off + r] = v;
  } else {
    const int row = out_off + r;
    a.y_out[a.perm_out ? static_cast<long long>(a.dof) * a.perm_out[row / a.dof] + (row % a.dof) : row] =
        static_cast<double>(v);
  }
}

struct NarrowChunk {
  long long data_off;
  int ncols, hpad, rows, out_off, g_off;
  uint32_t flags;
};

// Descriptor of chunk i; a malformed one (rows, columns or padded rows out of
// the kernel's range) sets the error word and reads as an empty chunk.
__device__ __forceinline__ NarrowChunk narrow_desc(const StreamArgs &a, int i, bool report) {
  const uint4 *dp = reinterpret_cast<const uint4 *>(a.chunks + i);
  const uint4 w0 = __ldg(dp), w1 = __ldg(dp + 1);
  NarrowChunk c;
  c.data_off = static_cast<long long>((static_cast<unsigned long long>(w0.y) << 32) | w0.x);
  c.ncols = static_cast<int>(w0.z);
  c.hpad = static_cast<int>(w0.w);
  c.rows = static_cast<int>(w1.x);
  c.out_off = static_cast<int>(w1.y);
  c.flags = w1.z;
  c.g_off = static_cast<int>(w1.w);
  if (c.hpad <= 0 || c.hpad > kNarrowRows || (c.hpad & 7) || c.ncols < 0 || c.ncols > kMaxCols || c.rows < 0 ||
      c.rows > c.hpad) {
    if (report) set_error(a.err, kErrBadChunk);
    c.ncols = 0;
    c.hpad = 8;
    c.rows = 0;
  }
  return c;
}

// Per-lane partial rows of an item: R rows (FP64 / FP32) or 2 x 8 (BF16).
template <typename S>
struct NarrowAcc {
  static constexpr bool kTensor = Store<S>::kRows == 0;
  static constexpr int R = kTensor ? 1 : 16 / Store<S>::kEsize;
  typename Store<S>::G acc[R];
  float tacc[2][8];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int k = 0; k < R; k++) acc[k] = 0;
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int k = 0; k < 8; k++) tacc[j][k] = 0.f;
  }
  __device__ __forceinline__ void add_chunk(const StreamArgs &a, const NarrowChunk &d, int lane) {
    using G = typename Store<S>::G;
    const unsigned char *gdata = static_cast<const unsigned char *>(a.data);
    if constexpr (kTensor) {
      const uint16_t *base = reinterpret_cast<const uint16_t *>(gdata) + d.data_off;
      const uint32_t *g = static_cast<const uint32_t *>(a.gsrc) + d.g_off;
      if (d.hpad > 32)
        narrow_bf16_chunk_t<true>(base, g, d.hpad, d.ncols, lane, tacc);
      else
        narrow_bf16_chunk_t<false>(base, g, d.hpad, d.ncols, lane, tacc);
    } else {
      narrow_fma_chunk<S, R>(gdata + d.data_off * Store<S>::kEsize, static_cast<const G *>(a.gsrc) + d.g_off, d.hpad,
                             d.ncols, narrow_lpc(d.hpad, R), lane, acc);
    }
  }
  // The item's rows summed over the warp's lanes; f(r, value) for every row
  // r < hpad, called by one lane per row.
  template <typename F>
  __device__ __forceinline__ void rows(int hpad, int lane, F &&f) {
    if constexpr (kTensor) {
      float v[2];
      narrow_bf16_rows(tacc, hpad, lane, v);
      const int rgl = narrow_rgl(hpad), rl = (lane >> 3) & (rgl - 1), cs = (lane >> 3) / rgl;
      if (cs == 0) {
        const int nrg = hpad >> 3;
        if (rl < nrg) f(rl * 8 + (lane & 7), v[0]);
        if (rl + 4 < nrg) f((rl + 4) * 8 + (lane & 7), v[1]);
      }
    } else {
      const int lpc = narrow_lpc(hpad, R);
      for (int o = lpc; o < 32; o <<= 1)
#pragma unroll
        for (int k = 0; k < R; k++) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
      if (lane < lpc) {
#pragma unroll
        for (int k = 0; k < R; k++)
          if (lane * R + k < hpad) f(lane * R + k, acc[k]);
      }
    }
  }
};

// Warp per unit: the warp walks the unit's chunks in order and writes each
// item's rows at its last chunk.
template <typename S>
__device__ __forceinline__ void narrow_unit_warp(const StreamArgs &a, int cb, int ce, int lane) {
  using G = typename Store<S>::G;
  NarrowAcc<S> ac;
  for (int i = cb; i < ce; i++) {
    const NarrowChunk d = narrow_desc(a, i, lane == 0);
    if (d.flags & kFirst) ac.zero();
    ac.add_chunk(a, d, lane);
    if (d.flags & kLast)
      ac.rows(d.hpad, lane, [&](int r, G v) {
        if (r < d.rows) narrow_store<G>(a, d.out_off, r, v);
      });
  }
}

// CTA per unit: item by item, warp w takes the item's chunks w, w + 16, ...,
// then the warps' rows meet in red (kNarrowWarps x kNarrowRows) and are summed
// in warp order.  Every thread of the CTA calls it.
template <typename S>
__device__ __forceinline__ void narrow_unit_cta(const StreamArgs &a, int cb, int ce, int lane, int wid,
                                                typename Store<S>::G *red) {
  using G = typename Store<S>::G;
  int i0 = cb;
  while (i0 < ce) {
    int i1 = i0;  // the item's last chunk
    while (i1 + 1 < ce && !(__ldg(&a.chunks[i1].flags) & kLast)) i1++;
    const NarrowChunk last = narrow_desc(a, i1, false);
    NarrowAcc<S> ac;
    ac.zero();
    for (int i = i0 + wid; i <= i1; i += kNarrowWarps) {
      const NarrowChunk d = narrow_desc(a, i, lane == 0);
      if (d.hpad == last.hpad) ac.add_chunk(a, d, lane);
    }
    ac.rows(last.hpad, lane, [&](int r, G v) { red[wid * kNarrowRows + r] = v; });
    __syncthreads();
    const int r = threadIdx.x;
    if (r < last.rows) {
      G sum = red[r];
      for (int w = 1; w < kNarrowWarps; w++) sum += red[w * kNarrowRows + r];
      narrow_store<G>(a, last.out_off, r, sum);
    }
    __syncthreads();
    i0 = i1 + 1;
  }
}

template <typename S>
__global__ void __launch_bounds__(32 * kNarrowWarps, 2) narrow_items_kernel(StreamArgs a) {
  using G = typename Store<S>::G;
  __shared__ G red[kNarrowWarps * kNarrowRows];
  __shared__ int unit;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // queue units [0, n_coop): the whole CTA per unit (queue[2] counts them)
  for (;;) {
    if (threadIdx.x == 0) unit = atomicAdd(&a.queue[2], 1);
    __syncthreads();
    const int u = unit;
    __syncthreads();
    if (u >= a.n_coop) break;
    narrow_unit_cta<S>(a, __ldg(a.item_ptr + u), __ldg(a.item_ptr + u + 1), lane, wid, red);
  }
  // the rest: warp per unit (queue[0] counts them)
  for (;;) {
    int it = 0;
    if (lane == 0) it = a.n_coop + atomicAdd(&a.queue[0], 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= a.n_items) break;
    narrow_unit_warp<S>(a, __ldg(a.item_ptr + it), __ldg(a.item_ptr + it + 1), lane);
  }
  // This CTA takes no more units; the last CTA returns the queue to zero.
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.queue[1], 1) == static_cast<int>(gridDim.x) - 1) {
      a.queue[0] = 0;
      a.queue[1] = 0;
      a.queue[2] = 0;
      __threadfence();
    }
  }
  // Launched programmatically after the phase's CTA-wide launch (whose
  // outputs it neither reads nor writes), this launch completes only after
  // that one has: the next launch on the stream sees both phases' outputs.
  pdl_wait();
}

// BF16 path: a vector value v is handed to the tensor cores as two BF16
// numbers, hi = bf16(v) and lo = bf16(v - hi), packed in one word (hi in the
// low half), so the consumers build mma B fragments with a byte permute.
__device__ __forceinline__ uint32_t pack_hilo(float v) {
  const float hi = __bfloat162float(__float2bfloat16_rn(v));
  return pack_bf16x2(hi, v - hi);
}

// G2[dst + c] = scale * src[src_off + c] for every run (src: gathered x or t):
// the phase-2 vector values laid out chunk by chunk.  Runs are short (10 to
// 60 values), so a warp takes kG2Runs = 32 of them at once and deals their
// values to its lanes densely: lane k loads run k's descriptor and a warp
// scan gives each run its first position in the warp's value list.  A round
// covers 32 consecutive positions [w0, w0 + 32): the run holding w0 is the
// last one starting at or before it (one ballot), every later run starting
// inside the window sets its bit in a 32-bit mask (one OR reduction), and the
// value at w0 + j belongs to the run holding w0 plus the number of bits at or
// below j.  This needs the runs to be non-empty, which the layout guarantees
// (build_chunks makes no empty run); a value whose run does not hold it is
// skipped, so malformed runs cannot index outside their source or G2.
// kPacked: store pack_hilo(value) words (BF16 path) instead of G values, and
// apply the runs' block scales (1 on the other paths).
constexpr int kG2Runs = 32;
constexpr int kG2Unroll = 4;  // rounds in flight per lane

template <typename G, bool kPacked>
__global__ void gather_g2_kernel(const GatherSeg *__restrict__ runs, int n_runs, const G *__restrict__ xp,
                                 const G *__restrict__ t, void *__restrict__ g2) {
  const int lane = threadIdx.x & 31;
  const int r0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kG2Runs;
  if (r0 >= n_runs) return;  // warp-uniform
  GatherSeg mine{};          // cols = 0 past the end
  if (r0 + lane < n_runs) mine = runs[r0 + lane];
  const int cols = static_cast<int>(mine.cols_src & 0x7fffffffu);
  int incl = cols;  // inclusive scan of the run lengths over the lanes
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int start = incl - cols;
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  const unsigned below = (2u << lane) - 1u;  // bits 0..lane
  for (int base = 0; base < total; base += 32 * kG2Unroll) {
    G v[kG2Unroll];
    int dst[kG2Unroll];
    float sc[kG2Unroll];
    bool ok[kG2Unroll];
#pragma unroll
    for (int u = 0; u < kG2Unroll; u++) {
      const int w0 = base + 32 * u, e = w0 + lane;
      const unsigned holds = __ballot_sync(0xffffffffu, cols > 0 && start <= w0);
      const int off = start - w0;
      const unsigned starts = __reduce_or_sync(0xffffffffu, (cols > 0 && off > 0 && off < 32) ? (1u << off) : 0u);
      const int r = (holds ? 31 - __clz(holds) : 0) + __popc(starts & below);
      const int rs = __shfl_sync(0xffffffffu, start, r);
      const int rc = __shfl_sync(0xffffffffu, cols, r);
      const int ro = __shfl_sync(0xffffffffu, mine.src_off, r);
      const uint32_t rf = __shfl_sync(0xffffffffu, mine.cols_src, r);
      const int rd = __shfl_sync(0xffffffffu, mine.dst, r);
      sc[u] = kPacked ? __shfl_sync(0xffffffffu, mine.scale, r) : 1.0f;
      const int k = e - rs;
      ok[u] = e < total && k >= 0 && k < rc;
      dst[u] = rd + k;
      v[u] = ok[u] ? ((rf >> 31) ? t : xp)[ro + k] : G(0);
    }
#pragma unroll
    for (int u = 0; u < kG2Unroll; u++) {
      if (ok[u]) {
        if constexpr (kPacked)
          static_cast<uint32_t *>(g2)[dst[u]] = pack_hilo(sc[u] * static_cast<float>(v[u]));
        else
          static_cast<G *>(g2)[dst[u]] = v[u];
      }
    }
  }
}

// x (FP64, caller's ordering) -> gathered copy in the compute type, permuted
// order: xp[dof*i + j] = x[dof*perm[i] + j] (Hmat::matvecOriginal,
// src/hmat/hmatrix/hmat.cc:586-593), or a plain cast when perm is null.
// xpk (BF16 path, else null) receives the same values as pack_hilo words.
template <typename G>
__global__ void gather_x_kernel(const double *__restrict__ x, G *__restrict__ xp, uint32_t *__restrict__ xpk,
                                const int32_t *__restrict__ perm, int dof, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int src = perm ? dof * perm[i / dof] + (i % dof) : i;
  const G v = static_cast<G>(x[src]);
  xp[i] = v;
  if (xpk) xpk[i] = pack_hilo(static_cast<float>(v));
}

}  // namespace bw
