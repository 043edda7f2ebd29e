// Device code of the streamed H-matrix matvec (sm_100a).
//
// One persistent kernel per phase (see bw_layout.h).  Each CTA owns a fixed,
// host-scheduled list of chunks.  Warp 0 is the producer: for every chunk it
// stages the block data with one TMA bulk copy (cp.async.bulk, 16-byte aligned
// window around the chunk) and gathers the chunk's vector values with
// cp.async, into a ring of kStages shared-memory stages guarded by mbarriers.
// Warps 1..8 are consumers: each thread owns two adjacent rows of the item and
// a contiguous range of the chunk's columns, accumulates in registers, and at
// the item's last chunk the column partial sums are reduced in shared memory
// and written once (t for phase 1, y for phase 2, with the row permutation
// applied on the fly).  Every wait is a bounded mbarrier try_wait loop; on
// timeout the kernel records an error word and returns.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "bw_layout.h"

namespace bw {

constexpr int kStages = 5;
constexpr int kConsumerWarps = 8;
constexpr int kConsumers = 32 * kConsumerWarps;
constexpr int kThreads = 32 + kConsumers;

// error words
constexpr int kErrTimeoutEmpty = 0x101;
constexpr int kErrTimeoutFull = 0x102;
constexpr int kErrTimeoutReduce = 0x103;
constexpr int kErrBadChunk = 0x104;

struct StreamArgs {
  const void *data;           // element array of the phase (storage type)
  const Chunk *chunks;        // ordered by CTA
  const int32_t *cta_ptr;     // grid + 1
  const void *xsrc;           // gathered x (compute type), permuted order
  const void *tsrc;           // t (compute type)
  void *t_out;                // phase-1 output (compute type)
  double *y_out;              // phase-2 output
  const int32_t *perm_out;    // phase 2: point permutation of the output, or null
  int dof;
  int phase;                  // 1 or 2
  int *err;
  long long spin_limit;        // bound of every wait, in nanoseconds
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
__device__ __forceinline__ void cp_async_4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// Arrive on `bar` once this thread's earlier cp.async copies have landed
// (counts against the barrier's expected arrivals).
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait: returns false when `limit_ns` nanoseconds passed without the
// phase completing.
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

// ----------------------------------------------------------------------------- storage traits
struct Bf16 {};  // storage tag: 16-bit brain float with per-chunk FP32 scale

template <typename S> struct Store;
template <> struct Store<double> {
  using G = double;   // compute / gather type
  static constexpr int kEsize = 8;
};
template <> struct Store<float> {
  using G = float;
  static constexpr int kEsize = 4;
};
template <> struct Store<Bf16> {
  using G = float;
  static constexpr int kEsize = 2;
};

// Partial sums of two adjacent rows over columns [c0, c1) of a staged chunk.
// `base` points at the chunk's first element in shared memory; pair p of
// column c is at element 2 * (c * hp + p).
template <typename S>
__device__ __forceinline__ void chunk_dot(const unsigned char *base, const typename Store<S>::G *g, int hp, int rp,
                                          int c0, int c1, typename Store<S>::G &o0, typename Store<S>::G &o1);

template <>
__device__ __forceinline__ void chunk_dot<double>(const unsigned char *base, const double *g, int hp, int rp, int c0,
                                                  int c1, double &o0, double &o1) {
  const double2 *d = reinterpret_cast<const double2 *>(base) + rp;
  double a0 = 0, a1 = 0, b0 = 0, b1 = 0;
  int c = c0;
#pragma unroll 1
  for (; c + 4 <= c1; c += 4) {
    const double2 w0 = d[(c + 0) * hp], w1 = d[(c + 1) * hp], w2 = d[(c + 2) * hp], w3 = d[(c + 3) * hp];
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
    const double2 w = d[c * hp];
    a0 = fma(w.x, g[c], a0);
    a1 = fma(w.y, g[c], a1);
  }
  o0 = a0 + b0;
  o1 = a1 + b1;
}

template <>
__device__ __forceinline__ void chunk_dot<float>(const unsigned char *base, const float *g, int hp, int rp, int c0,
                                                 int c1, float &o0, float &o1) {
  const float2 *d = reinterpret_cast<const float2 *>(base) + rp;
  float a0 = 0, a1 = 0, b0 = 0, b1 = 0;
  int c = c0;
#pragma unroll 1
  for (; c + 4 <= c1; c += 4) {
    const float2 w0 = d[(c + 0) * hp], w1 = d[(c + 1) * hp], w2 = d[(c + 2) * hp], w3 = d[(c + 3) * hp];
    const float g0 = g[c], g1 = g[c + 1], g2 = g[c + 2], g3 = g[c + 3];
    a0 = fmaf(w0.x, g0, a0);
    a1 = fmaf(w0.y, g0, a1);
    b0 = fmaf(w1.x, g1, b0);
    b1 = fmaf(w1.y, g1, b1);
    a0 = fmaf(w2.x, g2, a0);
    a1 = fmaf(w2.y, g2, a1);
    b0 = fmaf(w3.x, g3, b0);
    b1 = fmaf(w3.y, g3, b1);
  }
  for (; c < c1; c++) {
    const float2 w = d[c * hp];
    a0 = fmaf(w.x, g[c], a0);
    a1 = fmaf(w.y, g[c], a1);
  }
  o0 = a0 + b0;
  o1 = a1 + b1;
}

__device__ __forceinline__ float bf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

template <>
__device__ __forceinline__ void chunk_dot<Bf16>(const unsigned char *base, const float *g, int hp, int rp, int c0,
                                                int c1, float &o0, float &o1) {
  const uint32_t *d = reinterpret_cast<const uint32_t *>(base) + rp;
  float a0 = 0, a1 = 0, b0 = 0, b1 = 0;
  int c = c0;
#pragma unroll 1
  for (; c + 4 <= c1; c += 4) {
    const uint32_t w0 = d[(c + 0) * hp], w1 = d[(c + 1) * hp], w2 = d[(c + 2) * hp], w3 = d[(c + 3) * hp];
    const float g0 = g[c], g1 = g[c + 1], g2 = g[c + 2], g3 = g[c + 3];
    a0 = fmaf(bf_lo(w0), g0, a0);
    a1 = fmaf(bf_hi(w0), g0, a1);
    b0 = fmaf(bf_lo(w1), g1, b0);
    b1 = fmaf(bf_hi(w1), g1, b1);
    a0 = fmaf(bf_lo(w2), g2, a0);
    a1 = fmaf(bf_hi(w2), g2, a1);
    b0 = fmaf(bf_lo(w3), g3, b0);
    b1 = fmaf(bf_hi(w3), g3, b1);
  }
  for (; c < c1; c++) {
    const uint32_t w = d[c * hp];
    a0 = fmaf(bf_lo(w), g[c], a0);
    a1 = fmaf(bf_hi(w), g[c], a1);
  }
  o0 = a0 + b0;
  o1 = a1 + b1;
}

// ----------------------------------------------------------------------------- shared memory
template <typename S> struct SmemLayout {
  using G = typename Store<S>::G;
  static constexpr int kDataBytes = kStageBytes + 32;
  static constexpr int kGBytes = kMaxCols * sizeof(G);
  static constexpr int kStageSize = kDataBytes + kGBytes + (int)sizeof(Chunk);
  static constexpr int kRedBytes = 2 * 2 * kConsumers * (int)sizeof(G);  // double-buffered [Q][hpad]
  static constexpr int kBarBytes = (2 * kStages + 1) * 8;
  static constexpr int kTotal = kStages * kStageSize + kRedBytes + kBarBytes;
  static_assert(kStageSize % 16 == 0, "stage must keep 16-byte alignment");
};

// Words 0..15 of a descriptor, broadcast from lane `src`.
struct DescRegs {
  uint32_t w[16];
};

__device__ __forceinline__ void load_desc_batch(const Chunk *chunks, int idx, int end, DescRegs &r) {
  if (idx < end) {
    const uint4 *p = reinterpret_cast<const uint4 *>(chunks + idx);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint4 v = __ldg(p + k);
      r.w[4 * k + 0] = v.x;
      r.w[4 * k + 1] = v.y;
      r.w[4 * k + 2] = v.z;
      r.w[4 * k + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 16; k++) r.w[k] = 0;
  }
}

template <typename S>
__global__ void __launch_bounds__(kThreads, 1) stream_panels_kernel(StreamArgs a) {
  using G = typename Store<S>::G;
  using L = SmemLayout<S>;
  constexpr int es = Store<S>::kEsize;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *stage0 = smem;
  G *red = reinterpret_cast<G *>(smem + kStages * L::kStageSize);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + kStages * L::kStageSize + L::kRedBytes);
  uint64_t *empty = full + kStages;
  uint64_t *redbar = empty + kStages;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 33);                 // lane-0 arrive(.expect_tx) + 32 cp.async arrivals
      mbar_init(&empty[s], kConsumerWarps);    // one arrival per consumer warp
    }
    mbar_init(redbar, kConsumerWarps);
    fence_barrier_init();
  }
  __syncthreads();

  const int cb = a.cta_ptr[blockIdx.x], ce = a.cta_ptr[blockIdx.x + 1];
  if (cb >= ce) return;

  if (warp == 0) {
    // ------------------------------------------------------------------ producer
    const unsigned char *gdata = static_cast<const unsigned char *>(a.data);
    const G *xs = static_cast<const G *>(a.xsrc);
    const G *ts = static_cast<const G *>(a.tsrc);
    DescRegs cur, nxt;
    load_desc_batch(a.chunks, cb + lane, ce, nxt);
    bool ok = true;
    int issued = 0;
    for (int bb = cb; bb < ce && ok; bb += 32) {
      cur = nxt;
      load_desc_batch(a.chunks, bb + 32 + lane, ce, nxt);
      const int nb = min(32, ce - bb);
      for (int k = 0; k < nb; k++) {
        const int i = bb + k - cb;
        const int s = i % kStages;
        const uint32_t use = static_cast<uint32_t>(i / kStages);
        if (!mbar_wait(&empty[s], (use & 1u) ^ 1u, a.spin_limit)) {
          if (lane == 0) set_error(a.err, kErrTimeoutEmpty);
          ok = false;
          break;
        }
        uint32_t w[16];
#pragma unroll
        for (int q = 0; q < 16; q++) w[q] = __shfl_sync(0xffffffffu, cur.w[q], k);
        const long long data_off = static_cast<long long>((static_cast<unsigned long long>(w[1]) << 32) | w[0]);
        const int ncols = static_cast<int>(w[2]);
        const int hpad = static_cast<int>(w[3]);
        const uint32_t flags = w[7];
        unsigned char *st = stage0 + s * L::kStageSize;
        G *gs = reinterpret_cast<G *>(st + L::kDataBytes);
        if (lane == 0) {
          uint4 *dd = reinterpret_cast<uint4 *>(st + L::kDataBytes + L::kGBytes);
#pragma unroll
          for (int q = 0; q < 4; q++) dd[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
          const unsigned long long bytes = static_cast<unsigned long long>(ncols) * hpad * es;
          if (ncols > 0 && bytes <= static_cast<unsigned long long>(kStageBytes)) {
            const unsigned long long src = reinterpret_cast<unsigned long long>(gdata) +
                                           static_cast<unsigned long long>(data_off) * es;
            const unsigned long long lo = src & ~15ull;
            const unsigned long long hi = (src + bytes + 15ull) & ~15ull;
            mbar_arrive_expect_tx(&full[s], static_cast<uint32_t>(hi - lo));
            bulk_g2s(st, reinterpret_cast<const void *>(lo), static_cast<uint32_t>(hi - lo), &full[s]);
          } else {
            if (ncols > 0) set_error(a.err, kErrBadChunk);
            mbar_arrive(&full[s]);
          }
        }
        // gather the chunk's vector values
        const int nseg = static_cast<int>((flags >> 8) & 0xfu);
        const int e0 = static_cast<int>(w[12] & 0xffffu);
        const int e1 = e0 + static_cast<int>(w[12] >> 16);
        const int e2 = e1 + static_cast<int>(w[13] & 0xffffu);
        const int gcols = ncols <= kMaxCols ? ncols : 0;
        for (int c = lane; c < gcols; c += 32) {
          const int sg = (c >= e0) + (c >= e1) + (c >= e2);
          const int start = sg == 0 ? 0 : (sg == 1 ? e0 : (sg == 2 ? e1 : e2));
          if (sg < nseg) {
            const G *src = ((flags >> (16 + sg)) & 1u) ? ts : xs;
            const uint32_t so = sg == 0 ? w[8] : (sg == 1 ? w[9] : (sg == 2 ? w[10] : w[11]));
            const G *p = src + static_cast<int>(so) + (c - start);
            if (sizeof(G) == 8)
              cp_async_8(gs + c, p);
            else
              cp_async_4(gs + c, p);
          }
        }
        cp_async_arrive_noinc(&full[s]);
        issued++;
      }
    }
    if (!ok) {
      // let the copies already in flight land before the CTA can exit
      for (int i = max(0, issued - kStages); i < issued; i++) {
        const int s = i % kStages;
        mbar_wait(&full[s], static_cast<uint32_t>(i / kStages) & 1u, a.spin_limit);
      }
    }
    return;
  }

  // -------------------------------------------------------------------- consumers
  const int ct = threadIdx.x - 32;
  int hp = 1, Q = 1, rp = 0, cq = 0;
  bool active = false;
  G acc0 = 0, acc1 = 0;
  uint32_t items = 0;
  for (int i = 0; i < ce - cb; i++) {
    const int s = i % kStages;
    const uint32_t use = static_cast<uint32_t>(i / kStages);
    if (!mbar_wait(&full[s], use & 1u, a.spin_limit)) {
      if (lane == 0) set_error(a.err, kErrTimeoutFull);
      return;
    }
    const unsigned char *st = stage0 + s * L::kStageSize;
    const G *gs = reinterpret_cast<const G *>(st + L::kDataBytes);
    const Chunk &d = *reinterpret_cast<const Chunk *>(st + L::kDataBytes + L::kGBytes);
    const uint32_t flags = d.flags;
    const int ncols = d.ncols;
    const int hpad = d.hpad;
    if (flags & kFirst) {
      hp = hpad >> 1;
      Q = kConsumers / hp;
      rp = ct % hp;
      cq = ct / hp;
      active = cq < Q;
      acc0 = 0;
      acc1 = 0;
    }
    if (active && ncols > 0 && ncols <= kMaxCols) {
      const int c0 = (cq * ncols) / Q, c1 = ((cq + 1) * ncols) / Q;
      const int soff = static_cast<int>((static_cast<unsigned long long>(d.data_off) * es) & 15ull);
      G p0, p1;
      chunk_dot<S>(st + soff, gs, hp, rp, c0, c1, p0, p1);
      const G sc = static_cast<G>(d.scale);
      acc0 += sc * p0;
      acc1 += sc * p1;
    }
    const int rows = d.rows, out_off = d.out_off;
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (flags & kLast) {
      G *rb = red + (items & 1u) * (2 * kConsumers);
      if (active) {
        rb[cq * hpad + 2 * rp] = acc0;
        rb[cq * hpad + 2 * rp + 1] = acc1;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(redbar);
      if (!mbar_wait(redbar, items & 1u, a.spin_limit)) {
        if (lane == 0) set_error(a.err, kErrTimeoutReduce);
        return;
      }
      for (int r = ct; r < rows; r += kConsumers) {
        G sum = 0;
        for (int q = 0; q < Q; q++) sum += rb[q * hpad + r];
        if (a.phase == 1) {
          static_cast<G *>(a.t_out)[out_off + r] = sum;
        } else {
          const int row = out_off + r;
          long long dst = row;
          if (a.perm_out) dst = static_cast<long long>(a.dof) * a.perm_out[row / a.dof] + (row % a.dof);
          a.y_out[dst] = static_cast<double>(sum);
        }
      }
      items++;
    }
  }
}

// x (FP64, caller's ordering) -> gathered copy in the compute type, permuted
// order: xp[dof*i + j] = x[dof*perm[i] + j] (Hmat::matvecOriginal,
// src/hmat/hmatrix/hmat.cc:586-593), or a plain cast when perm is null.
template <typename G>
__global__ void gather_x_kernel(const double *__restrict__ x, G *__restrict__ xp, const int32_t *__restrict__ perm,
                                int dof, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int src = perm ? dof * perm[i / dof] + (i % dof) : i;
  xp[i] = static_cast<G>(x[src]);
}

}  // namespace bw
