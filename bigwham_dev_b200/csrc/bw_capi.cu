// C ABI of the B200 H-matrix backend (declarations: include/bigwham_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "bigwham_b200.h"
#include "bw_kernels.cuh"
#include "bw_mm_kernels.cuh"
#include "bw_aca_kernels.cuh"
#include "bw_assemble_kernels.cuh"
#include "bw_devlayout_kernels.cuh"
#include "bw_fields_kernels.cuh"
#include "bw_file.h"
#include "bw_layout.h"

namespace {

using bw::Chunk;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct OomError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct StateError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct UnsupportedError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define BW_CUDA(call)                                                                             \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

std::mutex g_err_mu;
std::string g_last_create_error;

int prec_index(int flags) {
  const int p = flags & (BW_FP64 | BW_FP32 | BW_BF16);
  if (p == BW_FP64) return 0;
  if (p == BW_FP32) return 1;
  if (p == BW_BF16) return 2;
  return -1;
}

// launches of one matvec: x gather, phase 1, G2 gather, phase 2
// Timed spans of one matvec: x gather, phase 1 CTA-wide, phase 1 unstaged,
// G2 gather, phase 2 CTA-wide, phase 2 unstaged.
constexpr int kTimedLaunches = 6;
constexpr size_t kEv = kTimedLaunches + 1;

struct DevPhase {
  void *data = nullptr;
  Chunk *chunks = nullptr;
  int32_t *items = nullptr;        // chunk ranges of the items, in the order CTAs take them
  int *queue = nullptr;            // [next item, CTAs done], zero between launches
  bw::GatherSeg *gsegs = nullptr;  // phase 2: runs that fill G2
  int64_t n_chunks = 0;
  int64_t n_items = 0;
  int64_t n_elems = 0;
  int64_t n_gsegs = 0;
  // Queue units [0, split.wide) run in the CTA-wide kernel, the rest in the
  // warp-per-item kernel, [split.wide, split.coop) CTA-cooperatively.
  bw::NarrowSplit split;
};

// Device data of one matmat phase (bw::MmPlan).
struct DevMm {
  uint16_t *data = nullptr;
  bw::MmChunk *chunks = nullptr;
  int32_t *items = nullptr;  // chunk ranges of the items, longest first
  int *queue = nullptr;      // [next item, CTAs done], zero between launches
  int64_t n_chunks = 0;
  int64_t n_items = 0;
};

}  // namespace

struct bw_hmat {
  int device = -1;
  int dof = 1;
  int64_t n_rows = 0, n_cols = 0;
  std::vector<int64_t> perm0, perm1;
  std::vector<int64_t> row_off, col_off;  // member k: rows [row_off[k], row_off[k+1]) (bw_create_batch)
  bw::Problem prob;
  bool finalized = false;
  bool plan_only = false;
  int stored = 0;          // precision mask
  bool has_t = false;      // transposed operator stored
  int grid = 148;
  bw::OperatorPlan op[2];  // forward, transposed
  DevPhase dev[2][3][2];   // [operator][precision][phase]
  std::vector<unsigned char> host_data[2][3][2];  // BW_PLAN_ONLY
  bool has_mm = false;     // matmat layout stored (BW_STORE_MATMAT)
  bw::MmPlan mm[2];        // forward, transposed
  DevMm dmm[2][2];         // [operator][phase]
  std::vector<uint16_t> mm_host[2][2];  // BW_PLAN_ONLY
  uint16_t *d_xt = nullptr, *d_t8 = nullptr;  // matmat operands (8x8 BF16 tiles, bw::kMmRhs columns)
  int32_t *d_perm0 = nullptr, *d_perm1 = nullptr;
  void *d_xp = nullptr, *d_t = nullptr, *d_g2 = nullptr;
  double *d_xh = nullptr, *d_yh = nullptr;
  double *h_xpin = nullptr, *h_ypin = nullptr;  // pinned staging of bw_matvec_host
  cudaEvent_t y_ready[4] = {nullptr, nullptr, nullptr, nullptr};  // bw_matvec_host: output pieces landed
  int *d_err = nullptr;
  int *h_err = nullptr;    // pinned
  cudaStream_t stream = nullptr;
  int64_t dev_bytes = 0, dev_limit = 0;
  int64_t entries = 0, sum_rank = 0;
  int64_t n_fr = 0, n_lr = 0;
  std::vector<double> diag_perm;
  std::string err;
  long long spin_limit = 2000000000LL;  // 2 s bound on every in-kernel wait
  int withhold = -1;                    // bw_test_withhold_chunk: applies to the next streaming launch only
  std::shared_ptr<void> borrowed;       // mapped block file the registered blocks point into (until finalize)
  // bw_add_flat_device: the blocks live in these device arrays (flat layout)
  const double *dev_fr = nullptr, *dev_lr = nullptr;
  int64_t dev_fr_len = 0, dev_lr_len = 0;
  std::vector<double> dev_max_fr, dev_max_a, dev_max_b;  // per-block maxima (device pass)
  std::vector<int> dev_bad_fr, dev_bad_lr;
  int take_withhold() {
    const int w = withhold;
    withhold = -1;
    return w;
  }
  // optional per-launch timing (bw_set_timing / bw_timing_read)
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;     // kTimedLaunches + 1 events per recorded matvec
  size_t ev_used = 0;                   // matvecs recorded since the last read

  cudaEvent_t *timing_slot() {
    if (!timing) return nullptr;
    const size_t kMax = 200000;
    if (ev_used >= kMax) return nullptr;
    if (kEv * (ev_used + 1) > ev_pool.size()) {
      const size_t grow = std::max<size_t>(64, ev_pool.size() / kEv);
      for (size_t i = 0; i < kEv * grow; i++) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) throw CudaError("cudaEventCreate failed");
        ev_pool.push_back(e);
      }
    }
    return &ev_pool[kEv * ev_used++];
  }

  void *dmalloc(size_t bytes) {
    if (dev_limit > 0 && dev_bytes + (int64_t)bytes > dev_limit)
      throw OomError("device allocation of " + std::to_string(bytes) + " bytes exceeds the configured limit");
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw OomError("cudaMalloc(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    dev_bytes += (int64_t)bytes;
    return p;
  }
  void release() {
    if (device >= 0) cudaSetDevice(device);
    for (auto &o : dev)
      for (auto &p : o)
        for (auto &ph : p) {
          cudaFree(ph.data);
          cudaFree(ph.chunks);
          cudaFree(ph.items);
          cudaFree(ph.queue);
          cudaFree(ph.gsegs);
          ph = DevPhase{};
        }
    for (auto &o : dmm)
      for (auto &ph : o) {
        cudaFree(ph.data);
        cudaFree(ph.chunks);
        cudaFree(ph.items);
        cudaFree(ph.queue);
        ph = DevMm{};
      }
    cudaFree(d_xt);
    cudaFree(d_t8);
    d_xt = d_t8 = nullptr;
    cudaFree(d_perm0);
    cudaFree(d_perm1);
    cudaFree(d_xp);
    cudaFree(d_t);
    cudaFree(d_g2);
    cudaFree(d_xh);
    cudaFree(d_yh);
    if (h_xpin) cudaFreeHost(h_xpin);
    if (h_ypin) cudaFreeHost(h_ypin);
    h_xpin = h_ypin = nullptr;
    for (cudaEvent_t &e : y_ready) {
      if (e) cudaEventDestroy(e);
      e = nullptr;
    }
    cudaFree(d_err);
    if (h_err) cudaFreeHost(h_err);
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    ev_pool.clear();
    ev_used = 0;
    if (stream) cudaStreamDestroy(stream);
    d_perm0 = d_perm1 = nullptr;
    d_xp = d_t = d_g2 = nullptr;
    d_xh = d_yh = nullptr;
    d_err = nullptr;
    h_err = nullptr;
    stream = nullptr;
    dev_bytes = 0;
  }
};

namespace {

template <typename F> int guarded(bw_hmat *h, F &&f) {
  try {
    return f();
  } catch (const OomError &e) {
    if (h) h->err = e.what();
    return BW_ERR_OOM;
  } catch (const CudaError &e) {
    if (h) h->err = e.what();
    return BW_ERR_CUDA;
  } catch (const StateError &e) {
    if (h) h->err = e.what();
    return BW_ERR_STATE;
  } catch (const UnsupportedError &e) {
    if (h) h->err = e.what();
    return BW_ERR_UNSUPPORTED;
  } catch (const std::bad_alloc &) {
    if (h) h->err = "host allocation failed";
    return BW_ERR_OOM;
  } catch (const std::exception &e) {
    if (h) h->err = e.what();
    return BW_ERR_ARG;
  }
}

// Dynamic shared-memory opt-in of a kernel, set once per device.  The flags
// are guarded by one mutex: first calls from several host threads (one per
// device, or several handles on one device) do not race on them.
std::mutex g_attr_mu;

template <typename K> void smem_attr_once(bool (&done)[64], K kernel, int bytes) {
  int dev = 0;
  BW_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(g_attr_mu);
  if (dev < 64 && done[dev]) return;
  BW_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  if (dev < 64) done[dev] = true;
}

template <typename S> void set_smem_attr() {
  static bool done[64] = {};
  smem_attr_once(done, bw::stream_panels_kernel<S>, bw::SmemLayout<S>::kTotal);
}

int64_t align256(int64_t v) { return (v + 255) / 256 * 256; }

// dst[0:n] = src[0:n] with up to 8 host threads (a vector of 1.5 MB copies in
// ~20 us instead of ~150 us on one thread).
void host_copy(double *dst, const double *src, int64_t n) {
  const int64_t kPart = 8192;  // doubles per thread's part (64 KB)
  const int64_t parts = (n + kPart - 1) / kPart;
#pragma omp parallel for num_threads(8) schedule(static) if (parts > 1)
  for (int64_t p = 0; p < parts; p++) {
    const int64_t a = p * kPart, b = std::min<int64_t>(n, a + kPart);
    std::memcpy(dst + a, src + a, (size_t)(b - a) * 8);
  }
}

// dst[0:bytes] = 0 with all host threads (staging pieces are 256 MB).
void par_zero(void *dst, size_t bytes) {
  const size_t kPart = size_t(4) << 20;
  const int64_t parts = (int64_t)((bytes + kPart - 1) / kPart);
#pragma omp parallel for schedule(static) if (parts > 1)
  for (int64_t p = 0; p < parts; p++) {
    const size_t a = (size_t)p * kPart, b = std::min(bytes, a + kPart);
    std::memset(static_cast<unsigned char *>(dst) + a, 0, b - a);
  }
}

// Bytes of the gathered-x region for a precision: the G values (+16 bytes,
// vector runs are staged in 16-byte aligned windows) and, for BF16, a second
// array of packed hi/lo words at the next 256-byte boundary.
int64_t xp_region_bytes(int prec, int64_t nin) {
  if (prec == 2) return align256(4 * nin + 16) + 4 * nin + 16;
  return nin * (prec == 0 ? 8 : 4) + 16;
}

// Bytes of the phase-2 gather array G2 over the stored precisions and operators.
int64_t g2_bytes(const bw_hmat *h, int mask, bool with_t) {
  int64_t b = 0;
  for (int o = 0; o < (with_t ? 2 : 1); o++)
    for (int p = 0; p < 3; p++)
      if (mask & (1 << p)) b = std::max<int64_t>(b, h->op[o].ph[1].cp[p].g_len * (p == 0 ? 8 : 4));
  return b;
}

// Copies an array of `n_elems` elements of `es` bytes to `dev`, built on the
// host in pieces of whole items through two pinned staging buffers:
// item_start(q) is the first element of item q (item_start(nit) = end of the
// last item), fill(q0, q1, e0, dst) writes items [q0, q1) into zeroed dst whose
// first element is element e0.  The slack after the last item is zeroed.
template <typename StartF, typename FillF>
void staged_upload(bw_hmat *h, void *dev, int64_t n_elems, int es, int64_t nit, StartF item_start, FillF fill) {
  const size_t kPiece = size_t(256) << 20;
  unsigned char *stage[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  BW_CUDA(cudaMallocHost(&stage[0], kPiece));
  BW_CUDA(cudaMallocHost(&stage[1], kPiece));
  BW_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  BW_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  bool used[2] = {false, false};
  try {
    int64_t q = 0;
    int which = 0;
    while (q < nit) {
      // grow the piece while it fits (at least one item)
      int64_t qe = q + 1;
      while (qe < nit && (item_start(qe + 1) - item_start(q)) * es <= (int64_t)kPiece) qe++;
      const int64_t e0 = item_start(q), e1 = item_start(qe);
      const size_t bytes = (size_t)(e1 - e0) * es;
      if (bytes > kPiece) {
        // a single item larger than the staging piece: fill a one-off host
        // buffer and copy it synchronously
        std::vector<unsigned char> big(bytes, 0);
        fill(q, qe, e0, big.data());
        BW_CUDA(cudaStreamSynchronize(h->stream));
        BW_CUDA(cudaMemcpy(static_cast<unsigned char *>(dev) + (size_t)e0 * es, big.data(), bytes,
                           cudaMemcpyHostToDevice));
        q = qe;
        continue;
      }
      if (used[which]) BW_CUDA(cudaEventSynchronize(ev[which]));
      par_zero(stage[which], bytes);
      fill(q, qe, e0, stage[which]);
      BW_CUDA(cudaMemcpyAsync(static_cast<unsigned char *>(dev) + (size_t)e0 * es, stage[which], bytes,
                              cudaMemcpyHostToDevice, h->stream));
      BW_CUDA(cudaEventRecord(ev[which], h->stream));
      used[which] = true;
      which ^= 1;
      q = qe;
    }
    // tail slack
    const int64_t tail0 = item_start(nit);
    BW_CUDA(cudaMemsetAsync(static_cast<unsigned char *>(dev) + (size_t)tail0 * es, 0,
                            (size_t)(n_elems - tail0) * es, h->stream));
    BW_CUDA(cudaStreamSynchronize(h->stream));
  } catch (...) {
    cudaStreamSynchronize(h->stream);
    cudaFreeHost(stage[0]);
    cudaFreeHost(stage[1]);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    throw;
  }
  cudaFreeHost(stage[0]);
  cudaFreeHost(stage[1]);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
}

// Scratch device memory of one call, freed when it goes out of scope (also on
// an exception).
struct DevTemp {
  void *p = nullptr;
  explicit DevTemp(size_t bytes) {
    const cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 1));
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      throw OomError("cudaMalloc(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
  }
  ~DevTemp() {
    if (p) cudaFree(p);
  }
  DevTemp(const DevTemp &) = delete;
  DevTemp &operator=(const DevTemp &) = delete;
  template <typename T> T *as() const { return static_cast<T *>(p); }
};

// Device-resident blocks (bw_add_flat_device): per-block maxima and
// non-finite flags on the device, for scales_from_maxima.
void device_maxima(bw_hmat *h) {
  const bw::Problem &p = h->prob;
  const int64_t nfr = (int64_t)p.fr.size(), nlr = (int64_t)p.lr.size();
  std::vector<bw::MaxSpan> spans;
  spans.reserve((size_t)(nfr + 2 * nlr));
  for (const bw::FullBlock &b : p.fr) spans.push_back({b.a.p - h->dev_fr, b.m, b.n, 0, 0});
  for (const bw::LowRankBlock &b : p.lr) spans.push_back({b.A.p - h->dev_lr, b.m, b.r, 1, 0});
  for (const bw::LowRankBlock &b : p.lr) spans.push_back({b.B.p - h->dev_lr, b.r, b.n, 1, 0});
  const int n = (int)spans.size();
  std::vector<double> mx(std::max(1, n), 0.0);
  std::vector<int> bad(std::max(1, n), 0);
  if (n) {
    DevTemp d_sp(sizeof(bw::MaxSpan) * spans.size()), d_mx(8 * (size_t)n), d_bad(4 * (size_t)n);
    BW_CUDA(cudaMemcpy(d_sp.p, spans.data(), sizeof(bw::MaxSpan) * spans.size(), cudaMemcpyHostToDevice));
    bw::block_maxabs_kernel<<<std::min(n, 148 * 8), bw::kDevLayoutThreads>>>(
        d_sp.as<bw::MaxSpan>(), n, h->dev_fr, h->dev_lr, d_mx.as<double>(), d_bad.as<int>());
    BW_CUDA(cudaGetLastError());
    BW_CUDA(cudaMemcpy(mx.data(), d_mx.p, 8 * (size_t)n, cudaMemcpyDeviceToHost));
    BW_CUDA(cudaMemcpy(bad.data(), d_bad.p, 4 * (size_t)n, cudaMemcpyDeviceToHost));
  }
  h->dev_max_fr.assign(mx.begin(), mx.begin() + nfr);
  h->dev_max_a.assign(mx.begin() + nfr, mx.begin() + nfr + nlr);
  h->dev_max_b.assign(mx.begin() + nfr + nlr, mx.begin() + nfr + 2 * nlr);
  h->dev_bad_fr.assign(bad.begin(), bad.begin() + nfr);
  h->dev_bad_lr.assign((size_t)nlr, 0);
  for (int64_t k = 0; k < nlr; k++) h->dev_bad_lr[k] = bad[nfr + k] | bad[nfr + nlr + k];
}

// Hmat::diagonal from device-resident full-rank blocks.
void device_diagonal(bw_hmat *h) {
  const int64_t n = std::max(h->n_rows, h->n_cols);
  h->diag_perm.assign((size_t)n, 0.0);
  std::vector<bw::DiagSpan> spans;
  for (const bw::FullBlock &b : h->prob.fr) {
    const int64_t lo = std::max(b.i0, b.j0), hi = std::min(b.i0 + b.m, b.j0 + b.n);
    if (lo < hi) spans.push_back({b.a.p - h->dev_fr, b.a.ld, b.i0, b.j0, lo, hi});
  }
  if (spans.empty() || n == 0) return;
  DevTemp d_sp(sizeof(bw::DiagSpan) * spans.size()), d_diag(8 * (size_t)n);
  BW_CUDA(cudaMemset(d_diag.p, 0, 8 * (size_t)n));
  BW_CUDA(cudaMemcpy(d_sp.p, spans.data(), sizeof(bw::DiagSpan) * spans.size(), cudaMemcpyHostToDevice));
  bw::diag_kernel<<<(int)std::min<size_t>(spans.size(), 148 * 8), bw::kDevLayoutThreads>>>(
      d_sp.as<bw::DiagSpan>(), (int)spans.size(), h->dev_fr, d_diag.as<double>());
  BW_CUDA(cudaGetLastError());
  BW_CUDA(cudaMemcpy(h->diag_perm.data(), d_diag.p, 8 * (size_t)n, cudaMemcpyDeviceToHost));
}

// The data of one phase packed on the device from device-resident blocks.
void pack_phase_device(bw_hmat *h, int o, int prec, int phase, void *dst) {
  std::vector<bw::PackRun> runs;
  bw::build_pack_runs(h->prob, o == 1, h->op[o], phase, prec, h->dev_fr, h->dev_fr_len, h->dev_lr, h->dev_lr_len,
                      runs);
  const int64_t es = bw::esize_of(prec), n_elems = h->op[o].ph[phase].n_elems[prec];
  BW_CUDA(cudaMemset(dst, 0, (size_t)(n_elems * es)));  // padding rows and tile slack
  if (runs.empty()) return;
  DevTemp d_runs(sizeof(bw::PackRun) * runs.size());
  BW_CUDA(cudaMemcpy(d_runs.p, runs.data(), sizeof(bw::PackRun) * runs.size(), cudaMemcpyHostToDevice));
  const long long nr = (long long)runs.size();
  const int grid = (int)std::min<long long>(nr, 148LL * 8);
  const bw::PackRun *r = d_runs.as<bw::PackRun>();
  if (prec == 0) bw::pack_runs_kernel<0><<<grid, bw::kDevLayoutThreads>>>(r, nr, h->dev_fr, h->dev_lr, dst);
  if (prec == 1) bw::pack_runs_kernel<1><<<grid, bw::kDevLayoutThreads>>>(r, nr, h->dev_fr, h->dev_lr, dst);
  if (prec == 2) bw::pack_runs_kernel<2><<<grid, bw::kDevLayoutThreads>>>(r, nr, h->dev_fr, h->dev_lr, dst);
  BW_CUDA(cudaGetLastError());
  BW_CUDA(cudaDeviceSynchronize());
}

// How a phase's queue units (in decreasing cost order) divide between the
// streaming kernels.  By default the CTA-wide kernel takes the units up to
// the last one with an item of more than narrow_rows padded rows or more than
// narrow_cols columns (the few long items of a phase, thousands of columns in
// a 2DS0-H phase 1, stream best through its staging ring), and the unstaged
// kernel the rest, warp per unit.  narrow_coop 1: the CTA-wide kernel only
// up to the last tall unit, the unstaged kernel's CTAs take the long ones
// after it whole (units [wide, coop)).  narrow_rows 0: everything CTA-wide.
bw::NarrowSplit narrow_split(const bw::ChunkPlan &cp, const bw::Tuning &tune) {
  const int64_t n_units = std::max<int64_t>(0, (int64_t)cp.item_ptr.size() - 1);
  bw::NarrowSplit sp{n_units, n_units};
  if (tune.narrow_rows <= 0) return sp;
  int64_t last_tall = -1, last_long = -1;
  for (int64_t u = 0; u < n_units; u++) {
    int64_t cols = 0;
    for (int32_t i = cp.item_ptr[u]; i < cp.item_ptr[u + 1]; i++) {
      const Chunk &c = cp.chunks[i];
      if (c.flags & bw::kFirst) cols = 0;
      cols += c.ncols;
      if (c.hpad > tune.narrow_rows) last_tall = u;
      if (cols > tune.narrow_cols) last_long = u;
    }
  }
  if (tune.narrow_coop) {
    sp.wide = last_tall + 1;
    sp.coop = std::max(sp.wide, last_long + 1);
  } else {
    sp.wide = std::max(last_tall, last_long) + 1;
    sp.coop = sp.wide;
  }
  return sp;
}

// Upload the data of one phase in pieces through two pinned staging buffers.
void upload_phase(bw_hmat *h, int o, int prec, int phase) {
  const bw::OperatorPlan &op = h->op[o];
  const bw::PhasePlan &ph = op.ph[phase];
  const int es = bw::esize_of(prec);
  DevPhase &dp = h->dev[o][prec][phase];
  dp.n_elems = ph.n_elems[prec];
  const bw::ChunkPlan &cp = ph.cp[prec];
  dp.n_chunks = (int64_t)cp.chunks.size();
  dp.n_gsegs = (int64_t)cp.gsegs.size();
  dp.split = narrow_split(cp, h->prob.tune);
  if (h->plan_only) {
    auto &buf = h->host_data[o][prec][phase];
    buf.assign((size_t)ph.n_elems[prec] * es, 0);
    bw::fill_items(h->prob, o == 1, op, phase, prec, 0, (int64_t)ph.items.size(), 0, buf.data());
    return;
  }
  dp.data = h->dmalloc((size_t)ph.n_elems[prec] * es);
  dp.chunks = static_cast<Chunk *>(h->dmalloc(std::max<size_t>(1, cp.chunks.size()) * sizeof(Chunk)));
  dp.n_items = (int64_t)cp.item_ptr.size() - 1;
  dp.items = static_cast<int32_t *>(h->dmalloc(cp.item_ptr.size() * sizeof(int32_t)));
  dp.queue = static_cast<int *>(h->dmalloc(8 * sizeof(int)));  // CTA-wide kernel [0, 2), the other [2, 5)
  BW_CUDA(cudaMemset(dp.queue, 0, 8 * sizeof(int)));
  if (!cp.chunks.empty())
    BW_CUDA(cudaMemcpy(dp.chunks, cp.chunks.data(), cp.chunks.size() * sizeof(Chunk), cudaMemcpyHostToDevice));
  BW_CUDA(cudaMemcpy(dp.items, cp.item_ptr.data(), cp.item_ptr.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  dp.n_gsegs = (int64_t)cp.gsegs.size();
  if (dp.n_gsegs) {
    dp.gsegs = static_cast<bw::GatherSeg *>(h->dmalloc(cp.gsegs.size() * sizeof(bw::GatherSeg)));
    BW_CUDA(cudaMemcpy(dp.gsegs, cp.gsegs.data(), cp.gsegs.size() * sizeof(bw::GatherSeg), cudaMemcpyHostToDevice));
  }

  const int64_t nit = (int64_t)ph.items.size();
  if (h->dev_fr || h->dev_lr) {
    pack_phase_device(h, o, prec, phase, dp.data);
    return;
  }
  staged_upload(
      h, dp.data, ph.n_elems[prec], es, nit,
      [&](int64_t q) { return q < nit ? ph.items[q].off[prec] : ph.n_elems[prec]; },
      [&](int64_t q0, int64_t q1, int64_t e0, void *dst) {
        bw::fill_items(h->prob, o == 1, op, phase, prec, q0, q1, e0, dst);
      });
}

// Upload one phase of the matmat layout (plan, chunks and BF16 data).
void upload_mm_phase(bw_hmat *h, int o, int phase) {
  const bw::MmPhase &ph = h->mm[o].ph[phase];
  const int64_t nit = (int64_t)ph.items.size();
  if (h->plan_only) {
    auto &buf = h->mm_host[o][phase];
    buf.assign((size_t)ph.n_elems, 0);
    bw::fill_mm_items(h->prob, o == 1, h->mm[o], phase, 0, nit, 0, buf.data());
    return;
  }
  DevMm &dm = h->dmm[o][phase];
  dm.n_chunks = (int64_t)ph.chunks.size();
  dm.data = static_cast<uint16_t *>(h->dmalloc((size_t)ph.n_elems * 2));
  dm.chunks = static_cast<bw::MmChunk *>(h->dmalloc(std::max<size_t>(1, ph.chunks.size()) * sizeof(bw::MmChunk)));
  dm.n_items = (int64_t)ph.item_ptr.size() - 1;
  dm.items = static_cast<int32_t *>(h->dmalloc(ph.item_ptr.size() * sizeof(int32_t)));
  dm.queue = static_cast<int *>(h->dmalloc(2 * sizeof(int)));
  BW_CUDA(cudaMemset(dm.queue, 0, 2 * sizeof(int)));
  if (!ph.chunks.empty())
    BW_CUDA(cudaMemcpy(dm.chunks, ph.chunks.data(), ph.chunks.size() * sizeof(bw::MmChunk), cudaMemcpyHostToDevice));
  BW_CUDA(cudaMemcpy(dm.items, ph.item_ptr.data(), ph.item_ptr.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  staged_upload(
      h, dm.data, ph.n_elems, 2, nit, [&](int64_t q) { return q < nit ? ph.items[q].off : ph.n_elems; },
      [&](int64_t q0, int64_t q1, int64_t e0, void *dst) {
        bw::fill_mm_items(h->prob, o == 1, h->mm[o], phase, q0, q1, e0, static_cast<uint16_t *>(dst));
      });
}

void compute_diagonal(bw_hmat *h) {
  // Hmat::diagonal (src/hmat/hmatrix/hmat.cc:256-285): entries of the FR blocks
  // with (i + i0) == (j + j0) in scalar units.  The reference skips FR blocks
  // that lie strictly below/above the diagonal; the index test covers that.
  const int64_t n = std::max(h->n_rows, h->n_cols);
  h->diag_perm.assign((size_t)n, 0.0);
  for (const bw::FullBlock &b : h->prob.fr) {
    const int64_t lo = std::max(b.i0, b.j0), hi = std::min(b.i0 + b.m, b.j0 + b.n);
    for (int64_t d = lo; d < hi; d++) h->diag_perm[(size_t)d] = b.a.at(d - b.i0, d - b.j0);
  }
}

// The launches of one matvec: x gather (+ permutation), phase 1 (t), G2
// gather, phase 2 (y), each phase in the CTA-wide and / or the unstaged
// kernel, with the given scratch vectors; `ev` (optional) receives
// kTimedLaunches + 1 events around them.
template <typename S>
void launch_matvec_impl(bw_hmat *h, int o, int prec, const double *x, double *y, bool permuted, cudaStream_t st,
                        void *xp_buf, void *t_buf, void *g2_buf, cudaEvent_t *ev) {
  using G = typename bw::Store<S>::G;
  const bw::OperatorPlan &op = h->op[o];
  const int32_t *perm_in = permuted ? nullptr : (o == 0 ? h->d_perm1 : h->d_perm0);
  const int32_t *perm_out = permuted ? nullptr : (o == 0 ? h->d_perm0 : h->d_perm1);
  const int n_in = (int)op.n_in;
  constexpr bool kPacked = bw::Store<S>::kRows == 0;  // tensor-core path takes pack_hilo vectors
  G *xp = static_cast<G *>(xp_buf);
  // BF16: the packed copy of x sits after the FP32 one in the same region
  uint32_t *xpk = kPacked ? reinterpret_cast<uint32_t *>(static_cast<unsigned char *>(xp_buf) +
                                                         align256(4 * (int64_t)n_in + 16))
                          : nullptr;
  G *t = static_cast<G *>(t_buf);
  if (ev) BW_CUDA(cudaEventRecord(ev[0], st));
  if (n_in > 0) {
    bw::gather_x_kernel<G><<<(n_in + 255) / 256, 256, 0, st>>>(x, xp, xpk, perm_in, h->dof, n_in);
    BW_CUDA(cudaGetLastError());
  }
  if (ev) BW_CUDA(cudaEventRecord(ev[1], st));
  set_smem_attr<S>();
  for (int phase = 0; phase < 2; phase++) {
    const DevPhase &dp = h->dev[o][prec][phase];
    if (phase == 1) {
      if (dp.n_gsegs > 0) {
        const int per_block = 8 * bw::kG2Runs;  // runs per 256-thread block (kG2Runs per warp)
        bw::gather_g2_kernel<G, kPacked><<<(int)((dp.n_gsegs + per_block - 1) / per_block), 256, 0, st>>>(
            dp.gsegs, (int)dp.n_gsegs, xp, t, g2_buf);
        BW_CUDA(cudaGetLastError());
      }
      if (ev) BW_CUDA(cudaEventRecord(ev[4], st));
    }
    if (dp.n_chunks > 0) {
      bw::StreamArgs a{};
      a.data = dp.data;
      a.chunks = dp.chunks;
      a.item_ptr = dp.items;
      a.n_items = (int)dp.n_items;
      a.queue = dp.queue;
      a.gsrc = phase == 0 ? (kPacked ? static_cast<const void *>(xpk) : static_cast<const void *>(xp))
                          : static_cast<const void *>(g2_buf);
      a.t_out = t;
      a.y_out = y;
      a.perm_out = perm_out;
      a.dof = h->dof;
      a.phase = phase + 1;
      a.err = h->d_err;
      a.spin_limit = h->spin_limit;
      a.withhold = h->take_withhold();  // the test hook applies to the CTA-wide kernel
      if (dp.split.wide > 0) {
        a.n_items = (int)dp.split.wide;
        bw::stream_panels_kernel<S><<<h->grid, bw::threads_of<S>(), bw::SmemLayout<S>::kTotal, st>>>(a);
        BW_CUDA(cudaGetLastError());
      }
      if (ev) BW_CUDA(cudaEventRecord(ev[phase == 0 ? 2 : 5], st));
      if (dp.split.wide < dp.n_items) {  // the items of at most narrow_rows rows, on their own queue
        a.item_ptr = dp.items + dp.split.wide;
        a.n_items = (int)(dp.n_items - dp.split.wide);
        a.n_coop = (int)(dp.split.coop - dp.split.wide);
        a.queue = dp.queue + 2;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * h->grid);
        cfg.blockDim = dim3(32 * bw::kNarrowWarps);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        // After the phase's CTA-wide launch (and no timing event between
        // them) it may start on the SMs that launch leaves free or frees.
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = (dp.split.wide > 0 && !ev) ? 1 : 0;
        BW_CUDA(cudaLaunchKernelEx(&cfg, bw::narrow_items_kernel<S>, a));
      }
    }
    if (ev) {
      if (dp.n_chunks == 0) BW_CUDA(cudaEventRecord(ev[phase == 0 ? 2 : 5], st));
      BW_CUDA(cudaEventRecord(ev[phase == 0 ? 3 : 6], st));
    }
  }
}

template <typename S>
void launch_matvec(bw_hmat *h, int o, int prec, const double *x, double *y, bool permuted, cudaStream_t st) {
  launch_matvec_impl<S>(h, o, prec, x, y, permuted, st, h->d_xp, h->d_t, h->d_g2, h->timing_slot());
}

// ----------------------------------------------------------------------------
// Static scratch for bw_matvec_static_scratch.
//
// Some callers cannot let a library allocate device memory: a host process
// whose device memory is owned by another allocator (a framework's caching
// pool, or a solver that reserved the whole card up front), and code on a
// latency-critical path where cudaMalloc / cudaFree are not allowed because
// they can synchronize the whole device.  For them this entry point keeps its
// scratch vectors (the gathered input and the low-rank intermediates t) in a
// fixed array that is part of the library image: BW_STATIC_SCRATCH_BYTES of
// device memory on every GPU that loads the library, held until the process
// exits.  All calls on a device share the one array, so calls whose kernels
// overlap on the GPU (several streams, several handles) race on it.
static __device__ __align__(256) unsigned char bw_static_scratch[BW_STATIC_SCRATCH_BYTES];

// Device address of bw_static_scratch, looked up once per device with that
// device current (the host-side name is only a stand-in for the symbol).
constexpr int kMaxStaticDevices = 64;
std::mutex g_static_mu;
void *g_static_ptr[kMaxStaticDevices] = {};

void *static_scratch_ptr(int device) {
  if (device < 0 || device >= kMaxStaticDevices) throw UnsupportedError("device ordinal too large for the static scratch");
  std::lock_guard<std::mutex> g(g_static_mu);
  if (!g_static_ptr[device]) {
    void *p = nullptr;
    BW_CUDA(cudaGetSymbolAddress(&p, bw_static_scratch));
    g_static_ptr[device] = p;
  }
  return g_static_ptr[device];
}

// Rows of the matmat operand X: the largest input size rounded up to a tile
// row, plus the zero rows that the widened windows of the last columns reach.
int64_t mm_xt_rows(const bw_hmat *h) { return (std::max(h->n_rows, h->n_cols) + 7) / 8 * 8 + bw::kMmPadRows; }

// Y[:, 0:nrhs] = op X[:, 0:nrhs] on the tensor cores, in passes of kMmRhs
// right-hand sides: X gather (+ permutation) into 8x8 BF16 tiles, phase 1
// (T8 = stacked B factors x X), phase 2 (row panels -> Y).
void launch_matmat_tc(bw_hmat *h, int o, const double *X, int64_t ldx, double *Y, int64_t ldy, int nrhs, bool permuted,
                      cudaStream_t st) {
  static bool attr_done[64] = {};
  smem_attr_once(attr_done, bw::mm_stream_kernel, bw::kMmSmem);
  const bw::MmPlan &mm = h->mm[o];
  const int32_t *perm_in = permuted ? nullptr : (o == 0 ? h->d_perm1 : h->d_perm0);
  const int32_t *perm_out = permuted ? nullptr : (o == 0 ? h->d_perm0 : h->d_perm1);
  const int n_in = (int)mm.n_in;
  const int n_pad = (n_in + 7) / 8 * 8;
  for (int c0 = 0; c0 < nrhs; c0 += bw::kMmRhs) {
    const int nr = std::min(bw::kMmRhs, nrhs - c0);
    if (n_pad > 0) {
      bw::gather_xt_kernel<<<(n_pad + 63) / 64, 256, 0, st>>>(X + (int64_t)c0 * ldx, ldx, nr, h->d_xt, perm_in,
                                                               h->dof, n_in, n_pad);
      BW_CUDA(cudaGetLastError());
    }
    for (int phase = 0; phase < 2; phase++) {
      const DevMm &dm = h->dmm[o][phase];
      if (dm.n_chunks == 0) continue;
      bw::MmArgs a{};
      a.data = dm.data;
      a.chunks = dm.chunks;
      a.item_ptr = dm.items;
      a.n_items = (int)dm.n_items;
      a.queue = dm.queue;
      a.xt = h->d_xt;
      a.t8 = h->d_t8;
      a.y = Y + (int64_t)c0 * ldy;
      a.ldy = ldy;
      a.perm_out = perm_out;
      a.dof = h->dof;
      a.nrhs = nr;
      a.phase = phase + 1;
      a.err = h->d_err;
      a.spin_limit = h->spin_limit;
      a.withhold = h->take_withhold();
      bw::mm_stream_kernel<<<h->grid, bw::kMmThreads, bw::kMmSmem, st>>>(a);
      BW_CUDA(cudaGetLastError());
    }
  }
}

// One matvec with its scratch vectors in the static array (no timing).
template <typename S>
void launch_matvec_on(bw_hmat *h, int o, int prec, const double *x, double *y, bool permuted, cudaStream_t st,
                      void *xp_buf, void *t_buf, void *g2_buf) {
  launch_matvec_impl<S>(h, o, prec, x, y, permuted, st, xp_buf, t_buf, g2_buf, nullptr);
}

}  // namespace

extern "C" {

const char *bw_version(void) { return "bigwham_b200 0.1 (sm_100a)"; }

int bw_batch_offsets(const bw_hmat *h, int member, int64_t *row0, int64_t *col0) {
  if (!h || member < 0 || member + 1 >= (int)h->row_off.size()) return BW_ERR_ARG;
  if (row0) *row0 = h->row_off[(size_t)member];
  if (col0) *col0 = h->col_off[(size_t)member];
  return BW_OK;
}

int bw_batch_count(const bw_hmat *h) { return h ? (int)h->row_off.size() - 1 : 0; }

int bw_set_wait_limit(bw_hmat *h, int64_t ns) {
  if (!h) return BW_ERR_ARG;
  if (ns < 1 || ns > 60000000000LL) {
    h->err = "wait limit must be in [1 ns, 60 s]";
    return BW_ERR_ARG;
  }
  h->spin_limit = ns;
  return BW_OK;
}

int bw_test_withhold_chunk(bw_hmat *h, int index) {
  if (!h || index < 0) return BW_ERR_ARG;
  h->withhold = index;
  return BW_OK;
}

int bw_set_tuning(bw_hmat *h, const char *key, int64_t value) {
  if (!h || !key) return BW_ERR_ARG;
  if (h->finalized) {
    h->err = "bw_set_tuning after bw_finalize";
    return BW_ERR_STATE;
  }
  const std::string k(key);
  bw::Tuning &t = h->prob.tune;
  if (k == "items_per_cta_phase1" || k == "items_per_cta_phase2" || k == "mm_items_per_cta") {
    if (value < 1 || value > 256) {
      h->err = k + " must be in [1, 256]";
      return BW_ERR_ARG;
    }
    if (k == "mm_items_per_cta")
      t.mm_items_per_cta = (int)value;
    else
      t.items_per_cta[k.back() - '1'] = (int)value;
    return BW_OK;
  }
  if (k == "narrow_rows") {
    if (value < 0 || value > bw::kNarrowRows) {
      h->err = "narrow_rows must be in [0, " + std::to_string(bw::kNarrowRows) + "]";
      return BW_ERR_ARG;
    }
    t.narrow_rows = (int)value;
    return BW_OK;
  }
  if (k == "narrow_coop") {
    if (value < 0 || value > 1) {
      h->err = "narrow_coop must be 0 or 1";
      return BW_ERR_ARG;
    }
    t.narrow_coop = (int)value;
    return BW_OK;
  }
  if (k == "narrow_cols") {
    if (value < 1 || value > (int64_t(1) << 30)) {
      h->err = "narrow_cols must be in [1, 2^30]";
      return BW_ERR_ARG;
    }
    t.narrow_cols = (int)value;
    return BW_OK;
  }
  if (k == "unit_bytes") {
    if (value < 0 || value > (int64_t(1) << 30)) {
      h->err = "unit_bytes must be in [0, 2^30]";
      return BW_ERR_ARG;
    }
    t.unit_bytes = (int)value;
    return BW_OK;
  }
  if (k == "chunk_bytes") {
    if (value < 4096 || value > bw::kStageBytes || value % 16) {
      h->err = "chunk_bytes must be a multiple of 16 in [4096, " + std::to_string(bw::kStageBytes) + "]";
      return BW_ERR_ARG;
    }
    t.chunk_bytes = (int)value;
    return BW_OK;
  }
  h->err = "unknown tuning key " + k;
  return BW_ERR_ARG;
}

int bw_create(int dof, int64_t n_rows, int64_t n_cols, const int64_t *perm0, const int64_t *perm1, int device,
              bw_hmat **out) {
  return bw_create_batch(dof, 1, &n_rows, &n_cols, &perm0, &perm1, device, out);
}

int bw_create_batch(int dof, int count, const int64_t *n_rows_k, const int64_t *n_cols_k,
                    const int64_t *const *perm0_k, const int64_t *const *perm1_k, int device, bw_hmat **out) {
  if (!out) return BW_ERR_ARG;
  *out = nullptr;
  auto fail = [](const std::string &m, int code) {
    std::lock_guard<std::mutex> g(g_err_mu);
    g_last_create_error = m;
    return code;
  };
  if (count < 1 || !n_rows_k || !n_cols_k || !perm0_k || !perm1_k) return fail("bad member list", BW_ERR_ARG);
  if (dof < 1) return fail("bad sizes: dof must be >= 1", BW_ERR_ARG);
  std::unique_ptr<bw_hmat> h(new bw_hmat);
  // Members are laid along the diagonal of one block-diagonal H-matrix: member
  // k's rows and columns start at the sums of the earlier members' sizes, and
  // its permutations are shifted by the earlier members' point counts.
  int64_t n_rows = 0, n_cols = 0;
  for (int k = 0; k < count; k++) {
    const int64_t m = n_rows_k[k], n = n_cols_k[k];
    if (m < 0 || n < 0 || m % dof || n % dof)
      return fail("bad sizes: n_rows and n_cols must be non-negative multiples of dof >= 1", BW_ERR_ARG);
    if ((m && !perm0_k[k]) || (n && !perm1_k[k])) return fail("null permutation", BW_ERR_ARG);
    if (m > INT32_MAX - n_rows || n > INT32_MAX - n_cols) return fail("sizes above 2^31-1 are not supported", BW_ERR_ARG);
    h->row_off.push_back(n_rows);
    h->col_off.push_back(n_cols);
    for (int64_t i = 0; i < m / dof; i++) {
      const int64_t v = perm0_k[k][i];
      if (v < 0 || v >= m / dof) return fail("permutation is not a permutation of 0..n-1", BW_ERR_ARG);
      h->perm0.push_back(v + n_rows / dof);
    }
    for (int64_t i = 0; i < n / dof; i++) {
      const int64_t v = perm1_k[k][i];
      if (v < 0 || v >= n / dof) return fail("permutation is not a permutation of 0..n-1", BW_ERR_ARG);
      h->perm1.push_back(v + n_cols / dof);
    }
    n_rows += m;
    n_cols += n;
  }
  h->row_off.push_back(n_rows);
  h->col_off.push_back(n_cols);
  h->dof = dof;
  h->n_rows = n_rows;
  h->n_cols = n_cols;
  for (auto *pv : {&h->perm0, &h->perm1}) {
    const int64_t np = (int64_t)pv->size();
    std::vector<char> seen((size_t)np, 0);
    for (int64_t v : *pv) {
      if (v < 0 || v >= np || seen[(size_t)v]) return fail("permutation is not a permutation of 0..n-1", BW_ERR_ARG);
      seen[(size_t)v] = 1;
    }
  }
  h->prob.dof = dof;
  h->prob.n_rows = n_rows;
  h->prob.n_cols = n_cols;
  if (count > 1) {
    h->prob.row_off = h->row_off;
    h->prob.col_off = h->col_off;
  }
  h->device = device;
  if (device >= 0) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device >= ndev) {
      cudaGetLastError();
      return fail("CUDA device " + std::to_string(device) + " not available", BW_ERR_CUDA);
    }
    if (cudaSetDevice(device) != cudaSuccess) return fail("cudaSetDevice failed", BW_ERR_CUDA);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    h->grid = sms > 0 ? sms : 148;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail("cudaStreamCreate failed", BW_ERR_CUDA);
  }
  *out = h.release();
  return BW_OK;
}

int bw_add_full(bw_hmat *h, int64_t i0, int64_t j0, int64_t m, int64_t n, const double *a, int64_t lda) {
  if (!h) return BW_ERR_ARG;
  if (h->finalized || h->dev_fr || h->dev_lr) {
    h->err = "bw_add_full after bw_finalize or bw_add_flat_device";
    return BW_ERR_STATE;
  }
  return guarded(h, [&] {
    h->prob.fr.push_back({i0, j0, m, n, bw::View{a, lda, false}});
    return BW_OK;
  });
}

int bw_add_flat_device(bw_hmat *h, int64_t n_fr, const int64_t *fr, int64_t n_lr, const int64_t *lr,
                       const double *fr_data, int64_t fr_len, const double *lr_data, int64_t lr_len) {
  if (!h) return BW_ERR_ARG;
  if (h->finalized || !h->prob.fr.empty() || !h->prob.lr.empty()) {
    h->err = "bw_add_flat_device needs an empty handle (before any bw_add_* and bw_finalize)";
    return BW_ERR_STATE;
  }
  return guarded(h, [&] {
    if (h->device < 0) throw StateError("bw_add_flat_device needs a handle with a device");
    if (n_fr < 0 || n_lr < 0 || fr_len < 0 || lr_len < 0 || (n_fr && (!fr || !fr_data)) ||
        (n_lr && (!lr || !lr_data)))
      throw std::invalid_argument("bw_add_flat_device: null or negative argument");
    const int64_t d = h->dof, rp = h->n_rows / d, cp = h->n_cols / d;
    auto extent = [&](int64_t a0, int64_t a1, int64_t lim, const char *what, int64_t k) {
      if (!(0 <= a0 && a0 < a1 && a1 <= lim))
        throw std::invalid_argument(std::string("bw_add_flat_device: ") + what + " block " + std::to_string(k) +
                                    " lies outside the matrix");
      return (a1 - a0) * d;
    };
    std::vector<bw::FullBlock> vf;
    std::vector<bw::LowRankBlock> vl;
    int64_t o = 0;
    for (int64_t k = 0; k < n_fr; k++) {
      const int64_t *c = fr + 4 * k;
      const int64_t m = extent(c[0], c[2], rp, "FR", k), n = extent(c[1], c[3], cp, "FR", k);
      if (m * n > fr_len - o) throw std::invalid_argument("bw_add_flat_device: fr_data shorter than the pattern");
      vf.push_back({c[0] * d, c[1] * d, m, n, bw::View{fr_data + o, m, false}});
      o += m * n;
    }
    o = 0;
    for (int64_t k = 0; k < n_lr; k++) {
      const int64_t *c = lr + 5 * k;
      const int64_t m = extent(c[0], c[2], rp, "LR", k), n = extent(c[1], c[3], cp, "LR", k), r = c[4];
      if (r < 0 || r > std::min(m, n)) throw std::invalid_argument("bw_add_flat_device: bad rank");
      if (r * (m + n) > lr_len - o) throw std::invalid_argument("bw_add_flat_device: lr_data shorter than the pattern");
      vl.push_back({c[0] * d, c[1] * d, m, n, r, bw::View{lr_data + o, std::max<int64_t>(1, m), false},
                    bw::View{lr_data + o + m * r, std::max<int64_t>(1, r), false}});
      o += r * (m + n);
    }
    h->prob.fr = std::move(vf);
    h->prob.lr = std::move(vl);
    h->dev_fr = fr_data;
    h->dev_lr = lr_data;
    h->dev_fr_len = fr_len;
    h->dev_lr_len = lr_len;
    return BW_OK;
  });
}

int bw_add_lowrank(bw_hmat *h, int64_t i0, int64_t j0, int64_t m, int64_t n, int64_t r, const double *A,
                   int64_t lda, const double *B, int64_t ldb) {
  if (!h) return BW_ERR_ARG;
  if (h->finalized || h->dev_fr || h->dev_lr) {
    h->err = "bw_add_lowrank after bw_finalize or bw_add_flat_device";
    return BW_ERR_STATE;
  }
  return guarded(h, [&] {
    h->prob.lr.push_back({i0, j0, m, n, r, bw::View{A, lda, false}, bw::View{B, ldb, false}});
    return BW_OK;
  });
}

int bw_set_device_limit(bw_hmat *h, int64_t bytes) {
  if (!h || bytes < 0) return BW_ERR_ARG;
  h->dev_limit = bytes;
  return BW_OK;
}

int bw_finalize(bw_hmat *h, int flags) {
  if (!h) return BW_ERR_ARG;
  if (h->finalized) {
    h->err = "bw_finalize called twice";
    return BW_ERR_STATE;
  }
  int rc = guarded(h, [&] {
    int mask = flags & (BW_FP64 | BW_FP32 | BW_BF16);
    if (!mask) mask = BW_FP64;
    h->plan_only = (flags & BW_PLAN_ONLY) != 0;
    if (!h->plan_only && h->device < 0) throw StateError("handle has no device; use BW_PLAN_ONLY");
    if (h->device >= 0) BW_CUDA(cudaSetDevice(h->device));
    const bool want_t = (flags & BW_STORE_TRANSPOSE) != 0;
    const bool check = (flags & BW_NO_FINITE_CHECK) == 0;
    const bool want_mm = (flags & BW_STORE_MATMAT) != 0;
    if ((h->dev_fr || h->dev_lr) && h->plan_only)
      throw StateError("device-resident blocks (bw_add_flat_device) cannot make a plan-only handle");
    if ((h->dev_fr || h->dev_lr) && want_mm)
      throw UnsupportedError("the matmat layout is not built from device-resident blocks");
    // statistics
    h->entries = 0;
    h->sum_rank = 0;
    h->n_fr = (int64_t)h->prob.fr.size();
    h->n_lr = (int64_t)h->prob.lr.size();
    for (auto &b : h->prob.fr) h->entries += b.m * b.n;
    for (auto &b : h->prob.lr) {
      h->entries += b.r * (b.m + b.n);
      h->sum_rank += b.r;
    }
    for (int o = 0; o < (want_t ? 2 : 1); o++) {
      bw::build_operator(h->prob, o == 1, h->grid, h->op[o]);
      if (h->dev_fr || h->dev_lr) {
        if (o == 0) device_maxima(h);
        bw::scales_from_maxima(h->prob, o == 1, check && o == 0, h->dev_max_fr.data(), h->dev_max_a.data(),
                               h->dev_max_b.data(), h->dev_bad_fr.data(), h->dev_bad_lr.data(), h->op[o]);
      } else {
        bw::compute_scales(h->prob, o == 1, check && o == 0, h->op[o]);
      }
      for (int p = 0; p < 3; p++)
        if (mask & (1 << p)) bw::build_chunks(h->prob, o == 1, p, h->grid, h->op[o]);
      if (want_mm) bw::build_mm_plan(h->prob, o == 1, h->grid, h->op[o], h->mm[o]);
    }
    if (h->dev_fr || h->dev_lr)
      device_diagonal(h);
    else
      compute_diagonal(h);
    if (!h->plan_only) {
      // size check before any allocation
      int64_t need = 0;
      for (int o = 0; o < (want_t ? 2 : 1); o++)
        for (int p = 0; p < 3; p++)
          if (mask & (1 << p))
            for (int ph = 0; ph < 2; ph++)
              need += h->op[o].ph[ph].n_elems[p] * bw::esize_of(p) +
                      (int64_t)h->op[o].ph[ph].cp[p].chunks.size() * (int64_t)sizeof(Chunk) +
                      (int64_t)h->op[o].ph[ph].cp[p].gsegs.size() * (int64_t)sizeof(bw::GatherSeg);
      int64_t t8_rows = 0;
      if (want_mm) {
        for (int o = 0; o < (want_t ? 2 : 1); o++) {
          for (int ph = 0; ph < 2; ph++)
            need += h->mm[o].ph[ph].n_elems * 2 + (int64_t)h->mm[o].ph[ph].chunks.size() * (int64_t)sizeof(bw::MmChunk);
          t8_rows = std::max<int64_t>(t8_rows, h->mm[o].t8_len);
        }
        need += (mm_xt_rows(h) + t8_rows + bw::kMmPadRows) * 2 * bw::kMmRhs;
      }
      if (h->dev_limit > 0 && need > h->dev_limit)
        throw OomError("layout needs " + std::to_string(need) + " device bytes, above the configured limit of " +
                       std::to_string(h->dev_limit));
      const int64_t nmax = std::max(h->n_rows, h->n_cols);
      std::vector<int32_t> p32;
      p32.assign(h->perm0.begin(), h->perm0.end());
      h->d_perm0 = static_cast<int32_t *>(h->dmalloc(std::max<size_t>(1, p32.size()) * 4));
      if (!p32.empty()) BW_CUDA(cudaMemcpy(h->d_perm0, p32.data(), p32.size() * 4, cudaMemcpyHostToDevice));
      p32.assign(h->perm1.begin(), h->perm1.end());
      h->d_perm1 = static_cast<int32_t *>(h->dmalloc(std::max<size_t>(1, p32.size()) * 4));
      if (!p32.empty()) BW_CUDA(cudaMemcpy(h->d_perm1, p32.data(), p32.size() * 4, cudaMemcpyHostToDevice));
      // +16 bytes: the kernels stage vector segments in 16-byte aligned windows
      h->d_xp = h->dmalloc((size_t)std::max({xp_region_bytes(0, nmax), xp_region_bytes(2, nmax), (int64_t)1}));
      h->d_t = h->dmalloc((size_t)std::max<int64_t>(1, h->sum_rank) * 8 + 16);
      h->d_g2 = h->dmalloc((size_t)std::max<int64_t>(1, g2_bytes(h, mask, want_t)) + 16);
      h->d_xh = static_cast<double *>(h->dmalloc((size_t)std::max<int64_t>(1, nmax) * 8));
      h->d_yh = static_cast<double *>(h->dmalloc((size_t)std::max<int64_t>(1, nmax) * 8));
      BW_CUDA(cudaMallocHost(&h->h_xpin, (size_t)std::max<int64_t>(1, nmax) * 8));
      BW_CUDA(cudaMallocHost(&h->h_ypin, (size_t)std::max<int64_t>(1, nmax) * 8));
      for (cudaEvent_t &e : h->y_ready) BW_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      if (want_mm) {
        const size_t xb = (size_t)mm_xt_rows(h) * 2 * bw::kMmRhs, tb = (size_t)(t8_rows + bw::kMmPadRows) * 2 * bw::kMmRhs;
        h->d_xt = static_cast<uint16_t *>(h->dmalloc(xb));
        h->d_t8 = static_cast<uint16_t *>(h->dmalloc(tb));
        BW_CUDA(cudaMemset(h->d_xt, 0, xb));
        BW_CUDA(cudaMemset(h->d_t8, 0, tb));
      }
      h->d_err = static_cast<int *>(h->dmalloc(sizeof(int)));
      BW_CUDA(cudaMemset(h->d_err, 0, sizeof(int)));
      BW_CUDA(cudaMallocHost(&h->h_err, sizeof(int)));
      *h->h_err = 0;
    }
    for (int o = 0; o < (want_t ? 2 : 1); o++)
      for (int p = 0; p < 3; p++)
        if (mask & (1 << p))
          for (int ph = 0; ph < 2; ph++) upload_phase(h, o, p, ph);
    if (want_mm)
      for (int o = 0; o < (want_t ? 2 : 1); o++)
        for (int ph = 0; ph < 2; ph++) upload_mm_phase(h, o, ph);
    h->has_mm = want_mm;
    h->stored = mask;
    h->has_t = want_t;
    h->finalized = true;
    return BW_OK;
  });
  // the borrowed block pointers are not used after this point (the host plan
  // keeps only indices; a plan-only handle keeps its converted copy)
  if (rc != BW_OK && !h->plan_only) h->release();
  if (rc == BW_OK) {
    h->prob.fr.clear();
    h->prob.lr.clear();
    h->prob.fr.shrink_to_fit();
    h->prob.lr.shrink_to_fit();
    h->borrowed.reset();
  }
  return rc;
}

int bw_matvec(bw_hmat *h, const double *x, double *y, int flags, void *stream) {
  if (!h) return BW_ERR_ARG;
  return guarded(h, [&] {
    if (!h->finalized) throw StateError("bw_matvec before bw_finalize");
    if (h->plan_only) throw StateError("handle was finalized with BW_PLAN_ONLY (no device data)");
    const int p = prec_index(flags);
    if (p < 0) throw std::invalid_argument("flags must name exactly one of BW_FP64, BW_FP32, BW_BF16");
    if (!(h->stored & (1 << p))) throw UnsupportedError("precision not stored by bw_finalize");
    const bool tr = (flags & BW_TRANSPOSE) != 0;
    if (tr && !h->has_t) throw UnsupportedError("transposed layout not stored (finalize with BW_STORE_TRANSPOSE)");
    const int64_t nin = tr ? h->n_rows : h->n_cols, nout = tr ? h->n_cols : h->n_rows;
    if ((nin && !x) || (nout && !y)) throw std::invalid_argument("null vector");
    if (x && y) {
      const char *xb = reinterpret_cast<const char *>(x), *yb = reinterpret_cast<const char *>(y);
      if (xb < yb + nout * 8 && yb < xb + nin * 8) throw std::invalid_argument("x and y overlap");
    }
    BW_CUDA(cudaSetDevice(h->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool perm = (flags & BW_PERMUTED) != 0;
    const int o = tr ? 1 : 0;
    if (p == 0)
      launch_matvec<double>(h, o, 0, x, y, perm, st);
    else if (p == 1)
      launch_matvec<float>(h, o, 1, x, y, perm, st);
    else
      launch_matvec<bw::Bf16>(h, o, 2, x, y, perm, st);
    return BW_OK;
  });
}

int bw_matvec_static_scratch(bw_hmat *h, const double *x, double *y, int flags, void *stream) {
  if (!h) return BW_ERR_ARG;
  return guarded(h, [&] {
    if (!h->finalized) throw StateError("bw_matvec_static_scratch before bw_finalize");
    if (h->plan_only) throw StateError("handle was finalized with BW_PLAN_ONLY (no device data)");
    const int p = prec_index(flags);
    if (p < 0) throw std::invalid_argument("flags must name exactly one of BW_FP64, BW_FP32, BW_BF16");
    if (!(h->stored & (1 << p))) throw UnsupportedError("precision not stored by bw_finalize");
    const bool tr = (flags & BW_TRANSPOSE) != 0;
    if (tr && !h->has_t) throw UnsupportedError("transposed layout not stored (finalize with BW_STORE_TRANSPOSE)");
    const int64_t nin = tr ? h->n_rows : h->n_cols, nout = tr ? h->n_cols : h->n_rows;
    if ((nin && !x) || (nout && !y)) throw std::invalid_argument("null vector");
    if (x && y) {
      const char *xb = reinterpret_cast<const char *>(x), *yb = reinterpret_cast<const char *>(y);
      if (xb < yb + nout * 8 && yb < xb + nin * 8) throw std::invalid_argument("x and y overlap");
    }
    // scratch: gathered x, t and the gather array G2, each at a 256-byte
    // boundary with 16 bytes of slack (vector runs are staged in 16-byte
    // aligned windows)
    const int64_t gsize = p == 0 ? 8 : 4;
    const int o_ = tr ? 1 : 0;
    const int64_t t_at = align256(xp_region_bytes(p, nin));
    const int64_t g2_at = (t_at + h->sum_rank * gsize + 16 + 255) / 256 * 256;
    const int64_t need = g2_at + h->op[o_].ph[1].cp[p].g_len * gsize + 16;
    if (need > (int64_t)BW_STATIC_SCRATCH_BYTES)
      throw std::invalid_argument("this H-matrix needs " + std::to_string(need) +
                                  " bytes of scratch, above the static maximum of " +
                                  std::to_string((long long)BW_STATIC_SCRATCH_BYTES) +
                                  " bytes; use bw_matvec instead");
    BW_CUDA(cudaSetDevice(h->device));
    unsigned char *base = static_cast<unsigned char *>(static_scratch_ptr(h->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool perm = (flags & BW_PERMUTED) != 0;
    const int o = tr ? 1 : 0;
    if (p == 0)
      launch_matvec_on<double>(h, o, 0, x, y, perm, st, base, base + t_at, base + g2_at);
    else if (p == 1)
      launch_matvec_on<float>(h, o, 1, x, y, perm, st, base, base + t_at, base + g2_at);
    else
      launch_matvec_on<bw::Bf16>(h, o, 2, x, y, perm, st, base, base + t_at, base + g2_at);
    return BW_OK;
  });
}

int bw_sync(bw_hmat *h, void *stream) {
  if (!h) return BW_ERR_ARG;
  return guarded(h, [&] {
    if (!h->finalized || h->plan_only) throw StateError("no device state");
    BW_CUDA(cudaSetDevice(h->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BW_CUDA(cudaMemcpyAsync(h->h_err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    BW_CUDA(cudaStreamSynchronize(st));
    if (*h->h_err != 0) {
      const int code = *h->h_err;
      BW_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(int), st));
      BW_CUDA(cudaStreamSynchronize(st));
      char buf[64];
      snprintf(buf, sizeof buf, "kernel error word 0x%x", code);
      h->err = buf;
      return BW_ERR_DEVICE;
    }
    return BW_OK;
  });
}

int bw_matvec_host(bw_hmat *h, const double *x, double *y, int flags) {
  if (!h) return BW_ERR_ARG;
  const bool tr = (flags & BW_TRANSPOSE) != 0;
  int64_t nin = 0, nout = 0;
  // Pieces of the vectors: the host copy of piece k overlaps the DMA of piece
  // k - 1 on the way in, and the DMA of piece k + 1 on the way out.
  constexpr int kPieces = 4;  // = the handle's y_ready events
  auto piece = [](int64_t n, int k) { return (n * k) / kPieces; };
  int rc = guarded(h, [&] {
    if (!h->finalized || h->plan_only) throw StateError("no device state");
    nin = tr ? h->n_rows : h->n_cols;
    nout = tr ? h->n_cols : h->n_rows;
    if ((nin && !x) || (nout && !y)) throw std::invalid_argument("null vector");
    BW_CUDA(cudaSetDevice(h->device));
    // through the handle's pinned vectors: a few host threads copy the
    // caller's (pageable) array, the DMA then runs at full link speed
    for (int k = 0; k < kPieces; k++) {
      const int64_t a = piece(nin, k), b = piece(nin, k + 1);
      if (b <= a) continue;
      host_copy(h->h_xpin + a, x + a, b - a);
      BW_CUDA(cudaMemcpyAsync(h->d_xh + a, h->h_xpin + a, (size_t)(b - a) * 8, cudaMemcpyHostToDevice, h->stream));
    }
    return BW_OK;
  });
  if (rc != BW_OK) return rc;
  rc = bw_matvec(h, h->d_xh, h->d_yh, flags, h->stream);
  if (rc != BW_OK) return rc;
  return guarded(h, [&] {
    for (int k = 0; k < kPieces; k++) {
      const int64_t a = piece(nout, k), b = piece(nout, k + 1);
      if (b > a)
        BW_CUDA(cudaMemcpyAsync(h->h_ypin + a, h->d_yh + a, (size_t)(b - a) * 8, cudaMemcpyDeviceToHost, h->stream));
      // the kernels' error word travels with the last piece: one wait covers both
      if (k == kPieces - 1)
        BW_CUDA(cudaMemcpyAsync(h->h_err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      BW_CUDA(cudaEventRecord(h->y_ready[k], h->stream));
    }
    for (int k = 0; k < kPieces; k++) {
      const int64_t a = piece(nout, k), b = piece(nout, k + 1);
      BW_CUDA(cudaEventSynchronize(h->y_ready[k]));
      if (b > a) host_copy(y + a, h->h_ypin + a, b - a);
    }
    if (*h->h_err != 0) {  // y is unspecified; clear the word as bw_sync does
      const int code = *h->h_err;
      BW_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream));
      BW_CUDA(cudaStreamSynchronize(h->stream));
      char buf[64];
      snprintf(buf, sizeof buf, "kernel error word 0x%x", code);
      h->err = buf;
      return BW_ERR_DEVICE;
    }
    return BW_OK;
  });
}

int bw_matmat(bw_hmat *h, const double *X, int64_t ldx, double *Y, int64_t ldy, int nrhs, int flags,
              void *stream) {
  if (!h) return BW_ERR_ARG;
  if (nrhs < 0) return BW_ERR_ARG;
  const bool tr = (flags & BW_TRANSPOSE) != 0;
  const int64_t nin = tr ? h->n_rows : h->n_cols, nout = tr ? h->n_cols : h->n_rows;
  if (ldx < nin || ldy < nout) {
    h->err = "leading dimension too small";
    return BW_ERR_ARG;
  }
  const int o = tr ? 1 : 0;
  if ((flags & BW_BF16) && h->has_mm && (o == 0 || h->has_t) && nrhs > 0) {
    // tensor-core path: BF16 matmat layout, kMmRhs right-hand sides per pass
    return guarded(h, [&] {
      if (!h->finalized || h->plan_only) throw StateError("bw_matmat needs a finalized handle with device data");
      if ((flags & (BW_FP64 | BW_FP32)) != 0) throw std::invalid_argument("flags must name exactly one precision");
      if ((nin && !X) || (nout && !Y)) throw std::invalid_argument("null matrix");
      if (X && Y) {
        const char *xb = reinterpret_cast<const char *>(X), *yb = reinterpret_cast<const char *>(Y);
        const int64_t xe = ((int64_t)(nrhs - 1) * ldx + nin) * 8, ye = ((int64_t)(nrhs - 1) * ldy + nout) * 8;
        if (xb < yb + ye && yb < xb + xe) throw std::invalid_argument("X and Y overlap");
      }
      BW_CUDA(cudaSetDevice(h->device));
      launch_matmat_tc(h, o, X, ldx, Y, ldy, nrhs, (flags & BW_PERMUTED) != 0, static_cast<cudaStream_t>(stream));
      return BW_OK;
    });
  }
  for (int k = 0; k < nrhs; k++) {
    int rc = bw_matvec(h, X + k * ldx, Y + k * ldy, flags, stream);
    if (rc != BW_OK) return rc;
  }
  return BW_OK;
}

int bw_mm_plan_export(const bw_hmat *h, int phase, int transposed, int64_t *n_chunks, int32_t *chunks,
                      int64_t *n_elems, uint16_t *data, int64_t *n_item_ptr, int32_t *item_ptr, int64_t *t8_len) {
  if (!h || phase < 1 || phase > 2) return BW_ERR_ARG;
  if (!h->finalized || !h->has_mm) return BW_ERR_STATE;
  const int o = transposed ? 1 : 0;
  if (o == 1 && !h->has_t) return BW_ERR_UNSUPPORTED;
  const bw::MmPhase &ph = h->mm[o].ph[phase - 1];
  if (n_chunks) *n_chunks = (int64_t)ph.chunks.size();
  if (n_elems) *n_elems = ph.n_elems;
  if (n_item_ptr) *n_item_ptr = (int64_t)ph.item_ptr.size();
  if (t8_len) *t8_len = h->mm[o].t8_len;
  if (chunks) std::memcpy(chunks, ph.chunks.data(), ph.chunks.size() * sizeof(bw::MmChunk));
  if (item_ptr) std::memcpy(item_ptr, ph.item_ptr.data(), ph.item_ptr.size() * sizeof(int32_t));
  if (data) {
    if (!h->plan_only) return BW_ERR_STATE;
    std::memcpy(data, h->mm_host[o][phase - 1].data(), (size_t)ph.n_elems * 2);
  }
  return BW_OK;
}

int bw_diagonal(bw_hmat *h, double *d, int flags) {
  if (!h || !d) return BW_ERR_ARG;
  return guarded(h, [&] {
    if (!h->finalized) throw StateError("bw_diagonal before bw_finalize");
    const int64_t n = (int64_t)h->diag_perm.size();
    if (flags & BW_PERMUTED) {
      std::memcpy(d, h->diag_perm.data(), (size_t)n * 8);
      return BW_OK;
    }
    // Hmat::diagonalOriginal (hmat.cc:240-254): permuted back with permutation_1_
    std::memset(d, 0, (size_t)n * 8);
    const int dof = h->dof;
    for (size_t i = 0; i < h->perm1.size(); i++)
      for (int j = 0; j < dof; j++) d[dof * h->perm1[i] + j] = h->diag_perm[dof * i + j];
    return BW_OK;
  });
}

int bw_info(const bw_hmat *h, int64_t *out, int n) {
  if (!h || !out) return BW_ERR_ARG;
  const int64_t v[] = {h->n_rows,
                       h->n_cols,
                       h->dof,
                       h->n_fr,
                       h->n_lr,
                       h->entries,
                       h->sum_rank,
                       h->op[0].n_panels,
                       h->dev_bytes,
                       h->grid,
                       (int64_t)h->op[0].ph[0].cp[0].chunks.size(),
                       (int64_t)h->op[0].ph[1].cp[0].chunks.size(),
                       h->stored};
  const int nv = (int)(sizeof(v) / sizeof(v[0]));
  for (int i = 0; i < n && i < nv; i++) out[i] = v[i];
  return BW_OK;
}

int bw_algorithmic_bytes(const bw_hmat *h, int precision, int64_t *bytes) {
  if (!h || !bytes) return BW_ERR_ARG;
  const int p = prec_index(precision);
  if (p < 0) return BW_ERR_ARG;
  int64_t b = h->entries * bw::esize_of(p) + 8 * (h->n_rows + h->n_cols);
  if (p == 2) b += 4 * ((int64_t)h->op[0].scale_fr.size() + 2 * (int64_t)h->op[0].scale_a.size());
  *bytes = b;
  return BW_OK;
}

int bw_last_error(const bw_hmat *h, char *buf, size_t len) {
  if (!buf || len == 0) return BW_ERR_ARG;
  std::string m;
  if (h) {
    m = h->err;
  } else {
    std::lock_guard<std::mutex> g(g_err_mu);
    m = g_last_create_error;
  }
  const size_t k = std::min(len - 1, m.size());
  std::memcpy(buf, m.data(), k);
  buf[k] = 0;
  return BW_OK;
}

int bw_plan_export(const bw_hmat *h, int precision, int phase, int transposed, int64_t *n_chunks, int32_t *chunks,
                   int64_t *n_elems, double *data, int64_t *n_item_ptr, int32_t *item_ptr) {
  if (!h || phase < 1 || phase > 2) return BW_ERR_ARG;
  const int p = prec_index(precision);
  if (p < 0 || !h->finalized || !(h->stored & (1 << p))) return BW_ERR_STATE;
  const int o = transposed ? 1 : 0;
  if (o == 1 && !h->has_t) return BW_ERR_UNSUPPORTED;
  const bw::PhasePlan &ph = h->op[o].ph[phase - 1];
  const bw::ChunkPlan &cp = ph.cp[p];
  if (n_chunks) *n_chunks = (int64_t)cp.chunks.size();
  if (n_elems) *n_elems = ph.n_elems[p];
  if (n_item_ptr) *n_item_ptr = (int64_t)cp.item_ptr.size();
  if (chunks) std::memcpy(chunks, cp.chunks.data(), cp.chunks.size() * sizeof(Chunk));  // kChunkWords int32 each
  if (item_ptr) std::memcpy(item_ptr, cp.item_ptr.data(), cp.item_ptr.size() * sizeof(int32_t));
  if (data) {
    if (!h->plan_only) return BW_ERR_STATE;
    const auto &buf = h->host_data[o][p][phase - 1];
    for (int64_t i = 0; i < ph.n_elems[p]; i++) {
      if (p == 0)
        data[i] = reinterpret_cast<const double *>(buf.data())[i];
      else if (p == 1)
        data[i] = reinterpret_cast<const float *>(buf.data())[i];
      else
        data[i] = bw::from_bf16(reinterpret_cast<const uint16_t *>(buf.data())[i]);
    }
  }
  return BW_OK;
}

int bw_plan_split(const bw_hmat *h, int precision, int phase, int transposed, int64_t *n_wide, int64_t *n_coop) {
  if (!h || !n_wide || !n_coop || phase < 1 || phase > 2) return BW_ERR_ARG;
  const int p = prec_index(precision);
  if (p < 0 || !h->finalized || !(h->stored & (1 << p))) return BW_ERR_STATE;
  const int o = transposed ? 1 : 0;
  if (o == 1 && !h->has_t) return BW_ERR_UNSUPPORTED;
  const bw::NarrowSplit sp = narrow_split(h->op[o].ph[phase - 1].cp[p], h->prob.tune);
  *n_wide = sp.wide;
  *n_coop = sp.coop;
  return BW_OK;
}

int bw_matvec_launches(const bw_hmat *h, int precision, int transposed, int64_t *n) {
  if (!h || !n) return BW_ERR_ARG;
  const int p = prec_index(precision);
  if (p < 0 || !h->finalized || !(h->stored & (1 << p))) return BW_ERR_STATE;
  const int o = transposed ? 1 : 0;
  if (o == 1 && !h->has_t) return BW_ERR_UNSUPPORTED;
  int64_t k = h->op[o].n_in > 0 ? 1 : 0;  // x gather
  for (int ph = 0; ph < 2; ph++) {
    const bw::ChunkPlan &cp = h->op[o].ph[ph].cp[p];
    const int64_t units = std::max<int64_t>(0, (int64_t)cp.item_ptr.size() - 1);
    if (ph == 1 && !cp.gsegs.empty()) k++;  // G2 gather
    if (cp.chunks.empty()) continue;
    const bw::NarrowSplit sp = narrow_split(cp, h->prob.tune);
    k += (sp.wide > 0 ? 1 : 0) + (sp.wide < units ? 1 : 0);
  }
  *n = k;
  return BW_OK;
}

int bw_set_timing(bw_hmat *h, int enable) {
  if (!h) return BW_ERR_ARG;
  h->timing = enable != 0;
  h->ev_used = 0;
  return BW_OK;
}

int bw_timing_read_launches(bw_hmat *h, double *ms, int64_t *n_matvecs) {
  if (!h || !ms) return BW_ERR_ARG;
  return guarded(h, [&] {
    for (int k = 0; k < kTimedLaunches; k++) ms[k] = 0.0;
    if (h->ev_used > 0) {
      BW_CUDA(cudaSetDevice(h->device));
      BW_CUDA(cudaEventSynchronize(h->ev_pool[kEv * h->ev_used - 1]));
      for (size_t i = 0; i < h->ev_used; i++)
        for (int k = 0; k < kTimedLaunches; k++) {
          float v = 0.0f;
          BW_CUDA(cudaEventElapsedTime(&v, h->ev_pool[kEv * i + k], h->ev_pool[kEv * i + k + 1]));
          ms[k] += v;
        }
    }
    if (n_matvecs) *n_matvecs = (int64_t)h->ev_used;
    h->ev_used = 0;
    return BW_OK;
  });
}

int bw_timing_read(bw_hmat *h, double *ms, int64_t *n_matvecs) {
  if (!h || !ms) return BW_ERR_ARG;
  double d[kTimedLaunches];
  const int st = bw_timing_read_launches(h, d, n_matvecs);
  if (st != BW_OK) return st;
  ms[0] = d[0];
  ms[1] = d[1] + d[2];
  ms[2] = d[3];
  ms[3] = d[4] + d[5];
  return BW_OK;
}

int bw_phase_bytes(const bw_hmat *h, int precision, int transposed, int64_t *phase1, int64_t *phase2) {
  if (!h || !phase1 || !phase2) return BW_ERR_ARG;
  const int p = prec_index(precision);
  if (p < 0) return BW_ERR_ARG;
  const int o = transposed ? 1 : 0;
  if (o == 1 && !h->has_t) return BW_ERR_UNSUPPORTED;
  // Algorithmic bytes per launch (the split of bw_algorithmic_bytes): stored
  // entries the launch streams, x (8 bytes per input) counted in phase 1, y
  // (8 bytes per output) and the BF16 block scales in phase 2.
  const int es = bw::esize_of(p);
  int64_t e[2] = {0, 0};
  for (int ph = 0; ph < 2; ph++)
    for (const bw::Item &it : h->op[o].ph[ph].items) e[ph] += int64_t(it.h) * it.ncols;
  *phase1 = e[0] * es + 8 * h->op[o].n_in;
  *phase2 = e[1] * es + 8 * h->op[o].n_out;
  if (p == 2) *phase2 += 4 * ((int64_t)h->op[o].scale_fr.size() + 2 * (int64_t)h->op[o].scale_a.size());
  return BW_OK;
}

int bw_plan_gather(const bw_hmat *h, int precision, int transposed, int64_t *n, int32_t *runs) {
  if (!h || !n) return BW_ERR_ARG;
  const int p = prec_index(precision);
  if (p < 0 || !h->finalized || !(h->stored & (1 << p))) return BW_ERR_STATE;
  const int o = transposed ? 1 : 0;
  if (o == 1 && !h->has_t) return BW_ERR_UNSUPPORTED;
  const std::vector<bw::GatherSeg> &g = h->op[o].ph[1].cp[p].gsegs;
  *n = (int64_t)g.size();
  if (runs) std::memcpy(runs, g.data(), g.size() * sizeof(bw::GatherSeg));
  return BW_OK;
}

int bw_plan_tscale(const bw_hmat *h, int transposed, int64_t *n, float *out) {
  if (!h || !n) return BW_ERR_ARG;
  if (!h->finalized) return BW_ERR_STATE;
  const int o = transposed ? 1 : 0;
  if (o == 1 && !h->has_t) return BW_ERR_UNSUPPORTED;
  const std::vector<float> &ts = h->op[o].t_scale;
  *n = (int64_t)ts.size();
  if (out) std::memcpy(out, ts.data(), ts.size() * 4);
  return BW_OK;
}

}  // extern "C"

namespace {

int file_fail(const std::string &m, int code) {
  std::lock_guard<std::mutex> g(g_err_mu);
  g_last_create_error = m;
  return code;
}

// Block-file entries have no handle: messages go where bw_create's do.
template <typename F> int file_guarded(F &&f) {
  try {
    return f();
  } catch (const std::invalid_argument &e) {
    return file_fail(e.what(), BW_ERR_ARG);
  } catch (const std::bad_alloc &) {
    return file_fail("host allocation failed", BW_ERR_OOM);
  } catch (const std::exception &e) {
    return file_fail(e.what(), BW_ERR_IO);
  }
}

// Handle-less device entries: as file_guarded, with CUDA and allocation
// failures reported as such.
template <typename F> int device_guarded(F &&f) {
  try {
    return f();
  } catch (const CudaError &e) {
    return file_fail(e.what(), BW_ERR_CUDA);
  } catch (const OomError &e) {
    return file_fail(e.what(), BW_ERR_OOM);
  } catch (const std::bad_alloc &) {
    return file_fail("host allocation failed", BW_ERR_OOM);
  } catch (const std::exception &e) {
    return file_fail(e.what(), BW_ERR_ARG);
  }
}

// Block extent in scalar units from pattern coordinates in points; throws
// unless 0 <= a0 < a1 <= limit.
int64_t extent(int64_t a0, int64_t a1, int64_t limit, int64_t dof, const char *what, int64_t k) {
  if (!(0 <= a0 && a0 < a1 && a1 <= limit))
    throw std::invalid_argument(std::string(what) + " block " + std::to_string(k) + " lies outside the matrix");
  return (a1 - a0) * dof;
}

// Copy in parallel (block data can be gigabytes).
void par_copy(void *dst, const void *src, int64_t bytes) {
  const int64_t step = int64_t(16) << 20;
#pragma omp parallel for schedule(static)
  for (int64_t o = 0; o < bytes; o += step)
    std::memcpy(static_cast<char *>(dst) + o, static_cast<const char *>(src) + o, (size_t)std::min(step, bytes - o));
}

// Shared checks and launch of the observation-field kernels.
template <typename Launch>
int fields_entry(const char *name, int device, int64_t n_elems, const double *records, const double *dd, double G,
                 double nu, int64_t n_pts, const double *pts, const double *stress, const double *disp, int threads,
                 Launch &&launch) {
  return device_guarded([&] {
    if (!records || !dd || n_elems < 1 || n_pts < 0 || (n_pts > 0 && (!pts || (!stress && !disp))))
      throw std::invalid_argument(std::string(name) + ": null or empty argument");
    if (n_elems >= (int64_t(1) << 31)) throw std::invalid_argument(std::string(name) + ": more than 2^31 elements");
    if (!(G > 0.0) || !(nu > -1.0 && nu < 0.5)) throw std::invalid_argument(std::string(name) + ": bad G or nu");
    if (n_pts == 0) return BW_OK;
    BW_CUDA(cudaSetDevice(device));
    int sms = 0;
    BW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int64_t need = (n_pts + threads - 1) / threads;
    launch(static_cast<int>(std::min<int64_t>(need, int64_t(std::max(1, sms)) * 4)));
    BW_CUDA(cudaGetLastError());
    return BW_OK;
  });
}

}  // namespace

extern "C" {

int bw_file_write(const char *path, int dof, int64_t n_rows, int64_t n_cols, const int64_t *perm0,
                  const int64_t *perm1, int64_t n_fr, const int64_t *fr, const double *fr_data, int64_t n_lr,
                  const int64_t *lr, const double *lr_data, const double *lr_error) {
  return file_guarded([&] {
    if (!path) throw std::invalid_argument("null path");
    if (dof < 1 || n_rows < 0 || n_cols < 0 || n_fr < 0 || n_lr < 0)
      throw std::invalid_argument("bad sizes or block counts");
    if ((n_fr && (!fr || !fr_data)) || (n_lr && (!lr || !lr_data)))
      throw std::invalid_argument("null pattern or block data");
    const int64_t rp = n_rows / dof, cp = n_cols / dof;
    std::vector<int64_t> frp(6 * n_fr), lrp(6 * n_lr), frl(n_fr), al(n_lr), bl(n_lr);
    std::vector<const double *> frb(n_fr), ab(n_lr), bb(n_lr);
    int64_t o = 0;
    for (int64_t k = 0; k < n_fr; k++) {
      const int64_t *c = fr + 4 * k;
      const int64_t m = extent(c[0], c[2], rp, dof, "FR", k), n = extent(c[1], c[3], cp, dof, "FR", k);
      int64_t *q = &frp[6 * k];
      q[0] = k;
      for (int i = 0; i < 4; i++) q[1 + i] = c[i];
      q[5] = 0;
      frb[k] = fr_data + o;
      frl[k] = m;
      o += m * n;
    }
    o = 0;
    for (int64_t k = 0; k < n_lr; k++) {
      const int64_t *c = lr + 5 * k;
      const int64_t m = extent(c[0], c[2], rp, dof, "LR", k), n = extent(c[1], c[3], cp, dof, "LR", k), r = c[4];
      if (r < 0) throw std::invalid_argument("LR block " + std::to_string(k) + " has a negative rank");
      int64_t *q = &lrp[6 * k];
      q[0] = k;
      for (int i = 0; i < 5; i++) q[1 + i] = c[i];
      ab[k] = lr_data + o;
      al[k] = std::max<int64_t>(1, m);
      bb[k] = lr_data + o + m * r;
      bl[k] = std::max<int64_t>(1, r);
      o += r * (m + n);
    }
    bw::FileBlocks b;
    b.dof = dof;
    b.n_rows = n_rows;
    b.n_cols = n_cols;
    b.perm0 = perm0;
    b.perm1 = perm1;
    b.n_fr = n_fr;
    b.fr_pattern = frp.data();
    b.fr = frb.data();
    b.fr_ld = frl.data();
    b.n_lr = n_lr;
    b.lr_pattern = lrp.data();
    b.lr_a = ab.data();
    b.lr_a_ld = al.data();
    b.lr_b = bb.data();
    b.lr_b_ld = bl.data();
    b.lr_error = lr_error;
    bw::write_block_file(path, b);
    return BW_OK;
  });
}

int bw_file_write_blocks(const char *path, int dof, int64_t n_rows, int64_t n_cols, const int64_t *perm0,
                         const int64_t *perm1, int64_t n_fr, const int64_t *fr_pattern, const double *const *fr,
                         const int64_t *fr_ld, int64_t n_lr, const int64_t *lr_pattern, const double *const *lr_a,
                         const int64_t *lr_a_ld, const double *const *lr_b, const int64_t *lr_b_ld,
                         const double *lr_error) {
  return file_guarded([&] {
    if (!path) throw std::invalid_argument("null path");
    bw::FileBlocks b;
    b.dof = dof;
    b.n_rows = n_rows;
    b.n_cols = n_cols;
    b.perm0 = perm0;
    b.perm1 = perm1;
    b.n_fr = n_fr;
    b.fr_pattern = fr_pattern;
    b.fr = fr;
    b.fr_ld = fr_ld;
    b.n_lr = n_lr;
    b.lr_pattern = lr_pattern;
    b.lr_a = lr_a;
    b.lr_a_ld = lr_a_ld;
    b.lr_b = lr_b;
    b.lr_b_ld = lr_b_ld;
    b.lr_error = lr_error;
    bw::write_block_file(path, b);
    return BW_OK;
  });
}

int bw_file_info(const char *path, int64_t info[9]) {
  return file_guarded([&] {
    if (!path || !info) throw std::invalid_argument("null path or output");
    auto f = bw::BlockFile::open(path, false);
    const bw::FileHeader &h = f->header();
    const int64_t v[9] = {h.dof,        h.n_rows,     h.n_cols, h.n_fr, h.n_lr, h.fr_entries,
                          h.lr_entries, h.flags & 1, f->file_bytes()};
    std::memcpy(info, v, sizeof v);
    return BW_OK;
  });
}

int bw_file_read(const char *path, int verify, int64_t *fr, int64_t *lr, double *fr_data, double *lr_data,
                 int64_t *perm0, int64_t *perm1, double *lr_error, int64_t *fr_pattern, int64_t *lr_pattern) {
  return file_guarded([&] {
    if (!path) throw std::invalid_argument("null path");
    auto f = bw::BlockFile::open(path, verify != 0);
    const bw::FileHeader &h = f->header();
    if ((h.n_fr && !fr) || (h.n_lr && !lr) || (h.n_rows && !perm0) || (h.n_cols && !perm1))
      throw std::invalid_argument("null output array");
    const int64_t *fp = f->fr_pattern(), *lp = f->lr_pattern();
    for (int64_t k = 0; k < h.n_fr; k++)
      for (int i = 0; i < 4; i++) fr[4 * k + i] = fp[6 * k + 1 + i];
    for (int64_t k = 0; k < h.n_lr; k++)
      for (int i = 0; i < 5; i++) lr[5 * k + i] = lp[6 * k + 1 + i];
    if (fr_pattern) std::memcpy(fr_pattern, fp, (size_t)(48 * h.n_fr));
    if (lr_pattern) std::memcpy(lr_pattern, lp, (size_t)(48 * h.n_lr));
    if (h.n_rows) std::memcpy(perm0, f->perm0(), (size_t)(8 * (h.n_rows / h.dof)));
    if (h.n_cols) std::memcpy(perm1, f->perm1(), (size_t)(8 * (h.n_cols / h.dof)));
    if (lr_error) {
      if (f->lr_error())
        std::memcpy(lr_error, f->lr_error(), (size_t)(8 * h.n_lr));
      else
        std::fill(lr_error, lr_error + h.n_lr, 0.0);
    }
    if (fr_data) par_copy(fr_data, f->fr_data(), 8 * h.fr_entries);
    if (lr_data) par_copy(lr_data, f->lr_data(), 8 * h.lr_entries);
    return BW_OK;
  });
}

int bw_create_from_file(const char *path, int device, int verify, bw_hmat **out) {
  if (!out) return BW_ERR_ARG;
  *out = nullptr;
  std::shared_ptr<bw::BlockFile> f;
  int rc = file_guarded([&] {
    if (!path) throw std::invalid_argument("null path");
    f = bw::BlockFile::open(path, verify != 0);
    return BW_OK;
  });
  if (rc != BW_OK) return rc;
  const bw::FileHeader &hd = f->header();
  bw_hmat *h = nullptr;
  rc = bw_create((int)hd.dof, hd.n_rows, hd.n_cols, f->perm0(), f->perm1(), device, &h);
  if (rc != BW_OK) return rc;
  const int64_t d = hd.dof;
  const int64_t *fp = f->fr_pattern(), *lp = f->lr_pattern();
  const double *fdat = f->fr_data(), *ldat = f->lr_data();
  int64_t o = 0;
  for (int64_t k = 0; k < hd.n_fr && rc == BW_OK; k++) {
    const int64_t *c = fp + 6 * k;
    const int64_t m = (c[3] - c[1]) * d, n = (c[4] - c[2]) * d;
    rc = bw_add_full(h, c[1] * d, c[2] * d, m, n, fdat + o, m);
    o += m * n;
  }
  o = 0;
  for (int64_t k = 0; k < hd.n_lr && rc == BW_OK; k++) {
    const int64_t *c = lp + 6 * k;
    const int64_t m = (c[3] - c[1]) * d, n = (c[4] - c[2]) * d, r = c[5];
    rc = bw_add_lowrank(h, c[1] * d, c[2] * d, m, n, r, ldat + o, std::max<int64_t>(1, m), ldat + o + m * r,
                        std::max<int64_t>(1, r));
    o += r * (m + n);
  }
  if (rc != BW_OK) {
    file_fail(std::string(path) + ": " + h->err, rc);
    bw_destroy(h);
    return rc;
  }
  h->borrowed = f;
  *out = h;
  return BW_OK;
}

int bw_s0_fields(int device, int64_t n_elems, const double *records, const double *dd, double G, double nu,
                 int64_t n_pts, const double *pts, double *stress, double *disp, void *stream) {
  return fields_entry("bw_s0_fields", device, n_elems, records, dd, G, nu, n_pts, pts, stress, disp, bw::kS0Threads,
                      [&](int grid) {
                        bw::s0_fields_kernel<<<grid, bw::kS0Threads, 0, static_cast<cudaStream_t>(stream)>>>(
                            records, dd, static_cast<int>(n_elems), pts, static_cast<long long>(n_pts), G, nu,
                            stress, disp);
                      });
}

int bw_r0_fields(int device, int64_t n_elems, const double *records, const double *dd, double G, double nu,
                 int64_t n_pts, const double *pts, double *stress, double *disp, void *stream) {
  return fields_entry("bw_r0_fields", device, n_elems, records, dd, G, nu, n_pts, pts, stress, disp,
                      bw::kR0FieldThreads, [&](int grid) {
                        bw::r0_fields_kernel<<<grid, bw::kR0FieldThreads, 0, static_cast<cudaStream_t>(stream)>>>(
                            records, dd, static_cast<int>(n_elems), pts, static_cast<long long>(n_pts), G, nu,
                            stress, disp);
                      });
}

int bw_r0_assemble_fr(int device, int64_t n_elems, const double *records, double G, double nu, int64_t n_fr,
                      const int64_t *fr, const int64_t *perm, int64_t n_points, double *out, int64_t out_len,
                      void *stream) {
  return device_guarded([&] {
    if (!records || n_elems < 1 || n_fr < 0 || n_points < 1 || (n_fr && (!fr || !perm || !out)))
      throw std::invalid_argument("bw_r0_assemble_fr: null or empty argument");
    if (n_elems >= (int64_t(1) << 31) || n_points >= (int64_t(1) << 31))
      throw std::invalid_argument("bw_r0_assemble_fr: more than 2^31 elements");
    if (!(G > 0.0) || !(nu > -1.0 && nu < 0.5)) throw std::invalid_argument("bw_r0_assemble_fr: bad G or nu");
    // every index the kernel reads or writes is checked here
    std::vector<int32_t> p32(n_points);
    for (int64_t i = 0; i < n_points; i++) {
      if (perm[i] < 0 || perm[i] >= n_elems) throw std::invalid_argument("bw_r0_assemble_fr: perm out of range");
      p32[i] = (int32_t)perm[i];
    }
    std::vector<bw::AsmBlock> blocks(n_fr);
    std::vector<bw::AsmTile> tiles;
    int64_t off = 0;
    for (int64_t k = 0; k < n_fr; k++) {
      const int64_t i0 = fr[4 * k], j0 = fr[4 * k + 1], i1 = fr[4 * k + 2], j1 = fr[4 * k + 3];
      if (!(0 <= i0 && i0 < i1 && i1 <= n_points && 0 <= j0 && j0 < j1 && j1 <= n_points))
        throw std::invalid_argument("bw_r0_assemble_fr: block " + std::to_string(k) + " outside the matrix");
      blocks[k] = {off, (int)i0, (int)j0, (int)(i1 - i0), (int)(j1 - j0)};
      for (int64_t ti = 0; ti < i1 - i0; ti += bw::kAsmTile)
        for (int64_t tj = 0; tj < j1 - j0; tj += bw::kAsmTile) tiles.push_back({(int)k, (int)ti, (int)tj, 0});
      off += 9 * (i1 - i0) * (j1 - j0);
    }
    if (off > out_len) throw std::invalid_argument("bw_r0_assemble_fr: out holds fewer than the blocks' entries");
    if (tiles.empty()) return BW_OK;
    BW_CUDA(cudaSetDevice(device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    void *d_rec = nullptr, *d_perm = nullptr, *d_blk = nullptr, *d_tile = nullptr;
    auto release = [&] {
      cudaFree(d_rec);
      cudaFree(d_perm);
      cudaFree(d_blk);
      cudaFree(d_tile);
    };
    try {
      const size_t rb = sizeof(double) * bw::r0::kFrameDoubles * (size_t)n_elems;
      BW_CUDA(cudaMalloc(&d_rec, rb));
      BW_CUDA(cudaMalloc(&d_perm, 4 * p32.size()));
      BW_CUDA(cudaMalloc(&d_blk, sizeof(bw::AsmBlock) * blocks.size()));
      BW_CUDA(cudaMalloc(&d_tile, sizeof(bw::AsmTile) * tiles.size()));
      BW_CUDA(cudaMemcpyAsync(d_rec, records, rb, cudaMemcpyHostToDevice, st));
      BW_CUDA(cudaMemcpyAsync(d_perm, p32.data(), 4 * p32.size(), cudaMemcpyHostToDevice, st));
      BW_CUDA(cudaMemcpyAsync(d_blk, blocks.data(), sizeof(bw::AsmBlock) * blocks.size(), cudaMemcpyHostToDevice, st));
      BW_CUDA(cudaMemcpyAsync(d_tile, tiles.data(), sizeof(bw::AsmTile) * tiles.size(), cudaMemcpyHostToDevice, st));
      const long long nt = (long long)tiles.size();
      const int grid = (int)std::min<long long>(nt, 148LL * 8);
      bw::r0_fr_assemble_kernel<<<grid, bw::kAsmTile * bw::kAsmTile, 0, st>>>(
          static_cast<const double *>(d_rec), static_cast<const int *>(d_perm),
          static_cast<const bw::AsmBlock *>(d_blk), static_cast<const bw::AsmTile *>(d_tile), nt, G, nu, out);
      BW_CUDA(cudaGetLastError());
      BW_CUDA(cudaStreamSynchronize(st));
    } catch (...) {
      cudaStreamSynchronize(st);
      release();
      throw;
    }
    release();
    return BW_OK;
  });
}

int bw_r0_aca(int device, int64_t n_elems, const double *records, double G, double nu, int64_t n_lr,
              const int64_t *lr, const int64_t *perm, int64_t n_points, double eps, int cap_blocks,
              double *factors_a, int64_t a_len, double *factors_b, int64_t b_len, int32_t *rank_out,
              double *err_out, void *stream) {
  return device_guarded([&] {
    if (!records || n_elems < 1 || n_lr < 0 || n_points < 1 || (n_lr && (!lr || !perm || !factors_a ||
                                                                        !factors_b || !rank_out || !err_out)))
      throw std::invalid_argument("bw_r0_aca: null or empty argument");
    if (n_elems >= (int64_t(1) << 31) || n_points >= (int64_t(1) << 31) || n_lr >= (int64_t(1) << 31))
      throw std::invalid_argument("bw_r0_aca: more than 2^31 elements or blocks");
    if (!(G > 0.0) || !(nu > -1.0 && nu < 0.5) || !(eps > 0.0) || cap_blocks < 1)
      throw std::invalid_argument("bw_r0_aca: bad G, nu, eps or capacity");
    std::vector<int32_t> p32(n_points);
    for (int64_t i = 0; i < n_points; i++) {
      if (perm[i] < 0 || perm[i] >= n_elems) throw std::invalid_argument("bw_r0_aca: perm out of range");
      p32[i] = (int32_t)perm[i];
    }
    std::vector<bw::AcaBlock> blocks(n_lr);
    int64_t ao = 0, bo = 0, slot = 1;
    for (int64_t k = 0; k < n_lr; k++) {
      const int64_t i0 = lr[4 * k], j0 = lr[4 * k + 1], i1 = lr[4 * k + 2], j1 = lr[4 * k + 3];
      if (!(0 <= i0 && i0 < i1 && i1 <= n_points && 0 <= j0 && j0 < j1 && j1 <= n_points))
        throw std::invalid_argument("bw_r0_aca: block " + std::to_string(k) + " outside the matrix");
      const int64_t n0 = i1 - i0, n1 = j1 - j0, cap = std::min<int64_t>(cap_blocks, std::min(n0, n1));
      blocks[k] = {ao, bo, 0, (int)i0, (int)j0, (int)n0, (int)n1, (int)cap, 0};
      ao += 9 * n0 * cap;
      bo += 9 * n1 * cap;
      slot = std::max<int64_t>(slot, 9 * n1 + n0 + n1 + 2);  // row band + used flags (ints)
    }
    if (ao > a_len || bo > b_len) throw std::invalid_argument("bw_r0_aca: factor storage smaller than the capacity");
    if (!n_lr) return BW_OK;
    BW_CUDA(cudaSetDevice(device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = (int)std::min<int64_t>(n_lr, 148 * 4);
    void *d_rec = nullptr, *d_perm = nullptr, *d_blk = nullptr, *d_scr = nullptr, *d_rank = nullptr, *d_err = nullptr;
    auto release = [&] {
      for (void *q : {d_rec, d_perm, d_blk, d_scr, d_rank, d_err}) cudaFree(q);
    };
    try {
      const size_t rb = sizeof(double) * bw::r0::kFrameDoubles * (size_t)n_elems;
      BW_CUDA(cudaMalloc(&d_rec, rb));
      BW_CUDA(cudaMalloc(&d_perm, 4 * p32.size()));
      BW_CUDA(cudaMalloc(&d_blk, sizeof(bw::AcaBlock) * blocks.size()));
      BW_CUDA(cudaMalloc(&d_scr, sizeof(double) * (size_t)slot * grid));
      BW_CUDA(cudaMalloc(&d_rank, 4 * (size_t)n_lr));
      BW_CUDA(cudaMalloc(&d_err, 8 * (size_t)n_lr));
      BW_CUDA(cudaMemcpyAsync(d_rec, records, rb, cudaMemcpyHostToDevice, st));
      BW_CUDA(cudaMemcpyAsync(d_perm, p32.data(), 4 * p32.size(), cudaMemcpyHostToDevice, st));
      BW_CUDA(cudaMemcpyAsync(d_blk, blocks.data(), sizeof(bw::AcaBlock) * blocks.size(), cudaMemcpyHostToDevice, st));
      bw::r0_aca_kernel<<<grid, bw::kAcaThreads, 0, st>>>(
          static_cast<const double *>(d_rec), static_cast<const int *>(d_perm),
          static_cast<const bw::AcaBlock *>(d_blk), (int)n_lr, G, nu, eps, factors_a, factors_b,
          static_cast<double *>(d_scr), slot, static_cast<int *>(d_rank), static_cast<double *>(d_err));
      BW_CUDA(cudaGetLastError());
      BW_CUDA(cudaMemcpyAsync(rank_out, d_rank, 4 * (size_t)n_lr, cudaMemcpyDeviceToHost, st));
      BW_CUDA(cudaMemcpyAsync(err_out, d_err, 8 * (size_t)n_lr, cudaMemcpyDeviceToHost, st));
      BW_CUDA(cudaStreamSynchronize(st));
    } catch (...) {
      cudaStreamSynchronize(st);
      release();
      throw;
    }
    release();
    for (int64_t k = 0; k < n_lr; k++)
      if (rank_out[k] > 0) rank_out[k] *= 3;  // scalar rank (LRB_pattern flag); -1: capacity too small
    return BW_OK;
  });
}

int bw_destroy(bw_hmat *h) {
  if (!h) return BW_OK;
  h->release();
  delete h;
  return BW_OK;
}

}  // extern "C"
