// RGF selected inversion / selected solve, Sancho-Rubio and the generator-form
// transport solve: host-side orchestration of the device kernels, and the C ABI
// of libqtxrgf.so (declared in include/qtx_rgf.h).
//
// Every sweep runs on the caller's stream over one energy batch at a time
// (qttools' max_batch_size slicing, src/qttools/utils/solvers_utils.py:7-32);
// the per-block dense recursion state (x_i, X^<_i, X^>_i) of a batch lives in
// one stream-ordered device allocation.  Dense DSDBSparse blocks are read and
// written in place (zero copy); blocks with a sparse pattern are gathered to /
// scattered from dense scratch blocks.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <condition_variable>
#include <deque>
#include <exception>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kernels.h"

thread_local int64_t* g_qtx_launch_counter = nullptr;

void qtx_opt_in_smem(const void* func, size_t bytes) {
  static std::mutex m;
  static std::map<std::pair<const void*, int>, size_t> set_bytes;
  int dev = 0;
  QTX_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(m);
  size_t& have = set_bytes[{func, dev}];
  if (bytes <= have) return;
  QTX_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  have = bytes;
}

// Per-kernel-class CUDA-event timing of the launches a context issues
// (enabled by qtx_ctx_set_timing): 0 = complex GEMM, 1 = inverse.
struct TimedLaunch {
  cudaEvent_t start, stop;
  int kind;
  double flops;
};

struct GraphKey {
  std::vector<uintptr_t> v;
  bool operator==(const GraphKey& o) const { return v == o.v; }
};

struct GraphEntry {
  GraphKey key;
  void* mem = nullptr;  // work space, stream-ordered allocation
  size_t bytes = 0;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t done = nullptr;  // recorded after every use of `mem`
  int64_t launches = 0;
  uint64_t last_use = 0;
};

// Graph captures and the library's own device-wide synchronisation never
// overlap: a device-wide synchronisation (or cudaFree) issued by one thread
// while another thread's stream is capturing invalidates that capture.
std::mutex g_capture_mutex;

// Small LRU cache of captured sweeps (each holds its work space).  Nothing here
// synchronises the device: an evicted entry's memory is freed in stream order
// after its last use (its `done` event), and an executable graph still in
// flight is released by the driver when it completes.
struct GraphCache {
  std::vector<GraphEntry> entries;
  uint64_t clock = 0;
  size_t capacity = 8;
  GraphEntry* find(const GraphKey& k) {
    for (auto& e : entries)
      if (e.key == k) {
        e.last_use = ++clock;
        return &e;
      }
    return nullptr;
  }
  static void release(GraphEntry& e, cudaStream_t s) {
    if (e.exec) cudaGraphExecDestroy(e.exec);
    if (e.mem) {
      if (e.done) cudaStreamWaitEvent(s, e.done, 0);
      cudaFreeAsync(e.mem, s);
    }
    if (e.done) cudaEventDestroy(e.done);
    e.exec = nullptr;
    e.mem = nullptr;
    e.done = nullptr;
  }
  GraphEntry* insert(const GraphKey& k, cudaStream_t s) {
    if (entries.size() >= capacity) {
      size_t victim = 0;
      for (size_t i = 1; i < entries.size(); ++i)
        if (entries[i].last_use < entries[victim].last_use) victim = i;
      release(entries[victim], s);
      entries.erase(entries.begin() + victim);
    }
    entries.push_back(GraphEntry{});
    entries.back().key = k;
    entries.back().last_use = ++clock;
    return &entries.back();
  }
  void erase(const GraphKey& k, cudaStream_t s) {
    for (size_t i = 0; i < entries.size(); ++i)
      if (entries[i].key == k) {
        release(entries[i], s);
        entries.erase(entries.begin() + i);
        return;
      }
  }
  void clear(cudaStream_t s) {
    for (auto& e : entries) release(e, s);
    entries.clear();
  }
};

// Pinned host words for small device-to-host reads (convergence counters).
// Process-wide and never freed: cudaFreeHost may synchronise the device.
std::mutex g_pinned_mutex;
std::vector<int*> g_pinned_free;
int* pinned_take() {
  std::lock_guard<std::mutex> lk(g_pinned_mutex);
  if (!g_pinned_free.empty()) {
    int* p = g_pinned_free.back();
    g_pinned_free.pop_back();
    return p;
  }
  int* p = nullptr;
  if (cudaMallocHost(&p, 4096) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
void pinned_give(int* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_pinned_mutex);
  g_pinned_free.push_back(p);
}

// Ring of page-locked host slots for the host-buffer streaming: every
// host<->device copy of that mode goes through it (the DMA engines read and
// write page-locked memory at full speed; the caller's arrays are pageable).
// Rings come from a process-wide pool and are never freed: cudaFreeHost may
// synchronise the device.
struct PinRing {
  static constexpr int kSlots = 8;
  static constexpr size_t kSlotBytes = 64u << 20;
  char* base = nullptr;
  cudaEvent_t ev[kSlots] = {};  // last DMA from / to each slot
  char* slot(int i) const { return base + (size_t)i * kSlotBytes; }
};
std::mutex g_ring_mutex;
std::vector<PinRing*> g_ring_free;
PinRing* ring_take() {
  {
    std::lock_guard<std::mutex> lk(g_ring_mutex);
    if (!g_ring_free.empty()) {
      PinRing* r = g_ring_free.back();
      g_ring_free.pop_back();
      return r;
    }
  }
  PinRing* r = new PinRing();
  if (cudaMallocHost(reinterpret_cast<void**>(&r->base), PinRing::kSlots * PinRing::kSlotBytes) != cudaSuccess) {
    cudaGetLastError();
    delete r;
    return nullptr;
  }
  for (auto& e : r->ev) {
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      e = nullptr;
    }
  }
  return r;
}
void ring_give(PinRing* r) {
  if (!r) return;
  for (auto& e : r->ev)
    if (e) cudaEventSynchronize(e);
  std::lock_guard<std::mutex> lk(g_ring_mutex);
  g_ring_free.push_back(r);
}

struct qtx_ctx {
  int device = 0;
  GraphCache graphs;
  cudaStream_t capture_stream = nullptr;  // graphs are captured here (the legacy stream cannot be)
  bool capturing = false;
  int64_t graph_replays = 0;
  std::string last_error;
  int64_t launches = 0;
  size_t mem_limit = 0;
  int* h_pinned = nullptr;     // pinned host words (process-wide pool)
  int* d_pinned = nullptr;     // their device alias: status words are stored there by a kernel
  PinRing* ring = nullptr;     // page-locked staging of the host-buffer mode (process-wide pool)
  bool timing = false;
  std::vector<TimedLaunch> timed;
  std::vector<cudaEvent_t> event_pool;
  double acc_ms[2] = {0, 0};
  double acc_flops[2] = {0, 0};
  int64_t acc_launches[2] = {0, 0};
};

thread_local qtx_ctx* g_timing_ctx = nullptr;

static cudaEvent_t pool_event(qtx_ctx* c) {
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// Bracket one launch with events when timing is on.
struct TimedScope {
  qtx_ctx* c;
  cudaStream_t s;
  TimedLaunch t;
  TimedScope(int kind, double flops, cudaStream_t stream) : c(g_timing_ctx), s(stream) {
    if (!c || !c->timing || c->capturing) { c = nullptr; return; }
    t.kind = kind;
    t.flops = flops;
    t.start = pool_event(c);
    t.stop = pool_event(c);
    cudaEventRecord(t.start, s);
  }
  ~TimedScope() {
    if (!c) return;
    cudaEventRecord(t.stop, s);
    c->timed.push_back(t);
  }
};

static void drain_timing(qtx_ctx* c) {
  for (auto& t : c->timed) {
    cudaEventSynchronize(t.stop);
    float ms = 0;
    cudaEventElapsedTime(&ms, t.start, t.stop);
    c->acc_ms[t.kind] += ms;
    c->acc_flops[t.kind] += t.flops;
    c->acc_launches[t.kind] += 1;
    c->event_pool.push_back(t.start);
    c->event_pool.push_back(t.stop);
  }
  c->timed.clear();
}

namespace {

constexpr cplx ONE = {1.0, 0.0};
constexpr cplx ZERO = {0.0, 0.0};
constexpr cplx MONE = {-1.0, 0.0};

struct LaunchScope {
  int64_t* prev;
  qtx_ctx* prev_ctx;
  explicit LaunchScope(qtx_ctx* c) : prev(g_qtx_launch_counter), prev_ctx(g_timing_ctx) {
    g_qtx_launch_counter = &c->launches;
    g_timing_ctx = c;
  }
  ~LaunchScope() {
    g_qtx_launch_counter = prev;
    g_timing_ctx = prev_ctx;
  }
};

// Stream-ordered device allocation (cudaMallocAsync on the context's pool).
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(size_t bytes, cudaStream_t s) : stream_(s), bytes_(bytes) {
    if (bytes == 0) return;
    ptr_ = qtx_malloc_async(bytes, s);
    if (!ptr_) throw QtxError(QTX_E_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    release();
    ptr_ = o.ptr_; stream_ = o.stream_; bytes_ = o.bytes_;
    o.ptr_ = nullptr;
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (ptr_) cudaFreeAsync(ptr_, stream_);
    ptr_ = nullptr;
  }
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(ptr_); }

 private:
  void* ptr_ = nullptr;
  cudaStream_t stream_ = nullptr;
  size_t bytes_ = 0;
};

inline int bidx(int i, int j) { return 2 * i + j; }

// ---------------------------------------------------------------------------
// DSDBSparse block access
// ---------------------------------------------------------------------------
struct Btd {
  const qtx_btd_desc* d = nullptr;
  cplx* data = nullptr;

  int nb() const { return d->num_blocks; }
  int size(int i) const { return d->block_sizes[i]; }
  int64_t off(int k) const { return d->block_offset[k]; }
  int64_t nnz(int k) const { return d->block_nnz[k]; }
  const int32_t* index(int k) const { return d->block_index ? d->block_index[k] : nullptr; }
  bool empty(int k) const { return off(k) < 0 || nnz(k) == 0; }
  bool dense(int k) const { return !index(k) && !empty(k); }
};

void validate_desc(const qtx_btd_desc* d, const char* name) {
  if (!d) throw QtxError(QTX_E_INVAL, std::string(name) + ": missing block descriptor");
  if (d->num_blocks < 1) throw QtxError(QTX_E_INVAL, std::string(name) + ": num_blocks < 1");
  if (!d->block_sizes || !d->block_offset || !d->block_nnz)
    throw QtxError(QTX_E_INVAL, std::string(name) + ": descriptor arrays missing");
  if (d->stack_size < 0) throw QtxError(QTX_E_INVAL, std::string(name) + ": negative stack size");
  const int nb = d->num_blocks;
  for (int i = 0; i < nb; ++i)
    if (d->block_sizes[i] < 1) throw QtxError(QTX_E_INVAL, std::string(name) + ": block size < 1");
  for (int i = 0; i < nb; ++i) {
    for (int j = std::max(0, i - 1); j <= std::min(nb - 1, i + 1); ++j) {
      int k = bidx(i, j);
      int64_t rows = d->block_sizes[i], cols = d->block_sizes[j];
      bool has_index = d->block_index && d->block_index[k];
      if (d->block_offset[k] >= 0 && d->block_nnz[k] > 0) {
        if (!has_index && d->block_nnz[k] != rows * cols)
          throw QtxError(QTX_E_INVAL, std::string(name) + ": dense block (" + std::to_string(i) + "," +
                                          std::to_string(j) + ") needs rows*cols entries");
        if (d->block_nnz[k] > rows * cols)
          throw QtxError(QTX_E_INVAL, std::string(name) + ": block has more entries than rows*cols");
        if (d->block_offset[k] + d->block_nnz[k] > d->stack_stride)
          throw QtxError(QTX_E_INVAL, std::string(name) + ": block slice beyond the data row");
      }
    }
  }
}

void check_same_blocks(const qtx_btd_desc* a, const qtx_btd_desc* b, const char* name) {
  if (a->num_blocks != b->num_blocks || a->stack_size != b->stack_size)
    throw QtxError(QTX_E_INVAL, std::string(name) + ": block count or stack size differs from the system matrix");
  for (int i = 0; i < a->num_blocks; ++i)
    if (a->block_sizes[i] != b->block_sizes[i])
      throw QtxError(QTX_E_INVAL, std::string(name) + ": block sizes differ from the system matrix");
}

struct Workspace {
  cudaStream_t s;
  int64_t ne;           // energies in the current batch slice
  int bmax;
  cplx* zero = nullptr;  // bmax^2 zeros (broadcast view)
};

// Read view of block (i, j) for energies [e0, e0 + ne); sparse blocks are
// gathered into `scratch` (ne * bmax^2 complex).
MatView in_block(const Btd& m, int i, int j, int64_t e0, int64_t ne, cplx* scratch, const Workspace& ws) {
  int k = bidx(i, j);
  int rows = m.size(i), cols = m.size(j);
  if (m.empty(k)) return MatView{ws.zero, cols, 0};
  cplx* base = m.data + e0 * m.d->stack_stride + m.off(k);
  if (m.dense(k)) return MatView{base, cols, m.d->stack_stride};
  MutView out{scratch, cols, (int64_t)rows * cols};
  launch_block_gather(rows, cols, ne, base, m.d->stack_stride, m.nnz(k), m.index(k), out, ws.s);
  return out;
}

// Store x (rows x cols of block (i, j), or its source for modes 1/2) into block (i, j).
void out_block(const Btd& m, int i, int j, int64_t e0, int64_t ne, MatView x, int mode, const Workspace& ws) {
  if (!m.data) return;
  int k = bidx(i, j);
  if (m.empty(k)) return;
  cplx* base = m.data + e0 * m.d->stack_stride + m.off(k);
  launch_block_scatter(m.size(i), m.size(j), ne, x, mode, base, m.d->stack_stride, m.nnz(k), m.index(k), ws.s);
}

// OBC block view (contiguous (stack, b, b)), or null view
MatView obc_view(const void* const* arr, int i, int b, int64_t e0) {
  if (!arr || !arr[i]) return MatView{};
  const cplx* p = reinterpret_cast<const cplx*>(arr[i]);
  return MatView{p + e0 * (int64_t)b * b, b, (int64_t)b * b};
}

void gemm(int m, int n, int k, int64_t batch, cplx alpha, MatView a, int op_a, MatView b, int op_b, MutView d,
          cudaStream_t s, MatView c = MatView{}, cplx beta = ZERO, MatView c2 = MatView{}, cplx gamma = ZERO,
          const int* active = nullptr, const cplx* diag_shift = nullptr, int precision = QTX_PREC_FP64) {
  GemmCall g;
  g.m = m; g.n = n; g.k = k; g.batch = batch;
  g.a = a; g.op_a = op_a; g.b = b; g.op_b = op_b;
  g.c = c; g.beta = beta; g.c2 = c2; g.gamma = gamma;
  g.d = d; g.alpha = alpha; g.active = active; g.diag_shift = diag_shift;
  TimedScope ts(0, 8.0 * m * n * (double)k * batch, s);
  if (precision == QTX_PREC_MIXED && mixed_supported(g)) launch_zgemm_mixed(g, s);
  else launch_zgemm(g, s);
}

// Block inverse with timing (8 n^3 algorithmic flops per matrix: getrf + getri).
void zinv(int n, int64_t batch, MatView a, MutView x, int* info, const int* active, cudaStream_t s) {
  TimedScope ts(1, 8.0 * n * (double)n * n * batch, s);
  launch_zinv(n, batch, a, x, info, active, s);
}

std::vector<int64_t> batch_offsets(int64_t num, int64_t max_batch) {
  // get_batches: num // min(max_batch, num) near-equal sections, larger first
  std::vector<int64_t> offs{0};
  if (num <= 0) return offs;
  int64_t mb = std::max<int64_t>(1, max_batch);
  int64_t nsec = num / std::min(mb, num);
  int64_t base = num / nsec, rem = num % nsec;
  for (int64_t q = 0; q < nsec; ++q) offs.push_back(offs.back() + base + (q < rem ? 1 : 0));
  return offs;
}

// Per-batch dense state: one (ne, b_i, b_i) slot per diagonal block.  Every
// slot (and every temporary) has the same per-energy stride bmax^2, so slot
// and temporary buffers can trade places (pointer swaps) whatever the block sizes.
struct BlockStack {
  std::vector<cplx*> ptr;
  std::vector<int> size;
  int64_t ne = 0;
  int64_t slot = 0;  // elements per energy of every slot (bmax^2)
  MutView view(int i) const { return MutView{ptr[i], size[i], slot}; }
};

size_t stack_elems(const std::vector<int>& sizes, int64_t ne) {
  int bmax = *std::max_element(sizes.begin(), sizes.end());
  return (size_t)bmax * bmax * ne * sizes.size();
}

BlockStack carve(cplx*& cursor, const std::vector<int>& sizes, int64_t ne, int bmax) {
  BlockStack st;
  st.ne = ne;
  st.size = sizes;
  st.slot = (int64_t)bmax * bmax;
  for (size_t q = 0; q < sizes.size(); ++q) {
    st.ptr.push_back(cursor);
    cursor += (size_t)st.slot * ne;
  }
  return st;
}

// Status words of a call, read through a kernel store into the context's
// mapped page-locked words (no copy engine: a status read must not queue
// behind a caller's large download running on another stream).
struct StatusRead {
  int first;  // 1 + index of the first nonzero entry, 0 if none
  int value;  // that entry
  int head;   // entry 0
};
StatusRead read_status(qtx_ctx* ctx, const int* d, int64_t n, cudaStream_t s) {
  launch_flag_reduce(d, n, ctx->d_pinned, s);
  QTX_CUDA_TRY(cudaStreamSynchronize(s));
  volatile int* h = ctx->h_pinned;
  return StatusRead{h[0], h[1], h[2]};
}

void read_info_or_throw(qtx_ctx* ctx, const int* d_info, int64_t n, cudaStream_t s, const char* what) {
  const StatusRead r = read_status(ctx, d_info, n, s);
  if (r.first)
    throw QtxError(QTX_E_SINGULAR, std::string(what) + ": exactly singular diagonal block (stack entry " +
                                       std::to_string(r.first - 1) + ", pivot " + std::to_string(r.value) + ")");
}

// ---------------------------------------------------------------------------
// selected_inv  (src/qttools/greens_function_solver/rgf.py:25-113)
// ---------------------------------------------------------------------------
void selected_inv_impl(qtx_ctx* ctx, const Btd& a, const void* const* obc_r, const Btd& out, int64_t max_batch,
                       int precision, cudaStream_t s) {
  const int nb = a.nb();
  std::vector<int> sizes(a.d->block_sizes, a.d->block_sizes + nb);
  const int bmax = *std::max_element(sizes.begin(), sizes.end());
  const int64_t NE = a.d->stack_size;
  auto offs = batch_offsets(NE, max_batch);
  int64_t ne_max = 0;
  for (size_t q = 0; q + 1 < offs.size(); ++q) ne_max = std::max(ne_max, offs[q + 1] - offs[q]);
  if (ne_max == 0) return;

  const size_t tmp = (size_t)bmax * bmax * ne_max;
  const size_t total = stack_elems(sizes, ne_max) + 7 * tmp + (size_t)bmax * bmax;
  DevBuf buf(total * sizeof(cplx) + sizeof(int) * ne_max * nb, s);
  cplx* cur = buf.as<cplx>();
  BlockStack x = carve(cur, sizes, ne_max, bmax);
  cplx* T[7];
  for (int q = 0; q < 7; ++q) { T[q] = cur; cur += tmp; }
  Workspace ws{s, ne_max, bmax, cur};
  launch_fill_int(reinterpret_cast<int*>(ws.zero), (int64_t)4 * bmax * bmax, 0, s);
  cur += (size_t)bmax * bmax;
  int* info = reinterpret_cast<int*>(cur);
  launch_fill_int(info, ne_max * nb, 0, s);

  for (size_t q = 0; q + 1 < offs.size(); ++q) {
    const int64_t e0 = offs[q], ne = offs[q + 1] - offs[q];
    auto tv = [&](int idx, int ld) { return MutView{T[idx], ld, (int64_t)bmax * bmax}; };
    // x_0 = inv(A_00 - Sigma_0)
    {
      const int b0 = sizes[0];
      MatView a00 = in_block(a, 0, 0, e0, ne, T[5], ws);
      MatView o = obc_view(obc_r, 0, b0, e0);
      if (o.ptr) {
        launch_axpby(b0, b0, ne, ONE, a00, MONE, o, tv(0, b0), s);
        zinv(b0, ne, tv(0, b0), x.view(0), info, nullptr, s);
      } else {
        zinv(b0, ne, a00, x.view(0), info, nullptr, s);
      }
    }
    // forward: x_j = inv(A_jj - Sigma_j - A_ji x_i A_ij)
    for (int i = 0; i + 1 < nb; ++i) {
      const int j = i + 1, bi = sizes[i], bj = sizes[j];
      MatView a_ji = in_block(a, j, i, e0, ne, T[4], ws);
      MatView a_ij = in_block(a, i, j, e0, ne, T[5], ws);
      MatView a_jj = in_block(a, j, j, e0, ne, T[6], ws);
      gemm(bj, bi, bi, ne, ONE, a_ji, OP_N, x.view(i), OP_N, tv(0, bi), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
           precision);
      MatView o = obc_view(obc_r, j, bj, e0);
      gemm(bj, bj, bi, ne, MONE, tv(0, bi), OP_N, a_ij, OP_N, tv(1, bj), s, a_jj, ONE, o, MONE, nullptr, nullptr,
           precision);
      zinv(bj, ne, tv(1, bj), x.view(j), info + (int64_t)j * ne_max, nullptr, s);
    }
    out_block(out, nb - 1, nb - 1, e0, ne, x.view(nb - 1), 0, ws);
    // backward
    for (int i = nb - 2; i >= 0; --i) {
      const int j = i + 1, bi = sizes[i], bj = sizes[j];
      MatView a_ji = in_block(a, j, i, e0, ne, T[5], ws);
      MatView a_ij = in_block(a, i, j, e0, ne, T[6], ws);
      // X_ji = -(X_jj A_ji) x_i
      gemm(bj, bi, bj, ne, ONE, x.view(j), OP_N, a_ji, OP_N, tv(0, bi), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
           precision);
      gemm(bj, bi, bi, ne, MONE, tv(0, bi), OP_N, x.view(i), OP_N, tv(1, bi), s, {}, ZERO, {}, ZERO, nullptr,
           nullptr, precision);
      out_block(out, j, i, e0, ne, tv(1, bi), 0, ws);
      // X_ij = -(x_i A_ij) X_jj
      gemm(bi, bj, bi, ne, ONE, x.view(i), OP_N, a_ij, OP_N, tv(2, bj), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
           precision);
      gemm(bi, bj, bj, ne, MONE, tv(2, bj), OP_N, x.view(j), OP_N, tv(3, bj), s, {}, ZERO, {}, ZERO, nullptr,
           nullptr, precision);
      out_block(out, i, j, e0, ne, tv(3, bj), 0, ws);
      // X_ii = x_i - (x_i A_ij) X_ji
      gemm(bi, bi, bj, ne, MONE, tv(2, bj), OP_N, tv(1, bi), OP_N, tv(4, bi), s, x.view(i), ONE, {}, ZERO, nullptr,
           nullptr, precision);
      std::swap(x.ptr[i], T[4]);
      out_block(out, i, i, e0, ne, x.view(i), 0, ws);
    }
  }
  read_info_or_throw(ctx, info, ne_max * nb, s, "selected_inv");
  if (precision == QTX_PREC_MIXED) mixed_check_error(s);
}

// ---------------------------------------------------------------------------
// selected_solve  (src/qttools/greens_function_solver/rgf.py:115-414)
// ---------------------------------------------------------------------------
struct SolveArgs {
  Btd a, sl, sg, xl, xg, xr;
  const qtx_obc* obc = nullptr;
  cplx* current = nullptr;
  unsigned flags = 0;
  int64_t max_batch = 100;
  int precision = QTX_PREC_FP64;
};

// Per block k of a Sigma operand: 1 if block k holds a nonzero entry anywhere
// in the stack (one pass over the operand's data and one small read-back).
std::vector<char> sigma_nonzero_blocks(const Btd& m, cudaStream_t s) {
  const int nb = m.nb(), nk = 3 * nb - 2;
  std::vector<char> out(nk, 0);
  if (!m.data || m.d->stack_size <= 0) return out;
  std::vector<int64_t> slices(2 * (size_t)nk, -1);
  for (int i = 0; i < nb; ++i)
    for (int j = std::max(0, i - 1); j <= std::min(nb - 1, i + 1); ++j) {
      const int k = bidx(i, j);
      slices[2 * k] = m.empty(k) ? -1 : m.off(k);
      slices[2 * k + 1] = m.empty(k) ? 0 : m.nnz(k);
    }
  DevBuf buf(sizeof(int64_t) * slices.size() + sizeof(int) * nk, s);
  int64_t* d_slices = buf.as<int64_t>();
  int* d_flags = reinterpret_cast<int*>(d_slices + slices.size());
  QTX_CUDA_TRY(cudaMemcpyAsync(d_slices, slices.data(), sizeof(int64_t) * slices.size(), cudaMemcpyHostToDevice, s));
  launch_fill_int(d_flags, nk, 0, s);
  for (int k0 = 0; k0 < nk; k0 += 65535)
    launch_block_nonzero(std::min(nk - k0, 65535), d_slices + 2 * k0, m.data, m.d->stack_stride, m.d->stack_size,
                         d_flags + k0, s);
  std::vector<int> h(nk);
  QTX_CUDA_TRY(cudaMemcpyAsync(h.data(), d_flags, sizeof(int) * nk, cudaMemcpyDeviceToHost, s));
  QTX_CUDA_TRY(cudaStreamSynchronize(s));
  for (int k = 0; k < nk; ++k) out[k] = h[k] != 0;
  return out;
}

void selected_solve_impl(qtx_ctx* ctx, const SolveArgs& A, cudaStream_t s) {
  const Btd& a = A.a;
  const int nb = a.nb();
  std::vector<int> sizes(a.d->block_sizes, a.d->block_sizes + nb);
  const int bmax = *std::max_element(sizes.begin(), sizes.end());
  const int64_t NE = a.d->stack_size;
  const bool want_r = (A.flags & QTX_FLAG_RETURN_RETARDED) != 0;
  const bool want_r_off = (A.flags & QTX_FLAG_RETARDED_OFFDIAG) != 0;
  const bool want_cur = (A.flags & QTX_FLAG_RETURN_CURRENT) != 0 && A.current != nullptr;
  const bool symmetric = (A.flags & QTX_FLAG_SYMMETRIC_OUT) != 0;
  const int prec = A.precision;
  auto offs = batch_offsets(NE, A.max_batch);
  int64_t ne_max = 0;
  for (size_t q = 0; q + 1 < offs.size(); ++q) ne_max = std::max(ne_max, offs[q + 1] - offs[q]);
  if (ne_max == 0) return;

  const int NT = 12;
  const size_t tmp = (size_t)bmax * bmax * ne_max;
  std::vector<int> cur_sizes(sizes.begin() + 1, sizes.end());
  size_t total = 3 * stack_elems(sizes, ne_max) + NT * tmp + (size_t)bmax * bmax;
  if (want_cur) total += 2 * (size_t)bmax * bmax * ne_max * cur_sizes.size();
  DevBuf buf(total * sizeof(cplx) + sizeof(int) * ne_max * nb, s);
  cplx* cur = buf.as<cplx>();
  BlockStack xr = carve(cur, sizes, ne_max, bmax);
  BlockStack xl = carve(cur, sizes, ne_max, bmax);
  BlockStack xg = carve(cur, sizes, ne_max, bmax);
  BlockStack stl, stg;  // Sigma-tilde per interface (for the layer current)
  if (want_cur) {
    stl = carve(cur, cur_sizes, ne_max, bmax);
    stg = carve(cur, cur_sizes, ne_max, bmax);
  }
  cplx* T[NT];
  for (int q = 0; q < NT; ++q) { T[q] = cur; cur += tmp; }
  Workspace ws{s, ne_max, bmax, cur};
  launch_fill_int(reinterpret_cast<int*>(ws.zero), (int64_t)4 * bmax * bmax, 0, s);
  cur += (size_t)bmax * bmax;
  int* info = reinterpret_cast<int*>(cur);
  launch_fill_int(info, ne_max * nb, 0, s);

  const void* const* obc_r = A.obc ? A.obc->retarded : nullptr;
  const void* const* obc_l = A.obc ? A.obc->lesser : nullptr;
  const void* const* obc_g = A.obc ? A.obc->greater : nullptr;

  // Which blocks of Sigma^< and Sigma^> hold a nonzero entry anywhere in the
  // stack.  ElectronSolver passes interior self-energies that are zero in the
  // ballistic case (only the OBC blocks inject); every product with a zero
  // block is then skipped, and the forward step of both components shares
  // W = x_j A_ji (X_j = W X_i W^H when nothing is injected at block j).
  const std::vector<char> nz_l = sigma_nonzero_blocks(A.sl, s), nz_g = sigma_nonzero_blocks(A.sg, s);
  auto nz = [&](int comp, int i, int j) { return (comp == 0 ? nz_l : nz_g)[bidx(i, j)] != 0; };

  for (size_t q = 0; q + 1 < offs.size(); ++q) {
    const int64_t e0 = offs[q], ne = offs[q + 1] - offs[q];
    auto tv = [&](int idx, int ld) { return MutView{T[idx], ld, (int64_t)bmax * bmax}; };
    // G0..G3 (T[8..11]) are gather scratch for sparse input blocks
    // ---- first block (rgf.py:207-231)
    {
      const int b0 = sizes[0];
      MatView a00 = in_block(a, 0, 0, e0, ne, T[8], ws);
      MatView o = obc_view(obc_r, 0, b0, e0);
      if (o.ptr) {
        launch_axpby(b0, b0, ne, ONE, a00, MONE, o, tv(0, b0), s);
        zinv(b0, ne, tv(0, b0), xr.view(0), info, nullptr, s);
      } else {
        zinv(b0, ne, a00, xr.view(0), info, nullptr, s);
      }
      for (int comp = 0; comp < 2; ++comp) {
        const Btd& S = comp == 0 ? A.sl : A.sg;
        const void* const* ob = comp == 0 ? obc_l : obc_g;
        BlockStack& X = comp == 0 ? xl : xg;
        MatView s00 = in_block(S, 0, 0, e0, ne, T[9], ws);
        MatView o2 = obc_view(ob, 0, b0, e0);
        MatView sv = s00;
        if (o2.ptr) {
          launch_axpby(b0, b0, ne, ONE, s00, ONE, o2, tv(1, b0), s);
          sv = tv(1, b0);
        }
        gemm(b0, b0, b0, ne, ONE, xr.view(0), OP_N, sv, OP_N, tv(2, b0), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
             prec);
        gemm(b0, b0, b0, ne, ONE, tv(2, b0), OP_N, xr.view(0), OP_C, X.view(0), s, {}, ZERO, {}, ZERO, nullptr,
             nullptr, prec);
      }
    }
    // ---- forward sweep (rgf.py:233-295)
    for (int i = 0; i + 1 < nb; ++i) {
      const int j = i + 1, bi = sizes[i], bj = sizes[j];
      MatView a_ji = in_block(a, j, i, e0, ne, T[8], ws);
      MatView a_ij = in_block(a, i, j, e0, ne, T[9], ws);
      {
        MatView a_jj = in_block(a, j, j, e0, ne, T[10], ws);
        // U = A_ji x_i ; M = A_jj - Sigma^R_j - U A_ij ; x_j = inv(M)
        gemm(bj, bi, bi, ne, ONE, a_ji, OP_N, xr.view(i), OP_N, tv(0, bi), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
             prec);
        gemm(bj, bj, bi, ne, MONE, tv(0, bi), OP_N, a_ij, OP_N, tv(1, bj), s, a_jj, ONE,
             obc_view(obc_r, j, bj, e0), MONE, nullptr, nullptr, prec);
        zinv(bj, ne, tv(1, bj), xr.view(j), info + (int64_t)j * ne_max, nullptr, s);
      }
      // W = x_j A_ji, shared by both components when neither injects at
      // (i, j) or (j, j): X_j = W X_i W^H (3 products for two components
      // instead of 8)
      bool shared_w = !want_cur;
      for (int comp = 0; comp < 2; ++comp)
        shared_w = shared_w && !nz(comp, i, j) && !nz(comp, j, j) && !obc_view(comp == 0 ? obc_l : obc_g, j, bj, e0).ptr;
      if (shared_w) {
        gemm(bj, bi, bj, ne, ONE, xr.view(j), OP_N, a_ji, OP_N, tv(2, bi), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
             prec);
        for (int comp = 0; comp < 2; ++comp) {
          BlockStack& X = comp == 0 ? xl : xg;
          gemm(bj, bi, bi, ne, ONE, tv(2, bi), OP_N, X.view(i), OP_N, tv(5, bi), s, {}, ZERO, {}, ZERO, nullptr,
               nullptr, prec);
          gemm(bj, bj, bi, ne, ONE, tv(5, bi), OP_N, tv(2, bi), OP_C, X.view(j), s, {}, ZERO, {}, ZERO, nullptr,
               nullptr, prec);
        }
        continue;
      }
      for (int comp = 0; comp < 2; ++comp) {
        const Btd& S = comp == 0 ? A.sl : A.sg;
        const void* const* ob = comp == 0 ? obc_l : obc_g;
        BlockStack& X = comp == 0 ? xl : xg;
        const bool inj_ij = nz(comp, i, j);
        MatView s_ij = inj_ij ? in_block(S, i, j, e0, ne, T[10], ws) : MatView{};
        MatView s_jj = nz(comp, j, j) ? in_block(S, j, j, e0, ne, T[11], ws) : MatView{};
        // W = U S_ij (zero when S_ij is)
        if (inj_ij)
          gemm(bj, bj, bi, ne, ONE, tv(0, bi), OP_N, s_ij, OP_N, tv(2, bj), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
               prec);
        // V = X_i A_ji^H
        gemm(bi, bj, bi, ne, ONE, X.view(i), OP_N, a_ji, OP_C, tv(3, bj), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
             prec);
        if (want_cur) {
          BlockStack& ST = comp == 0 ? stl : stg;
          // Sigma~ = A_ji V + W^H - W  (kept for the layer current)
          gemm(bj, bj, bi, ne, ONE, a_ji, OP_N, tv(3, bj), OP_N, ST.view(i), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
               prec);
          if (inj_ij) launch_skew_combine(bj, ne, ST.view(i), tv(2, bj), ST.view(i), s);
          launch_axpby(bj, bj, ne, ONE, ST.view(i), ONE, s_jj.ptr ? s_jj : MatView{ws.zero, bj, 0}, tv(4, bj), s);
          MatView o2 = obc_view(ob, j, bj, e0);
          if (o2.ptr) launch_axpby(bj, bj, ne, ONE, tv(4, bj), ONE, o2, tv(4, bj), s);
        } else {
          // Q = A_ji V + S_jj + Sigma^<_obc,j ; Q += W^H - W
          gemm(bj, bj, bi, ne, ONE, a_ji, OP_N, tv(3, bj), OP_N, tv(4, bj), s, s_jj, ONE, obc_view(ob, j, bj, e0),
               ONE, nullptr, nullptr, prec);
          if (inj_ij) launch_skew_combine(bj, ne, tv(4, bj), tv(2, bj), tv(4, bj), s);
        }
        // X_j = x_j Q x_j^H
        gemm(bj, bj, bj, ne, ONE, xr.view(j), OP_N, tv(4, bj), OP_N, tv(5, bj), s, {}, ZERO, {}, ZERO, nullptr,
             nullptr, prec);
        gemm(bj, bj, bj, ne, ONE, tv(5, bj), OP_N, xr.view(j), OP_C, X.view(j), s, {}, ZERO, {}, ZERO, nullptr,
             nullptr, prec);
      }
    }
    // ---- last diagonal blocks (rgf.py:297-305)
    {
      const int n = nb - 1;
      out_block(A.xl, n, n, e0, ne, xl.view(n), 1, ws);
      out_block(A.xg, n, n, e0, ne, xg.view(n), 1, ws);
      if (want_r) out_block(A.xr, n, n, e0, ne, xr.view(n), 0, ws);
    }
    // ---- backward sweep (rgf.py:307-404)
    for (int i = nb - 2; i >= 0; --i) {
      const int j = i + 1, bi = sizes[i], bj = sizes[j];
      MatView a_ij = in_block(a, i, j, e0, ne, T[8], ws);
      MatView a_ji = in_block(a, j, i, e0, ne, T[9], ws);
      // P1 = x_i A_ij (bi x bj), P2 = X_jj A_ji (bj x bi), P3 = P1 X_jj, P4 = P1 P2
      gemm(bi, bj, bi, ne, ONE, xr.view(i), OP_N, a_ij, OP_N, tv(0, bj), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
           prec);
      gemm(bj, bi, bj, ne, ONE, xr.view(j), OP_N, a_ji, OP_N, tv(1, bi), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
           prec);
      gemm(bi, bj, bj, ne, ONE, tv(0, bj), OP_N, xr.view(j), OP_N, tv(2, bj), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
           prec);
      gemm(bi, bi, bj, ne, ONE, tv(0, bj), OP_N, tv(1, bi), OP_N, tv(3, bi), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
           prec);
      if (want_r_off) {
        // X^R_ij = -P3 ; X^R_ji = -P2 x_i
        launch_axpby(bi, bj, ne, MONE, tv(2, bj), ZERO, {}, tv(4, bj), s);
        out_block(A.xr, i, j, e0, ne, tv(4, bj), 0, ws);
        gemm(bj, bi, bi, ne, MONE, tv(1, bi), OP_N, xr.view(i), OP_N, tv(4, bi), s, {}, ZERO, {}, ZERO, nullptr,
             nullptr, prec);
        out_block(A.xr, j, i, e0, ne, tv(4, bi), 0, ws);
      }
      for (int comp = 0; comp < 2; ++comp) {
        const Btd& S = comp == 0 ? A.sl : A.sg;
        const Btd& OUT = comp == 0 ? A.xl : A.xg;
        BlockStack& X = comp == 0 ? xl : xg;
        const bool inj_ij = nz(comp, i, j);
        MatView s_ij = inj_ij ? in_block(S, i, j, e0, ne, T[10], ws) : MatView{};
        // Y = x_i S_ij (zero when S_ij is)
        if (inj_ij)
          gemm(bi, bj, bi, ne, ONE, xr.view(i), OP_N, s_ij, OP_N, tv(4, bj), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
               prec);
        // t1 = P4 X_i - Y P3^H ; t1 -= t1^H
        gemm(bi, bi, bi, ne, ONE, tv(3, bi), OP_N, X.view(i), OP_N, tv(5, bi), s, {}, ZERO, {}, ZERO, nullptr,
             nullptr, prec);
        if (inj_ij)
          gemm(bi, bi, bj, ne, MONE, tv(4, bj), OP_N, tv(2, bj), OP_C, tv(5, bi), s, tv(5, bi), ONE, {}, ZERO,
               nullptr, nullptr, prec);
        launch_sub_herm_inplace(bi, ne, tv(5, bi), s);
        // t2 = P1 X_j
        gemm(bi, bj, bj, ne, ONE, tv(0, bj), OP_N, X.view(j), OP_N, tv(6, bj), s, {}, ZERO, {}, ZERO, nullptr,
             nullptr, prec);
        // X_ij = Y X_jj^H - t2 - X_i P2^H
        if (inj_ij) {
          gemm(bi, bj, bj, ne, ONE, tv(4, bj), OP_N, xr.view(j), OP_C, tv(7, bj), s, tv(6, bj), MONE, {}, ZERO,
               nullptr, nullptr, prec);
          gemm(bi, bj, bi, ne, MONE, X.view(i), OP_N, tv(1, bi), OP_C, tv(7, bj), s, tv(7, bj), ONE, {}, ZERO,
               nullptr, nullptr, prec);
        } else {
          gemm(bi, bj, bi, ne, MONE, X.view(i), OP_N, tv(1, bi), OP_C, tv(7, bj), s, tv(6, bj), MONE, {}, ZERO,
               nullptr, nullptr, prec);
        }
        out_block(OUT, i, j, e0, ne, tv(7, bj), 0, ws);
        if (!symmetric) out_block(OUT, j, i, e0, ne, tv(7, bj), 2, ws);
        // X_i += t2 P1^H + t1
        gemm(bi, bi, bj, ne, ONE, tv(6, bj), OP_N, tv(0, bj), OP_C, X.view(i), s, X.view(i), ONE, tv(5, bi), ONE,
             nullptr, nullptr, prec);
        out_block(OUT, i, i, e0, ne, X.view(i), 1, ws);
      }
      if (want_cur) {
        // current_i = Tr[Sigma~^>_i X^<_j - X^>_j Sigma~^<_i]
        cplx* cur_out = T[11];
        launch_trace_product(bj, bj, ne, stg.view(i), xl.view(j), ONE, reinterpret_cast<cplx*>(cur_out), false, s);
        launch_trace_product(bj, bj, ne, xg.view(j), stl.view(i), MONE, reinterpret_cast<cplx*>(cur_out), true, s);
        // scatter into current[(e0 + e) * (nb - 1) + i]
        launch_axpby(1, 1, ne, ONE, MatView{cur_out, 1, 1}, ZERO, {}, MutView{A.current + e0 * (nb - 1) + i, 1, nb - 1},
                     s);
      }
      // x_i <- x_i + P4 x_i  (full G^R_ii)
      gemm(bi, bi, bi, ne, ONE, tv(3, bi), OP_N, xr.view(i), OP_N, tv(4, bi), s, xr.view(i), ONE, {}, ZERO, nullptr,
           nullptr, prec);
      std::swap(xr.ptr[i], T[4]);
      if (want_r) out_block(A.xr, i, i, e0, ne, xr.view(i), 0, ws);
    }
  }
  read_info_or_throw(ctx, info, ne_max * nb, s, "selected_solve");
  if (prec == QTX_PREC_MIXED) mixed_check_error(s);
}

// ---------------------------------------------------------------------------
// Sancho-Rubio (src/qttools/boundary_conditions/obc/sancho_rubio.py:33-86)
// ---------------------------------------------------------------------------
// Returns true when every entry converged.
bool sancho_rubio_impl(qtx_ctx* ctx, int n, int64_t batch, MatView a_ii, MatView a_ij, MatView a_ji, double tol,
                       int max_iter, MutView x, int* iterations, cudaStream_t s) {
  const size_t mat = (size_t)n * n * batch;
  DevBuf buf(sizeof(cplx) * 9 * mat + sizeof(int) * (3 * batch + 2), s);
  cplx* p = buf.as<cplx>();
  auto slot = [&](int q) { return MutView{p + q * mat, n, (int64_t)n * n}; };
  MutView eps = slot(0), eps_s = slot(1), alpha = slot(2), beta = slot(3), inv = slot(4), t0 = slot(5),
          t1 = slot(6), t2 = slot(7), t3 = slot(8);
  int* active = reinterpret_cast<int*>(p + 9 * mat);
  int* its = active + batch;
  int* num_active = its + batch;
  int* info = num_active + 2;  // zero pivots of the decimation inverses (sticky over the iterations)
  launch_fill_int(info, batch, 0, s);
  launch_axpby(n, n, batch, ONE, a_ii, ZERO, {}, eps, s);
  launch_axpby(n, n, batch, ONE, a_ii, ZERO, {}, eps_s, s);
  launch_axpby(n, n, batch, ONE, a_ji, ZERO, {}, alpha, s);
  launch_axpby(n, n, batch, ONE, a_ij, ZERO, {}, beta, s);
  launch_fill_int(active, batch, 1, s);
  launch_fill_int(its, batch, 0, s);
  bool converged = false;
  for (int it = 0; it < max_iter; ++it) {
    zinv(n, batch, eps, inv, info, active, s);
    gemm(n, n, n, batch, ONE, alpha, OP_N, inv, OP_N, t0, s, {}, ZERO, {}, ZERO, active);   // a inv
    gemm(n, n, n, batch, ONE, beta, OP_N, inv, OP_N, t1, s, {}, ZERO, {}, ZERO, active);    // b inv
    gemm(n, n, n, batch, ONE, t0, OP_N, beta, OP_N, t2, s, {}, ZERO, {}, ZERO, active);     // a inv b
    launch_axpby(n, n, batch, ONE, eps_s, MONE, t2, eps_s, s, active);                      // eps_s -= a inv b
    // eps = eps - a inv b - b inv a
    gemm(n, n, n, batch, MONE, t1, OP_N, alpha, OP_N, eps, s, eps, ONE, t2, MONE, active);
    gemm(n, n, n, batch, ONE, t0, OP_N, alpha, OP_N, t3, s, {}, ZERO, {}, ZERO, active);    // a inv a
    gemm(n, n, n, batch, ONE, t1, OP_N, beta, OP_N, t2, s, {}, ZERO, {}, ZERO, active);     // b inv b
    std::swap(alpha.ptr, t3.ptr);
    std::swap(beta.ptr, t2.ptr);
    launch_fill_int(num_active, 1, 0, s);
    launch_sr_norm_update(n, batch, alpha, beta, tol, active, its, num_active, s);
    if (read_status(ctx, num_active, 1, s).head == 0) {
      converged = true;
      break;
    }
  }
  zinv(n, batch, eps_s, x, info, nullptr, s);
  if (iterations) launch_copy_int(iterations, 1, its, 1, batch, s);
  read_info_or_throw(ctx, info, batch, s, "sancho_rubio (decimation block)");
  return converged;
}

// ---------------------------------------------------------------------------
// Generator-form transport solve (ElectronSolver.solve for a device whose leads
// repeat its end cells; interior scattering self-energies are zero)
// ---------------------------------------------------------------------------
// Work space of one energy batch: couplings, the three block stacks, temporaries,
// contact buffers and small per-energy arrays, carved from one allocation.
struct TransportWS {
  int nb = 0, b = 0;
  int64_t ne_max = 0;
  cplx* a_up = nullptr;  // A_i,i+1 = -H_i,i+1
  cplx* a_lo = nullptr;  // A_i+1,i = -H_i,i+1^H
  BlockStack xr, xl, xg;
  cplx* T[10];
  cplx* C[10];  // g_L, g_R, SigR_L, SigR_R, SigL_L, SigL_R, SigG_L, SigG_R, Gam_L, Gam_R
  cplx *shift = nullptr, *tr = nullptr, *cl = nullptr, *cr = nullptr;
  double *occ_l = nullptr, *occ_r = nullptr;
  int *info = nullptr, *its = nullptr;
};

size_t transport_ws_bytes(int nb, int b, int64_t ne_max) {
  const size_t bb = (size_t)b * b, tmp = bb * ne_max;
  const size_t cplx_elems = 2 * bb * std::max(nb - 1, 1) + 3 * (size_t)nb * tmp + 20 * tmp + 4 * ne_max;
  return sizeof(cplx) * cplx_elems + sizeof(double) * 2 * ne_max + sizeof(int) * (nb + 2) * ne_max + 256;
}

TransportWS carve_transport_ws(void* mem, int nb, int b, int64_t ne_max) {
  TransportWS w;
  w.nb = nb;
  w.b = b;
  w.ne_max = ne_max;
  const int64_t bb = (int64_t)b * b;
  const size_t tmp = (size_t)bb * ne_max;
  cplx* cur = reinterpret_cast<cplx*>(mem);
  w.a_up = cur;
  cur += bb * std::max(nb - 1, 1);
  w.a_lo = cur;
  cur += bb * std::max(nb - 1, 1);
  std::vector<int> sizes(nb, b);
  w.xr = carve(cur, sizes, ne_max, b);
  w.xl = carve(cur, sizes, ne_max, b);
  w.xg = carve(cur, sizes, ne_max, b);
  for (int q = 0; q < 10; ++q) { w.T[q] = cur; cur += tmp; }
  for (int q = 0; q < 10; ++q) { w.C[q] = cur; cur += tmp; }
  w.shift = cur; cur += ne_max;
  w.tr = cur; cur += ne_max;
  w.cl = cur; cur += ne_max;
  w.cr = cur; cur += ne_max;
  w.occ_l = reinterpret_cast<double*>(cur);
  w.occ_r = w.occ_l + ne_max;
  w.info = reinterpret_cast<int*>(w.occ_r + ne_max);
  w.its = w.info + nb * ne_max;
  return w;
}

// A_i,i+1 = -H_i,i+1 ; A_i+1,i = -H_i,i+1^H (energy independent)
void transport_couplings(const TransportWS& w, const cplx* h_upper, cudaStream_t s) {
  const int b = w.b;
  const int64_t bb = (int64_t)b * b;
  for (int i = 0; i + 1 < w.nb; ++i) {
    launch_axpby(b, b, 1, MONE, MatView{h_upper + i * bb, b, bb}, ZERO, {}, MutView{w.a_up + i * bb, b, bb}, s);
    launch_neg_herm(b, h_upper + i * bb, w.a_lo + i * bb, s);
  }
}

// Contacts of energies [e0, e0 + ne) (src/quatrex/electron/solver.py:305-386):
// Sancho-Rubio on both leads (host-synchronising convergence checks), then
// Sigma^R, Gamma, Sigma^<, Sigma^> and the (E + i eta) shifts, all into `w`.
bool transport_contacts(qtx_ctx* ctx, const TransportWS& w, const qtx_transport_problem& P,
                        const qtx_transport_outputs& O, int64_t e0, int64_t ne, cudaStream_t s) {
  const int nb = w.nb, b = w.b;
  const int64_t bb = (int64_t)b * b;
  const cplx* h_diag = reinterpret_cast<const cplx*>(P.h_diag);
  auto up = [&](int i) { return MatView{w.a_up + i * bb, b, 0}; };
  auto lo = [&](int i) { return MatView{w.a_lo + i * bb, b, 0}; };
  auto V = [&](cplx* p) { return MutView{p, b, bb}; };
  const double* en = P.energies + e0;
  launch_energy_shift(ne, en, P.eta, w.shift, s);
  // left: g_L = SR(A_00, A_01, A_10)
  launch_assemble_diag(b, ne, h_diag, en, P.eta, V(w.T[0]), s);
  bool okl = sancho_rubio_impl(ctx, b, ne, V(w.T[0]), up(0), lo(0), P.sr_tol, P.sr_max_iterations, V(w.C[0]), w.its,
                               s);
  if (O.sr_iterations) launch_copy_int(O.sr_iterations + 2 * e0, 2, w.its, 1, ne, s);
  // right: g_R = SR(A_nn, A_nm, A_mn)
  launch_assemble_diag(b, ne, h_diag + (int64_t)(nb - 1) * bb, en, P.eta, V(w.T[0]), s);
  bool okr = sancho_rubio_impl(ctx, b, ne, V(w.T[0]), lo(nb - 2), up(nb - 2), P.sr_tol, P.sr_max_iterations,
                               V(w.C[1]), w.its, s);
  if (O.sr_iterations) launch_copy_int(O.sr_iterations + 2 * e0 + 1, 2, w.its, 1, ne, s);
  // Sigma^R_L = A_10 g_L A_01 ; Sigma^R_R = A_mn g_R A_nm
  gemm(b, b, b, ne, ONE, lo(0), OP_N, V(w.C[0]), OP_N, V(w.T[1]), s);
  gemm(b, b, b, ne, ONE, V(w.T[1]), OP_N, up(0), OP_N, V(w.C[2]), s);
  gemm(b, b, b, ne, ONE, up(nb - 2), OP_N, V(w.C[1]), OP_N, V(w.T[1]), s);
  gemm(b, b, b, ne, ONE, V(w.T[1]), OP_N, lo(nb - 2), OP_N, V(w.C[3]), s);
  launch_fermi(ne, en, P.mu_left, P.kt, w.occ_l, s);
  launch_fermi(ne, en, P.mu_right, P.kt, w.occ_r, s);
  launch_obc_lesser_greater(b, ne, V(w.C[2]), w.occ_l, V(w.C[4]), V(w.C[6]), V(w.C[8]), s);
  launch_obc_lesser_greater(b, ne, V(w.C[3]), w.occ_r, V(w.C[5]), V(w.C[7]), V(w.C[9]), s);
  return okl && okr;
}

// Selected solve and observables of energies [e0, e0 + ne) once the contacts
// are in `w`.  Only kernel launches and device-to-device copies: it can be
// captured into a CUDA graph.  `w` is taken by value: the buffer swaps of the
// recursion permute this copy only, so every call starts from the same layout.
//
// Keldysh part.  The contacts are the only sources: Sigma^<_c = i f_c Gamma_c,
// Sigma^>_c = i (f_c - 1) Gamma_c with scalar occupations f_c, and the
// recursion for X = G^R Sigma G^A is linear in Sigma.  So it runs for the two
// contact sources instead of the two Keldysh components:
//   X_L: source i Gamma_L at block 0,  X_R: source i Gamma_R at block nb - 1,
//   G^< = f_L X_L + f_R X_R,  G^> = (f_L - 1) X_L + (f_R - 1) X_R
// (keldysh_mix).  X_R vanishes in the whole forward sweep (its source is the
// last block), and the forward X_L step is W X_L,i W^H with W = x_j A_ji, so
// a forward step takes 6 block products instead of 11 and a backward step 13
// instead of 15; the outputs are the same blocks.
void transport_sweep(TransportWS w, const qtx_transport_problem& P, const qtx_transport_outputs& O, int64_t e0,
                     int64_t ne, int prec, cudaStream_t s) {
  const int nb = w.nb, b = w.b;
  const int64_t bb = (int64_t)b * b;
  const int64_t ne_max = w.ne_max;
  const cplx* h_diag = reinterpret_cast<const cplx*>(P.h_diag);
  auto up = [&](int i) { return MatView{w.a_up + i * bb, b, 0}; };
  auto lo = [&](int i) { return MatView{w.a_lo + i * bb, b, 0}; };
  auto hd = [&](int i) { return MatView{h_diag + i * bb, b, 0}; };
  auto V = [&](cplx* p) { return MutView{p, b, bb}; };
  cplx** T = w.T;
  cplx** C = w.C;
  BlockStack& xr = w.xr;
  BlockStack& yl = w.xl;  // X_L
  BlockStack& yr = w.xg;  // X_R
  cplx* shift = w.shift;
  cplx* tr = w.tr;
  cplx* cl = w.cl;
  cplx* cr = w.cr;
  int* info = w.info;
  const double* fl = w.occ_l;
  const double* fr = w.occ_r;
  const cplx I1 = cmk(0, 1);
  auto obc_r = [&](int i) { return i == 0 ? MatView(V(C[2])) : (i == nb - 1 ? MatView(V(C[3])) : MatView{}); };
  auto tv = [&](int idx) { return V(T[idx]); };
  auto out_at = [&](void* base, int64_t blocks_per_e, int blk) {
    return MutView{reinterpret_cast<cplx*>(base) + (e0 * blocks_per_e + blk) * bb, b, blocks_per_e * bb};
  };
  auto out_ptr = [&](void* base, int64_t blocks_per_e, int blk) {
    return base ? reinterpret_cast<cplx*>(base) + (e0 * blocks_per_e + blk) * bb : nullptr;
  };
  // the G^< upper blocks are formed whenever an output needs them
  const bool uppers = O.gl_upper || O.gg_upper || O.layer_current;
  const cplx* h_up = reinterpret_cast<const cplx*>(P.h_upper);
  double* dos = O.dos ? O.dos + e0 * nb : nullptr;
  cplx* lcur = O.layer_current ? reinterpret_cast<cplx*>(O.layer_current) + e0 * (nb - 1) : nullptr;

  // ---- first block: x_0 = inv(A_00 - Sigma^R_L), X_L,0 = x_0 (i Gamma_L) x_0^H
  // M_0 = (E + i eta) I - H_00 - Sigma^R_L
  // (a K = 0 product: the epilogue alone forms -H_00 - Sigma^R_L + shift on the diagonal)
  gemm(b, b, 0, ne, ONE, tv(0), OP_N, tv(0), OP_N, tv(1), s, hd(0), MONE, obc_r(0), MONE, nullptr, shift);
  zinv(b, ne, tv(1), xr.view(0), info, nullptr, s);
  gemm(b, b, b, ne, I1, xr.view(0), OP_N, V(C[8]), OP_N, tv(2), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
  gemm(b, b, b, ne, ONE, tv(2), OP_N, xr.view(0), OP_C, yl.view(0), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
  // ---- forward sweep
  for (int i = 0; i + 1 < nb; ++i) {
    const int j = i + 1;
    gemm(b, b, b, ne, ONE, lo(i), OP_N, xr.view(i), OP_N, tv(0), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    // M = (E + i eta) I - H_jj - Sigma^R_j - U A_ij
    gemm(b, b, b, ne, MONE, tv(0), OP_N, up(i), OP_N, tv(1), s, hd(j), MONE, obc_r(j), MONE, nullptr, shift, prec);
    zinv(b, ne, tv(1), xr.view(j), info + (int64_t)j * ne_max, nullptr, s);
    // X_L,j = x_j A_ji X_L,i A_ji^H x_j^H = W X_L,i W^H with W = x_j A_ji
    // (no source past block 0)
    gemm(b, b, b, ne, ONE, xr.view(j), OP_N, lo(i), OP_N, tv(3), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    gemm(b, b, b, ne, ONE, tv(3), OP_N, yl.view(i), OP_N, tv(4), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    gemm(b, b, b, ne, ONE, tv(4), OP_N, tv(3), OP_C, yl.view(j), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
  }
  // ---- last block: X_R,n = x_n (i Gamma_R) x_n^H, outputs, corner chain start
  const int n = nb - 1;
  gemm(b, b, b, ne, I1, xr.view(n), OP_N, V(C[9]), OP_N, tv(2), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
  gemm(b, b, b, ne, ONE, tv(2), OP_N, xr.view(n), OP_C, yr.view(n), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
  launch_keldysh_combine(b, ne, yl.view(n), yr.view(n), fl, fr, 1.0, true, out_ptr(O.gl_diag, nb, n), nb * bb,
                         out_ptr(O.gg_diag, nb, n), nb * bb, s);
  if (O.gr_diag) launch_axpby(b, b, ne, ONE, xr.view(n), ZERO, {}, out_at(O.gr_diag, nb, n), s);
  launch_block_dos(b, ne, xr.view(n), dos, nb, n, s);
  launch_keldysh_density(b, ne, yl.view(n), yr.view(n), fl, fr, O.density ? O.density + e0 * nb : nullptr,
                         O.hole_density ? O.hole_density + e0 * nb : nullptr, nb, n, s);
  // contact current at the right contact uses the symmetrised G^<_nn, G^>_nn
  if (O.current_right) {
    launch_keldysh_combine(b, ne, yl.view(n), yr.view(n), fl, fr, 1.0, true, T[6], bb, T[7], bb, s);
    launch_trace_product(b, b, ne, V(C[7]), tv(6), ONE, cr, false, s);
    launch_trace_product(b, b, ne, tv(7), V(C[5]), MONE, cr, true, s);
    launch_axpby(1, 1, ne, ONE, MatView{cr, 1, 1}, ZERO, {}, MutView{reinterpret_cast<cplx*>(O.current_right) + e0, 1, 1},
                 s);
  }
  cplx* corner = T[8];
  cplx* corner2 = T[9];
  if (O.transmission) launch_axpby(b, b, ne, ONE, xr.view(n), ZERO, {}, V(corner), s);
  // ---- backward sweep
  for (int i = nb - 2; i >= 0; --i) {
    const int j = i + 1;
    gemm(b, b, b, ne, ONE, xr.view(i), OP_N, up(i), OP_N, tv(0), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    gemm(b, b, b, ne, ONE, xr.view(j), OP_N, lo(i), OP_N, tv(1), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    // G^R_ij = -P1 G_jj: only an output, so written there directly (and
    // skipped when it is not asked for)
    if (O.gr_upper)
      gemm(b, b, b, ne, MONE, tv(0), OP_N, xr.view(j), OP_N, out_at(O.gr_upper, nb - 1, i), s, {}, ZERO, {}, ZERO,
           nullptr, nullptr, prec);
    gemm(b, b, b, ne, ONE, tv(0), OP_N, tv(1), OP_N, tv(3), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    if (O.gr_lower)
      gemm(b, b, b, ne, MONE, tv(1), OP_N, xr.view(i), OP_N, out_at(O.gr_lower, nb - 1, i), s, {}, ZERO, {}, ZERO,
           nullptr, nullptr, prec);
    if (O.transmission) {
      // G_{i,N-1} = -(x_i A_ij) G_{j,N-1}
      gemm(b, b, b, ne, MONE, tv(0), OP_N, V(corner), OP_N, V(corner2), s, {}, ZERO, {}, ZERO, nullptr, nullptr,
           prec);
      std::swap(corner, corner2);
    }
    // X_L: t1 = P4 X_i - (P4 X_i)^H ; t2 = P1 X_j ; X_ij = -t2 - X_i P2^H ; X_i += t2 P1^H + t1
    gemm(b, b, b, ne, ONE, tv(3), OP_N, yl.view(i), OP_N, tv(5), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    launch_sub_herm_inplace(b, ne, tv(5), s);
    gemm(b, b, b, ne, ONE, tv(0), OP_N, yl.view(j), OP_N, tv(6), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    if (uppers)
      gemm(b, b, b, ne, MONE, yl.view(i), OP_N, tv(1), OP_C, tv(7), s, tv(6), MONE, {}, ZERO, nullptr, nullptr, prec);
    gemm(b, b, b, ne, ONE, tv(6), OP_N, tv(0), OP_C, yl.view(i), s, yl.view(i), ONE, tv(5), ONE, nullptr, nullptr,
         prec);
    // X_R (zero in the forward sweep): t2 = P1 X_j ; X_ij = -t2 ; X_i = t2 P1^H
    gemm(b, b, b, ne, ONE, tv(0), OP_N, yr.view(j), OP_N, tv(5), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    gemm(b, b, b, ne, ONE, tv(5), OP_N, tv(0), OP_C, yr.view(i), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    if (uppers)
      launch_keldysh_combine(b, ne, tv(7), tv(5), fl, fr, -1.0, false, out_ptr(O.gl_upper, nb - 1, i),
                             (nb - 1) * bb, out_ptr(O.gg_upper, nb - 1, i), (nb - 1) * bb, s);
    launch_layer_current(b, ne, tv(7), tv(5), fl, fr, -1.0, h_up + i * bb, lcur, nb - 1, i, s);
    launch_keldysh_combine(b, ne, yl.view(i), yr.view(i), fl, fr, 1.0, true, out_ptr(O.gl_diag, nb, i), nb * bb,
                           out_ptr(O.gg_diag, nb, i), nb * bb, s);
    launch_keldysh_density(b, ne, yl.view(i), yr.view(i), fl, fr, O.density ? O.density + e0 * nb : nullptr,
                           O.hole_density ? O.hole_density + e0 * nb : nullptr, nb, i, s);
    gemm(b, b, b, ne, ONE, tv(3), OP_N, xr.view(i), OP_N, tv(4), s, xr.view(i), ONE, {}, ZERO, nullptr, nullptr,
         prec);
    std::swap(xr.ptr[i], T[4]);
    if (O.gr_diag) launch_axpby(b, b, ne, ONE, xr.view(i), ZERO, {}, out_at(O.gr_diag, nb, i), s);
    launch_block_dos(b, ne, xr.view(i), dos, nb, i, s);
  }
  if (O.current_left) {
    launch_keldysh_combine(b, ne, yl.view(0), yr.view(0), fl, fr, 1.0, true, T[6], bb, T[7], bb, s);
    launch_trace_product(b, b, ne, V(C[6]), tv(6), ONE, cl, false, s);
    launch_trace_product(b, b, ne, tv(7), V(C[4]), MONE, cl, true, s);
    launch_axpby(1, 1, ne, ONE, MatView{cl, 1, 1}, ZERO, {}, MutView{reinterpret_cast<cplx*>(O.current_left) + e0, 1, 1},
                 s);
  }
  if (O.transmission) {
    // T = Tr[Gamma_L G_0N Gamma_R G_0N^H]
    gemm(b, b, b, ne, ONE, V(C[8]), OP_N, V(corner), OP_N, tv(0), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    gemm(b, b, b, ne, ONE, tv(0), OP_N, V(C[9]), OP_N, tv(1), s, {}, ZERO, {}, ZERO, nullptr, nullptr, prec);
    launch_trace_product_h(b, b, ne, tv(1), V(corner), tr, s);
    launch_real_part(ne, tr, O.transmission + e0, s);
  }
}

void transport_impl(qtx_ctx* ctx, const qtx_transport_problem& P, const qtx_transport_outputs& O, int prec,
                    cudaStream_t s, bool& all_converged) {
  const int nb = P.num_blocks, b = P.block_size;
  const int64_t NE = P.num_energies;
  auto offs = batch_offsets(NE, P.max_batch_size > 0 ? P.max_batch_size : NE);
  int64_t ne_max = 0;
  for (size_t q = 0; q + 1 < offs.size(); ++q) ne_max = std::max(ne_max, offs[q + 1] - offs[q]);
  if (ne_max == 0) return;
  DevBuf mem(transport_ws_bytes(nb, b, ne_max), s);
  TransportWS w = carve_transport_ws(mem.as<void>(), nb, b, ne_max);
  transport_couplings(w, reinterpret_cast<const cplx*>(P.h_upper), s);
  launch_fill_int(w.info, (int64_t)nb * ne_max, 0, s);
  for (size_t q = 0; q + 1 < offs.size(); ++q) {
    const int64_t e0 = offs[q], ne = offs[q + 1] - offs[q];
    all_converged = transport_contacts(ctx, w, P, O, e0, ne, s) && all_converged;
    transport_sweep(w, P, O, e0, ne, prec, s);
  }
  read_info_or_throw(ctx, w.info, (int64_t)nb * ne_max, s, "transport_solve");
  if (prec == QTX_PREC_MIXED) mixed_check_error(s);
}

// CUDA-graph form: the sweep of a single-batch call is captured once per
// (shapes, buffers, precision) and replayed; the contacts run eagerly each call
// (their convergence checks synchronise with the host).
void transport_graph_impl(qtx_ctx* ctx, const qtx_transport_problem& P, const qtx_transport_outputs& O, int prec,
                          cudaStream_t s, bool& all_converged) {
  const int nb = P.num_blocks, b = P.block_size;
  const int64_t ne = P.num_energies;
  if (ne == 0) return;
  GraphKey key;
  key.v = {(uintptr_t)P.h_diag, (uintptr_t)P.h_upper, (uintptr_t)P.energies, (uintptr_t)nb, (uintptr_t)b,
           (uintptr_t)ne, (uintptr_t)prec, (uintptr_t)O.gr_diag, (uintptr_t)O.gr_upper, (uintptr_t)O.gr_lower,
           (uintptr_t)O.gl_diag, (uintptr_t)O.gl_upper, (uintptr_t)O.gg_diag, (uintptr_t)O.gg_upper,
           (uintptr_t)O.density, (uintptr_t)O.hole_density, (uintptr_t)O.transmission, (uintptr_t)O.current_left,
           (uintptr_t)O.current_right, (uintptr_t)O.dos, (uintptr_t)O.layer_current};
  // scalars are baked into the captured launches: they are part of the key
  for (double v : {P.eta, P.mu_left, P.mu_right, P.kt, P.sr_tol}) {
    uint64_t bits;
    memcpy(&bits, &v, sizeof bits);
    key.v.push_back((uintptr_t)bits);
  }
  key.v.push_back((uintptr_t)P.sr_max_iterations);
  key.v.push_back((uintptr_t)P.max_batch_size);
  GraphEntry* g = ctx->graphs.find(key);
  if (!g) {
    g = ctx->graphs.insert(key, s);
    g->bytes = transport_ws_bytes(nb, b, ne);
    QTX_CUDA_TRY(cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming));
    g->mem = qtx_malloc_async(g->bytes, s);
    if (!g->mem) {
      ctx->graphs.erase(key, s);
      throw QtxError(QTX_E_NOMEM, "transport graph: work space allocation failed");
    }
    QTX_CUDA_TRY(cudaEventRecord(g->done, s));
  }
  TransportWS w = carve_transport_ws(g->mem, nb, b, ne);
  transport_couplings(w, reinterpret_cast<const cplx*>(P.h_upper), s);
  launch_fill_int(w.info, (int64_t)nb * ne, 0, s);
  all_converged = transport_contacts(ctx, w, P, O, 0, ne, s) && all_converged;
  if (!g->exec) {
    std::lock_guard<std::mutex> capture_lock(g_capture_mutex);
    const int64_t before = ctx->launches;
    ctx->capturing = true;
    if (!ctx->capture_stream) QTX_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->capture_stream, cudaStreamNonBlocking));
    cudaStream_t cs = ctx->capture_stream;
    QTX_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    try {
      transport_sweep(w, P, O, 0, ne, prec, cs);
    } catch (...) {
      cudaGraph_t dummy = nullptr;
      cudaStreamEndCapture(cs, &dummy);
      if (dummy) cudaGraphDestroy(dummy);
      ctx->capturing = false;
      throw;
    }
    cudaGraph_t graph = nullptr;
    QTX_CUDA_TRY(cudaStreamEndCapture(cs, &graph));
    ctx->capturing = false;
    cudaError_t e = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      g->exec = nullptr;
      throw QtxError(QTX_E_CUDA, std::string("transport graph instantiation: ") + cudaGetErrorString(e));
    }
    g->launches = ctx->launches - before;
    ctx->launches = before;
  }
  QTX_CUDA_TRY(cudaGraphLaunch(g->exec, s));
  QTX_CUDA_TRY(cudaEventRecord(g->done, s));
  ctx->launches += g->launches;
  ctx->graph_replays += 1;
  read_info_or_throw(ctx, w.info, (int64_t)nb * ne, s, "transport_solve");
  if (prec == QTX_PREC_MIXED) mixed_check_error(s);
}

// ---------------------------------------------------------------------------
// Grouped transport solve: every energy of several problems of one block size
// in one persistent launch (rgf_grouped.cu).
// ---------------------------------------------------------------------------
struct GroupedPlan {
  std::vector<GroupedProblem> problems;  // longest first
  std::vector<int> source;               // index of each in the caller's array
  int64_t items = 0;
  int max_nb = 0, b = 0;
};

GroupedPlan grouped_plan(int32_t count, const qtx_transport_problem* p, const qtx_transport_outputs* o) {
  GroupedPlan plan;
  plan.b = p[0].block_size;
  if (plan.b < 1 || plan.b > GROUPED_MAX_B)
    throw QtxError(QTX_E_UNSUPPORTED, "qtx_transport_solve_grouped: block size must be 1..64");
  std::vector<int> order(count);
  for (int q = 0; q < count; ++q) {
    const qtx_transport_problem& x = p[q];
    if (x.block_size != plan.b) throw QtxError(QTX_E_INVAL, "qtx_transport_solve_grouped: mixed block sizes");
    if (x.num_blocks < 2 || x.num_energies < 0 || !x.h_diag || !x.h_upper || (x.num_energies > 0 && !x.energies) ||
        x.kt <= 0 || x.sr_max_iterations < 1)
      throw QtxError(QTX_E_INVAL, "qtx_transport_solve_grouped: bad problem");
    order[q] = q;
  }
  // longest problems first: their pairs are handed out first
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return p[x].num_blocks > p[y].num_blocks; });
  for (int q : order) {
    const qtx_transport_problem& x = p[q];
    const qtx_transport_outputs& y = o[q];
    GroupedProblem g;
    g.nb = x.num_blocks;
    g.b = x.block_size;
    g.num_energies = x.num_energies;
    g.item0 = plan.items;
    g.h_diag = reinterpret_cast<const cplx*>(x.h_diag);
    g.h_upper = reinterpret_cast<const cplx*>(x.h_upper);
    g.energies = x.energies;
    g.eta = x.eta;
    g.mu_left = x.mu_left;
    g.mu_right = x.mu_right;
    g.kt = x.kt;
    g.sr_tol = x.sr_tol;
    g.sr_max_iterations = x.sr_max_iterations;
    g.gr_diag = reinterpret_cast<cplx*>(y.gr_diag);
    g.gr_upper = reinterpret_cast<cplx*>(y.gr_upper);
    g.gr_lower = reinterpret_cast<cplx*>(y.gr_lower);
    g.gl_diag = reinterpret_cast<cplx*>(y.gl_diag);
    g.gl_upper = reinterpret_cast<cplx*>(y.gl_upper);
    g.gg_diag = reinterpret_cast<cplx*>(y.gg_diag);
    g.gg_upper = reinterpret_cast<cplx*>(y.gg_upper);
    g.density = y.density;
    g.hole_density = y.hole_density;
    g.transmission = y.transmission;
    g.current_left = reinterpret_cast<cplx*>(y.current_left);
    g.current_right = reinterpret_cast<cplx*>(y.current_right);
    g.sr_iterations = y.sr_iterations;
    g.dos = y.dos;
    g.layer_current = reinterpret_cast<cplx*>(y.layer_current);
    plan.items += x.num_energies;
    plan.max_nb = std::max(plan.max_nb, x.num_blocks);
    if (x.num_energies > 0) {
      plan.problems.push_back(g);
      plan.source.push_back(q);
    }
  }
  return plan;
}

// descriptors | work counter and flags | per-CTA work spaces
size_t grouped_desc_bytes(const GroupedPlan& plan) {
  return (sizeof(GroupedProblem) * plan.problems.size() + 255) / 256 * 256;
}
size_t grouped_flag_bytes(const GroupedPlan& plan) {
  return (64 + sizeof(int) * (1 + plan.problems.size()) + 255) / 256 * 256;
}
size_t grouped_bytes(const GroupedPlan& plan, int grid) {
  return grouped_desc_bytes(plan) + grouped_flag_bytes(plan) +
         sizeof(cplx) * (size_t)grid * (size_t)grouped_ws_elems(plan.max_nb, plan.b);
}

// Returns the flags of the caller's problems (count entries; bit 0 a zero
// pivot, bit 1 a lead that did not converge).
std::vector<int> transport_grouped_impl(int32_t count, const qtx_transport_problem* p,
                                        const qtx_transport_outputs* o, cudaStream_t s) {
  GroupedPlan plan = grouped_plan(count, p, o);
  std::vector<int> out(count, 0);
  if (plan.items == 0) return out;
  const int grid = grouped_grid(plan.b, plan.items);
  DevBuf mem(grouped_bytes(plan, grid), s);
  char* base = mem.as<char>();
  const size_t desc = grouped_desc_bytes(plan);
  GroupedProblem* d_problems = reinterpret_cast<GroupedProblem*>(base);
  unsigned long long* counter = reinterpret_cast<unsigned long long*>(base + desc);
  int* flags = reinterpret_cast<int*>(base + desc + 64);
  cplx* ws = reinterpret_cast<cplx*>(base + desc + grouped_flag_bytes(plan));
  QTX_CUDA_TRY(cudaMemcpyAsync(d_problems, plan.problems.data(), sizeof(GroupedProblem) * plan.problems.size(),
                               cudaMemcpyHostToDevice, s));
  QTX_CUDA_TRY(cudaMemsetAsync(base + desc, 0, grouped_flag_bytes(plan), s));
  launch_transport_grouped(plan.b, d_problems, (int)plan.problems.size(), plan.items, counter, flags, ws,
                           grouped_ws_elems(plan.max_nb, plan.b), plan.max_nb, grid, s);
  std::vector<int> h_flags(1 + plan.problems.size());
  QTX_CUDA_TRY(cudaMemcpyAsync(h_flags.data(), flags, sizeof(int) * h_flags.size(), cudaMemcpyDeviceToHost, s));
  QTX_CUDA_TRY(cudaStreamSynchronize(s));
  for (size_t k = 0; k < plan.problems.size(); ++k) out[plan.source[k]] = h_flags[1 + k];
  return out;
}

// ---------------------------------------------------------------------------
// host-buffer streaming for qtx_selected_inv / qtx_selected_solve
// (QTX_FLAG_HOST_BUFFERS)
// ---------------------------------------------------------------------------
// The stack is processed in energy batches: the batch's rows of every array
// are copied into one of two device staging sets, solved on the caller's
// stream and copied back, so that the upload of batch q + 1 and the download
// of batch q - 1 overlap the solve of batch q.  The copies run on a copy
// thread through the context's ring of page-locked slots (host memcpy over a
// few threads, then DMA), because the caller's arrays are pageable: through
// the driver's own staging they ran at about 10 GB/s, and page-locking them
// for each call (cudaHostRegister) was slower still.  Device memory is
// bounded by two staging sets and the solver's own work space of one batch,
// whatever the stack size.
size_t desc_row_bytes(const qtx_btd_desc* d) { return sizeof(cplx) * (size_t)d->stack_stride; }

// One host array of the call: rows of `row_bytes`, `rows` of them.
struct HostArr {
  const char* h = nullptr;  // host base
  char* hw = nullptr;       // writable host base (outputs)
  size_t row_bytes = 0;
  bool in = false, out = false;
  char* dev[2] = {nullptr, nullptr};
};

// Energies per streamed batch: two staging sets plus the solver's work space
// (about (3 nb + 20) bmax^2 complex per energy) in 70 % of the free memory.
int64_t host_batch(int64_t max_batch, int64_t NE, size_t staging_per_energy, int nb, int bmax) {
  size_t free_b = 0, total_b = 0;
  QTX_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  const size_t ws = sizeof(cplx) * (size_t)(3 * nb + 20) * bmax * bmax;
  const size_t per = 2 * staging_per_energy + ws;
  int64_t ne = (int64_t)((double)free_b * 0.7 / (double)std::max<size_t>(per, 1));
  ne = std::max<int64_t>(1, std::min<int64_t>({ne, max_batch, NE}));
  return ne;
}

// Copies between the caller's pageable arrays and device memory through a
// PinRing: host memcpy into a slot (split over a few host threads), then an
// async DMA on `cs`; a slot is reused only after its previous DMA completed.
// Downloads keep up to kSlots - 1 DMAs in flight ahead of the host copies.
struct RingCopier {
  PinRing& R;
  cudaStream_t cs;
  int next = 0;
  struct Pending {
    int slot;
    char* host;
    size_t len;
  };
  std::deque<Pending> pending;

  static void memcpy_mt(char* dst, const char* src, size_t n) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>({8, (size_t)std::max(1u, hw / 2), n / (4u << 20) + 1});
    if (nt <= 1) {
      memcpy(dst, src, n);
      return;
    }
    std::vector<std::thread> th;
    const size_t part = (n + nt - 1) / nt;
    for (size_t t = 0; t < nt; ++t) {
      const size_t off = t * part;
      if (off >= n) break;
      const size_t len = std::min(part, n - off);
      th.emplace_back([=] { memcpy(dst + off, src + off, len); });
    }
    for (auto& x : th) x.join();
  }
  int take_slot() {
    const int sl = next;
    next = (next + 1) % PinRing::kSlots;
    // a pending download in this slot is copied out first
    while (!pending.empty() && std::any_of(pending.begin(), pending.end(), [&](const Pending& p) { return p.slot == sl; }))
      drain_one();
    QTX_CUDA_TRY(cudaEventSynchronize(R.ev[sl]));
    return sl;
  }
  void upload(char* dev, const char* host, size_t n) {
    for (size_t off = 0; off < n; off += PinRing::kSlotBytes) {
      const size_t len = std::min(PinRing::kSlotBytes, n - off);
      const int sl = take_slot();
      memcpy_mt(R.slot(sl), host + off, len);
      QTX_CUDA_TRY(cudaMemcpyAsync(dev + off, R.slot(sl), len, cudaMemcpyHostToDevice, cs));
      QTX_CUDA_TRY(cudaEventRecord(R.ev[sl], cs));
    }
  }
  void download(char* host, const char* dev, size_t n) {
    for (size_t off = 0; off < n; off += PinRing::kSlotBytes) {
      const size_t len = std::min(PinRing::kSlotBytes, n - off);
      if ((int)pending.size() >= PinRing::kSlots - 1) drain_one();
      const int sl = take_slot();
      QTX_CUDA_TRY(cudaMemcpyAsync(R.slot(sl), dev + off, len, cudaMemcpyDeviceToHost, cs));
      QTX_CUDA_TRY(cudaEventRecord(R.ev[sl], cs));
      pending.push_back({sl, host + off, len});
    }
  }
  void drain_one() {
    Pending p = pending.front();
    pending.pop_front();
    QTX_CUDA_TRY(cudaEventSynchronize(R.ev[p.slot]));
    memcpy_mt(p.host, R.slot(p.slot), p.len);
  }
  void drain_all() {
    while (!pending.empty()) drain_one();
  }
};

// One host thread running copy tasks in order (uploads and downloads of the
// streamed batches) while the calling thread runs the solver.
struct CopyWorker {
  std::mutex m;
  std::condition_variable cv;
  std::deque<std::function<void()>> tasks;
  bool stop = false;
  std::exception_ptr error;
  int64_t done = 0, posted = 0;
  std::thread th;
  CopyWorker() : th([this] { run(); }) {}
  ~CopyWorker() {
    {
      std::lock_guard<std::mutex> lk(m);
      stop = true;
    }
    cv.notify_all();
    th.join();
  }
  void run() {
    for (;;) {
      std::function<void()> f;
      {
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [&] { return stop || !tasks.empty(); });
        if (tasks.empty()) return;
        f = std::move(tasks.front());
        tasks.pop_front();
      }
      try {
        if (!error) f();
      } catch (...) {
        std::lock_guard<std::mutex> lk(m);
        if (!error) error = std::current_exception();
      }
      {
        std::lock_guard<std::mutex> lk(m);
        ++done;
      }
      cv.notify_all();
    }
  }
  int64_t post(std::function<void()> f) {
    std::lock_guard<std::mutex> lk(m);
    tasks.push_back(std::move(f));
    cv.notify_all();
    return ++posted;
  }
  // wait until task number `ticket` (1-based) has run; rethrows its failure
  void wait(int64_t ticket) {
    std::unique_lock<std::mutex> lk(m);
    cv.wait(lk, [&] { return done >= ticket; });
    if (error) std::rethrow_exception(error);
  }
};

// Streams `solve(e0, ne, set)` over the stack.  `arrs` are the per-energy
// arrays (inputs copied up, outputs copied down; outputs are also copied up so
// that entries the solver does not write keep their values).  With the
// context's PinRing, a copy thread uploads batch q + 1 and downloads batch
// q - 1 through page-locked slots while the solver runs batch q; without one
// (page-locked memory refused) the copies go straight from the pageable arrays.
template <typename F>
void stream_host_batches(qtx_ctx* ctx, std::vector<HostArr>& arrs, int64_t NE, int64_t ne_b, cudaStream_t s,
                         F&& solve) {
  size_t per_set = 0;
  for (auto& a : arrs) per_set += ((a.row_bytes * ne_b + 255) / 256) * 256;
  DevBuf staging(2 * per_set, s);
  for (int set = 0; set < 2; ++set) {
    char* cur = staging.as<char>() + set * per_set;
    for (auto& a : arrs) {
      a.dev[set] = cur;
      cur += ((a.row_bytes * ne_b + 255) / 256) * 256;
    }
  }
  if (!ctx->ring) ctx->ring = ring_take();
  bool use_ring = ctx->ring != nullptr;
  if (use_ring)
    for (auto e : ctx->ring->ev) use_ring = use_ring && e != nullptr;
  cudaStream_t cs = nullptr;
  QTX_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaEvent_t up[2] = {nullptr, nullptr}, solved = nullptr;
  auto cleanup = [&] {
    cudaStreamSynchronize(cs);
    for (auto& e : up)
      if (e) cudaEventDestroy(e);
    if (solved) cudaEventDestroy(solved);
    cudaStreamDestroy(cs);
  };
  const int64_t nbatch = (NE + ne_b - 1) / ne_b;
  try {
    QTX_CUDA_TRY(cudaEventCreateWithFlags(&up[0], cudaEventDisableTiming));
    QTX_CUDA_TRY(cudaEventCreateWithFlags(&up[1], cudaEventDisableTiming));
    QTX_CUDA_TRY(cudaEventCreateWithFlags(&solved, cudaEventDisableTiming));
    // the staging memory was allocated on s: the copy stream starts after it
    QTX_CUDA_TRY(cudaEventRecord(solved, s));
    QTX_CUDA_TRY(cudaStreamWaitEvent(cs, solved, 0));
    if (use_ring) {
      RingCopier rc{*ctx->ring, cs, 0, {}};
      CopyWorker w;
      auto upload = [&](int64_t e0, int64_t ne, int set) {
        return w.post([&, e0, ne, set] {
          for (auto& a : arrs)
            if (a.in || a.out) rc.upload(a.dev[set], (a.out ? a.hw : a.h) + e0 * a.row_bytes, ne * a.row_bytes);
          QTX_CUDA_TRY(cudaEventRecord(up[set], cs));
        });
      };
      auto download = [&](int64_t e0, int64_t ne, int set) {
        return w.post([&, e0, ne, set] {
          for (auto& a : arrs)
            if (a.out) rc.download(a.hw + e0 * a.row_bytes, a.dev[set], ne * a.row_bytes);
          rc.drain_all();
        });
      };
      int64_t t_cur = nbatch > 0 ? upload(0, std::min(ne_b, NE), 0) : 0, t_last = t_cur;
      for (int64_t q = 0; q < nbatch; ++q) {
        const int set = (int)(q & 1);
        const int64_t e0 = q * ne_b, ne = std::min(ne_b, NE - e0);
        // queued behind the download of batch q - 1, which last read set ^ 1
        int64_t t_next = 0;
        if (q + 1 < nbatch) t_next = upload(e0 + ne_b, std::min(ne_b, NE - e0 - ne_b), set ^ 1);
        w.wait(t_cur);
        QTX_CUDA_TRY(cudaStreamWaitEvent(s, up[set], 0));
        solve(e0, ne, set);  // ends with a synchronisation of s
        t_last = download(e0, ne, set);
        t_cur = t_next;
      }
      w.wait(t_last);
    } else {
      auto upload = [&](int64_t e0, int64_t ne, int set) {
        for (auto& a : arrs)
          if (a.in || a.out)
            QTX_CUDA_TRY(cudaMemcpyAsync(a.dev[set], (a.out ? a.hw : a.h) + e0 * a.row_bytes, ne * a.row_bytes,
                                         cudaMemcpyHostToDevice, cs));
        QTX_CUDA_TRY(cudaEventRecord(up[set], cs));
      };
      if (nbatch > 0) upload(0, std::min(ne_b, NE), 0);
      for (int64_t q = 0; q < nbatch; ++q) {
        const int set = (int)(q & 1);
        const int64_t e0 = q * ne_b, ne = std::min(ne_b, NE - e0);
        if (q + 1 < nbatch) upload(e0 + ne_b, std::min(ne_b, NE - e0 - ne_b), set ^ 1);
        QTX_CUDA_TRY(cudaStreamWaitEvent(s, up[set], 0));
        solve(e0, ne, set);  // ends with a synchronisation of s
        QTX_CUDA_TRY(cudaEventRecord(solved, s));
        QTX_CUDA_TRY(cudaStreamWaitEvent(cs, solved, 0));
        for (auto& a : arrs)
          if (a.out)
            QTX_CUDA_TRY(cudaMemcpyAsync(a.hw + e0 * a.row_bytes, a.dev[set], ne * a.row_bytes,
                                         cudaMemcpyDeviceToHost, cs));
      }
    }
    QTX_CUDA_TRY(cudaStreamSynchronize(cs));
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
  // staging is freed on s after everything queued on it
}

// qtx_btd_desc of one streamed batch: the same blocks, ne rows
qtx_btd_desc batch_desc(const qtx_btd_desc* d, int64_t ne) {
  qtx_btd_desc b = *d;
  b.stack_size = ne;
  return b;
}

// per-block OBC arrays (host pointers, (stack, b_i, b_i)) as streamed arrays
void add_obc_arrays(std::vector<HostArr>& arrs, const void* const* obc, const qtx_btd_desc* d,
                    std::vector<int>& which) {
  if (!obc) return;
  for (int i = 0; i < d->num_blocks; ++i) {
    if (!obc[i]) continue;
    HostArr a;
    a.h = reinterpret_cast<const char*>(obc[i]);
    a.row_bytes = sizeof(cplx) * (size_t)d->block_sizes[i] * d->block_sizes[i];
    a.in = true;
    which.push_back(i);
    arrs.push_back(a);
  }
}

template <typename F>
qtx_status guarded(qtx_ctx* ctx, F&& f) {
  if (!ctx) return QTX_E_INVAL;
  LaunchScope scope(ctx);
  try {
    QTX_CUDA_TRY(cudaSetDevice(ctx->device));
    f();
    ctx->last_error.clear();
    return QTX_OK;
  } catch (const QtxError& e) {
    ctx->last_error = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    ctx->last_error = e.what();
    return QTX_E_CUDA;
  }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* qtx_version(void) { return "qtx-rgf 0.1 (sm_100a)"; }

qtx_status qtx_ctx_create(int device, qtx_ctx** out) {
  if (!out) return QTX_E_INVAL;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return QTX_E_CUDA;
  }
  if (cudaSetDevice(device) != cudaSuccess) return QTX_E_CUDA;
  qtx_ctx* c = new qtx_ctx();
  c->device = device;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  c->h_pinned = pinned_take();
  if (!c->h_pinned) {
    delete c;
    return QTX_E_NOMEM;
  }
  if (cudaHostGetDevicePointer((void**)&c->d_pinned, c->h_pinned, 0) != cudaSuccess) {
    cudaGetLastError();
    pinned_give(c->h_pinned);
    delete c;
    return QTX_E_CUDA;
  }
  *out = c;
  return QTX_OK;
}

qtx_status qtx_ctx_destroy(qtx_ctx* ctx) {
  if (!ctx) return QTX_E_INVAL;
  cudaSetDevice(ctx->device);
  // Work already enqueued by this context keeps running; the graph work spaces
  // are freed in stream order after their last use, without a device-wide
  // synchronisation (other threads may be capturing graphs meanwhile).
  cudaStream_t rs = nullptr;
  if (cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    rs = ctx->capture_stream;
  }
  ctx->graphs.clear(rs);
  if (rs) {
    cudaStreamSynchronize(rs);
    if (rs != ctx->capture_stream) cudaStreamDestroy(rs);
  }
  if (ctx->capture_stream) cudaStreamDestroy(ctx->capture_stream);
  for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
  pinned_give(ctx->h_pinned);
  ring_give(ctx->ring);
  delete ctx;
  return QTX_OK;
}

const char* qtx_last_error(const qtx_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

qtx_status qtx_ctx_set_memory_limit(qtx_ctx* ctx, size_t bytes) {
  if (!ctx) return QTX_E_INVAL;
  ctx->mem_limit = bytes;
  return QTX_OK;
}

qtx_status qtx_ctx_trim(qtx_ctx* ctx) {
  return guarded(ctx, [&] {
    cudaMemPool_t pool;
    QTX_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
    std::lock_guard<std::mutex> capture_lock(g_capture_mutex);
    QTX_CUDA_TRY(cudaDeviceSynchronize());
    ctx->graphs.clear(nullptr);
    QTX_CUDA_TRY(cudaDeviceSynchronize());
    QTX_CUDA_TRY(cudaMemPoolTrimTo(pool, 0));
  });
}

int64_t qtx_launch_count(const qtx_ctx* ctx) { return ctx ? ctx->launches : -1; }

int64_t qtx_graph_replays(const qtx_ctx* ctx) { return ctx ? ctx->graph_replays : -1; }

size_t qtx_transport_footprint(int32_t num_blocks, int32_t block_size, int64_t energies_per_call, int32_t precision) {
  if (num_blocks < 2 || block_size < 1 || energies_per_call < 1) return 0;
  const size_t b = (size_t)block_size, ne = (size_t)energies_per_call;
  size_t bytes = transport_ws_bytes(num_blocks, block_size, energies_per_call);
  bytes += sizeof(cplx) * 9 * b * b * ne + sizeof(int) * (2 * ne + 2);  // Sancho-Rubio
  if (precision == QTX_PREC_MIXED)
    bytes += mixed_workspace_bytes(block_size, block_size, block_size, energies_per_call, energies_per_call);
  bytes += zinv_workspace_bytes(block_size, energies_per_call);
  return bytes + (4u << 20);  // allocator granularity
}

qtx_status qtx_ctx_release_graphs(qtx_ctx* ctx, qtx_stream stream) {
  return guarded(ctx, [&] { ctx->graphs.clear(static_cast<cudaStream_t>(stream)); });
}

qtx_status qtx_ctx_set_timing(qtx_ctx* ctx, int enable) {
  if (!ctx) return QTX_E_INVAL;
  cudaSetDevice(ctx->device);
  drain_timing(ctx);
  ctx->timing = enable != 0;
  for (int k = 0; k < 2; ++k) {
    ctx->acc_ms[k] = ctx->acc_flops[k] = 0;
    ctx->acc_launches[k] = 0;
  }
  return QTX_OK;
}

qtx_status qtx_ctx_timing_report(qtx_ctx* ctx, int32_t kind, double* total_ms, double* total_flops,
                                 int64_t* launches) {
  if (!ctx || kind < 0 || kind > 1) return QTX_E_INVAL;
  cudaSetDevice(ctx->device);
  drain_timing(ctx);
  if (total_ms) *total_ms = ctx->acc_ms[kind];
  if (total_flops) *total_flops = ctx->acc_flops[kind];
  if (launches) *launches = ctx->acc_launches[kind];
  return QTX_OK;
}

qtx_status qtx_inv(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a, int64_t stride_a, void* x,
                   int64_t stride_x, qtx_stream stream) {
  return guarded(ctx, [&] {
    if (n < 1 || batch < 0 || !a || !x) throw QtxError(QTX_E_INVAL, "qtx_inv: bad arguments");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    DevBuf info(sizeof(int) * std::max<int64_t>(batch, 1), s);
    launch_fill_int(info.as<int>(), std::max<int64_t>(batch, 1), 0, s);
    zinv(n, batch, MatView{reinterpret_cast<const cplx*>(a), n, stride_a},
                MutView{reinterpret_cast<cplx*>(x), n, stride_x}, info.as<int>(), nullptr, s);
    read_info_or_throw(ctx, info.as<int>(), batch, s, "qtx_inv");
  });
}

qtx_status qtx_zgemm(qtx_ctx* ctx, int32_t m, int32_t n, int32_t k, int64_t batch, double alpha_re,
                     double alpha_im, const void* a, int64_t lda, int64_t stride_a, int32_t op_a, const void* b,
                     int64_t ldb, int64_t stride_b, int32_t op_b, double beta_re, double beta_im, const void* c,
                     int64_t ldc, int64_t stride_c, void* d, int64_t ldd, int64_t stride_d, int32_t precision,
                     qtx_stream stream) {
  return guarded(ctx, [&] {
    if (m < 0 || n < 0 || k < 0 || batch < 0 || !a || !b || !d || (op_a != 0 && op_a != 1) ||
        (op_b != 0 && op_b != 1))
      throw QtxError(QTX_E_INVAL, "qtx_zgemm: bad arguments");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    gemm(m, n, k, batch, cmk(alpha_re, alpha_im), MatView{reinterpret_cast<const cplx*>(a), lda, stride_a}, op_a,
         MatView{reinterpret_cast<const cplx*>(b), ldb, stride_b}, op_b,
         MutView{reinterpret_cast<cplx*>(d), ldd, stride_d}, s,
         MatView{reinterpret_cast<const cplx*>(c), ldc, stride_c}, cmk(beta_re, beta_im), MatView{}, ZERO, nullptr,
         nullptr, precision);
    if (precision == QTX_PREC_MIXED) mixed_check_error(s);
  });
}

qtx_status qtx_selected_inv(qtx_ctx* ctx, const qtx_btd_desc* a_desc, const void* a,
                            const void* const* obc_retarded, const qtx_btd_desc* out_desc, void* out,
                            int64_t max_batch_size, int32_t precision, uint32_t flags, qtx_stream stream) {
  return guarded(ctx, [&] {
    validate_desc(a_desc, "a");
    validate_desc(out_desc, "out");
    check_same_blocks(a_desc, out_desc, "out");
    if (!a || !out) throw QtxError(QTX_E_INVAL, "qtx_selected_inv: null data");
    if (max_batch_size < 1) throw QtxError(QTX_E_INVAL, "qtx_selected_inv: max_batch_size < 1");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (flags & QTX_FLAG_HOST_BUFFERS) {
      const int nb = a_desc->num_blocks;
      const int bmax = *std::max_element(a_desc->block_sizes, a_desc->block_sizes + nb);
      std::vector<HostArr> arrs(2);
      arrs[0].h = reinterpret_cast<const char*>(a);
      arrs[0].row_bytes = desc_row_bytes(a_desc);
      arrs[0].in = true;
      arrs[1].hw = reinterpret_cast<char*>(out);
      arrs[1].row_bytes = desc_row_bytes(out_desc);
      arrs[1].out = true;
      std::vector<int> obc_i;
      add_obc_arrays(arrs, obc_retarded, a_desc, obc_i);
      size_t per_e = 0;
      for (auto& x : arrs) per_e += x.row_bytes;
      const int64_t NE = a_desc->stack_size;
      const int64_t ne_b = host_batch(max_batch_size, NE, per_e, nb, bmax);
      stream_host_batches(ctx, arrs, NE, ne_b, s, [&](int64_t, int64_t ne, int set) {
        qtx_btd_desc ad = batch_desc(a_desc, ne), od = batch_desc(out_desc, ne);
        std::vector<const void*> obc(nb, nullptr);
        for (size_t q = 0; q < obc_i.size(); ++q) obc[obc_i[q]] = arrs[2 + q].dev[set];
        Btd A{&ad, reinterpret_cast<cplx*>(arrs[0].dev[set])};
        Btd O{&od, reinterpret_cast<cplx*>(arrs[1].dev[set])};
        selected_inv_impl(ctx, A, obc_retarded ? obc.data() : nullptr, O, ne, precision, s);
      });
      return;
    }
    Btd A{a_desc, const_cast<cplx*>(reinterpret_cast<const cplx*>(a))};
    Btd O{out_desc, reinterpret_cast<cplx*>(out)};
    selected_inv_impl(ctx, A, obc_retarded, O, max_batch_size, precision, s);
  });
}

qtx_status qtx_selected_solve(qtx_ctx* ctx, const qtx_btd_desc* a_desc, const void* a,
                              const qtx_btd_desc* sl_desc, const void* sigma_lesser, const qtx_btd_desc* sg_desc,
                              const void* sigma_greater, const qtx_obc* obc, const qtx_btd_desc* xl_desc, void* xl,
                              const qtx_btd_desc* xg_desc, void* xg, const qtx_btd_desc* xr_desc, void* xr,
                              void* current, int64_t max_batch_size, int32_t precision, uint32_t flags,
                              qtx_stream stream) {
  return guarded(ctx, [&] {
    validate_desc(a_desc, "a");
    validate_desc(sl_desc, "sigma_lesser");
    validate_desc(sg_desc, "sigma_greater");
    validate_desc(xl_desc, "xl");
    validate_desc(xg_desc, "xg");
    check_same_blocks(a_desc, sl_desc, "sigma_lesser");
    check_same_blocks(a_desc, sg_desc, "sigma_greater");
    check_same_blocks(a_desc, xl_desc, "xl");
    check_same_blocks(a_desc, xg_desc, "xg");
    if ((flags & (QTX_FLAG_RETURN_RETARDED | QTX_FLAG_RETARDED_OFFDIAG)) && (!xr_desc || !xr))
      throw QtxError(QTX_E_INVAL, "qtx_selected_solve: retarded output requested without xr");
    if (xr_desc) {
      validate_desc(xr_desc, "xr");
      check_same_blocks(a_desc, xr_desc, "xr");
    }
    if ((flags & QTX_FLAG_RETURN_CURRENT) && !current)
      throw QtxError(QTX_E_INVAL, "qtx_selected_solve: current requested without a buffer");
    if (!a || !sigma_lesser || !sigma_greater || !xl || !xg)
      throw QtxError(QTX_E_INVAL, "qtx_selected_solve: null data");
    if (max_batch_size < 1) throw QtxError(QTX_E_INVAL, "qtx_selected_solve: max_batch_size < 1");
    if (flags & QTX_FLAG_HOST_BUFFERS) {
      cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
      const int nb = a_desc->num_blocks;
      const int bmax = *std::max_element(a_desc->block_sizes, a_desc->block_sizes + nb);
      const bool want_xr = xr_desc && xr;
      const bool want_cur = (flags & QTX_FLAG_RETURN_CURRENT) != 0;
      std::vector<HostArr> arrs;
      auto add = [&](const qtx_btd_desc* d, const void* p, bool is_out) {
        HostArr h;
        h.row_bytes = desc_row_bytes(d);
        if (is_out) {
          h.hw = reinterpret_cast<char*>(const_cast<void*>(p));
          h.out = true;
        } else {
          h.h = reinterpret_cast<const char*>(p);
          h.in = true;
        }
        arrs.push_back(h);
      };
      add(a_desc, a, false);
      add(sl_desc, sigma_lesser, false);
      add(sg_desc, sigma_greater, false);
      add(xl_desc, xl, true);
      add(xg_desc, xg, true);
      if (want_xr) add(xr_desc, xr, true);
      if (want_cur) {
        HostArr h;
        h.hw = reinterpret_cast<char*>(current);
        h.row_bytes = sizeof(cplx) * (size_t)(nb - 1);
        h.out = true;
        arrs.push_back(h);
      }
      const size_t first_obc = arrs.size();
      std::vector<int> oi_r, oi_l, oi_g;
      add_obc_arrays(arrs, obc ? obc->retarded : nullptr, a_desc, oi_r);
      add_obc_arrays(arrs, obc ? obc->lesser : nullptr, a_desc, oi_l);
      add_obc_arrays(arrs, obc ? obc->greater : nullptr, a_desc, oi_g);
      size_t per_e = 0;
      for (auto& x : arrs) per_e += x.row_bytes;
      const int64_t NE = a_desc->stack_size;
      const int64_t ne_b = host_batch(max_batch_size, NE, per_e, nb, bmax);
      stream_host_batches(ctx, arrs, NE, ne_b, s, [&](int64_t, int64_t ne, int set) {
        qtx_btd_desc ad = batch_desc(a_desc, ne), sld = batch_desc(sl_desc, ne), sgd = batch_desc(sg_desc, ne);
        qtx_btd_desc xld = batch_desc(xl_desc, ne), xgd = batch_desc(xg_desc, ne);
        qtx_btd_desc xrd = want_xr ? batch_desc(xr_desc, ne) : qtx_btd_desc{};
        std::vector<const void*> r(nb, nullptr), l(nb, nullptr), g(nb, nullptr);
        size_t q = first_obc;
        for (int i : oi_r) r[i] = arrs[q++].dev[set];
        for (int i : oi_l) l[i] = arrs[q++].dev[set];
        for (int i : oi_g) g[i] = arrs[q++].dev[set];
        qtx_obc ob{oi_r.empty() ? nullptr : r.data(), oi_l.empty() ? nullptr : l.data(),
                   oi_g.empty() ? nullptr : g.data()};
        SolveArgs S;
        S.a = Btd{&ad, reinterpret_cast<cplx*>(arrs[0].dev[set])};
        S.sl = Btd{&sld, reinterpret_cast<cplx*>(arrs[1].dev[set])};
        S.sg = Btd{&sgd, reinterpret_cast<cplx*>(arrs[2].dev[set])};
        S.xl = Btd{&xld, reinterpret_cast<cplx*>(arrs[3].dev[set])};
        S.xg = Btd{&xgd, reinterpret_cast<cplx*>(arrs[4].dev[set])};
        S.xr = want_xr ? Btd{&xrd, reinterpret_cast<cplx*>(arrs[5].dev[set])} : Btd{};
        S.obc = obc ? &ob : nullptr;
        S.current = want_cur ? reinterpret_cast<cplx*>(arrs[want_xr ? 6 : 5].dev[set]) : nullptr;
        S.flags = flags & ~QTX_FLAG_HOST_BUFFERS;
        S.max_batch = ne;
        S.precision = precision;
        selected_solve_impl(ctx, S, s);
      });
      return;
    }
    SolveArgs S;
    S.a = Btd{a_desc, const_cast<cplx*>(reinterpret_cast<const cplx*>(a))};
    S.sl = Btd{sl_desc, const_cast<cplx*>(reinterpret_cast<const cplx*>(sigma_lesser))};
    S.sg = Btd{sg_desc, const_cast<cplx*>(reinterpret_cast<const cplx*>(sigma_greater))};
    S.xl = Btd{xl_desc, reinterpret_cast<cplx*>(xl)};
    S.xg = Btd{xg_desc, reinterpret_cast<cplx*>(xg)};
    S.xr = Btd{xr_desc, reinterpret_cast<cplx*>(xr)};
    S.obc = obc;
    S.current = reinterpret_cast<cplx*>(current);
    S.flags = flags;
    S.max_batch = max_batch_size;
    S.precision = precision;
    selected_solve_impl(ctx, S, reinterpret_cast<cudaStream_t>(stream));
  });
}

qtx_status qtx_sancho_rubio(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                            const void* a_ij, int64_t stride_ij, const void* a_ji, int64_t stride_ji,
                            double convergence_tol, int32_t max_iterations, void* x, int32_t* iterations,
                            qtx_stream stream) {
  bool ok = true;
  qtx_status st = guarded(ctx, [&] {
    if (n < 1 || batch < 0 || max_iterations < 1 || (batch > 0 && (!a_ii || !a_ij || !a_ji || !x)))
      throw QtxError(QTX_E_INVAL, "qtx_sancho_rubio: bad arguments");
    if (batch == 0) return;  // an empty energy batch: nothing to decimate
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    ok = sancho_rubio_impl(ctx, n, batch, MatView{reinterpret_cast<const cplx*>(a_ii), n, stride_ii},
                           MatView{reinterpret_cast<const cplx*>(a_ij), n, stride_ij},
                           MatView{reinterpret_cast<const cplx*>(a_ji), n, stride_ji}, convergence_tol,
                           max_iterations, MutView{reinterpret_cast<cplx*>(x), n, (int64_t)n * n}, iterations, s);
    QTX_CUDA_TRY(cudaStreamSynchronize(s));
  });
  if (st == QTX_OK && !ok) {
    ctx->last_error = "Surface Green's function did not converge.";
    return QTX_E_NOT_CONVERGED;
  }
  return st;
}

qtx_status qtx_block_combine(qtx_ctx* ctx, int32_t rows, int32_t cols, int64_t batch, double alpha_re,
                             double alpha_im, const void* x, int64_t ldx, int64_t stride_x, int32_t op_x,
                             double beta_re, double beta_im, const void* y, int64_t ldy, int64_t stride_y,
                             int32_t op_y, void* out, int64_t ldo, int64_t stride_out, qtx_stream stream) {
  return guarded(ctx, [&] {
    if (rows < 0 || cols < 0 || batch < 0 || !x || !out || (op_x != 0 && op_x != 1) || (op_y != 0 && op_y != 1))
      throw QtxError(QTX_E_INVAL, "qtx_block_combine: bad arguments");
    if ((op_x == OP_C && x == out) || (y && op_y == OP_C && y == out))
      throw QtxError(QTX_E_INVAL, "qtx_block_combine: a transposed operand may not alias the output");
    launch_block_combine(rows, cols, batch, cmk(alpha_re, alpha_im),
                         MatView{reinterpret_cast<const cplx*>(x), ldx, stride_x}, op_x, cmk(beta_re, beta_im),
                         MatView{reinterpret_cast<const cplx*>(y), ldy, stride_y}, op_y,
                         MutView{reinterpret_cast<cplx*>(out), ldo, stride_out}, reinterpret_cast<cudaStream_t>(stream));
  });
}

qtx_status qtx_beyn_moments(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                            const void* a_ij, int64_t stride_ij, const void* a_ji, int64_t stride_ji, double r_o,
                            double r_i, int32_t num_quad_points, const void* y, int32_t m0, void* p0, void* p1,
                            qtx_stream stream) {
  return guarded(ctx, [&] {
    if (n < 1 || batch < 0 || m0 < 1 || num_quad_points < 1 || !a_ii || !a_ij || !a_ji || !y || !p0 || !p1 ||
        !(r_o > r_i) || !(r_i > 0))
      throw QtxError(QTX_E_INVAL, "qtx_beyn_moments: bad arguments");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int nq = num_quad_points;
    const int64_t nn = (int64_t)n * n;
    // energies per pass: the 2 nq operator inverses of a pass stay below 4 GiB
    const int64_t per_energy = (int64_t)2 * nq * nn * (int64_t)sizeof(cplx);
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(batch, ((int64_t)4 << 30) / per_energy));
    DevBuf buf(sizeof(cplx) * (size_t)(chunk * 2 * nq * nn + 2 * chunk * nn) + sizeof(int) * (size_t)(chunk * 2 * nq),
               s);
    cplx* ops = buf.as<cplx>();
    cplx* q = ops + chunk * 2 * nq * nn;
    int* info = reinterpret_cast<int*>(q + 2 * chunk * nn);
    launch_fill_int(info, chunk * 2 * nq, 0, s);
    for (int64_t e0 = 0; e0 < batch; e0 += chunk) {
      const int64_t ne = std::min(chunk, batch - e0);
      MatView aii{reinterpret_cast<const cplx*>(a_ii) + e0 * stride_ii, n, stride_ii};
      MatView aij{reinterpret_cast<const cplx*>(a_ij) + e0 * stride_ij, n, stride_ij};
      MatView aji{reinterpret_cast<const cplx*>(a_ji) + e0 * stride_ji, n, stride_ji};
      launch_contour_operator(n, ne, nq, r_o, r_i, aii, aij, aji, ops, s);
      zinv(n, ne * 2 * nq, MatView{ops, n, nn}, MutView{ops, n, nn}, info, nullptr, s);
      MutView q0{q, n, nn}, q1{q + ne * nn, n, nn};
      launch_contour_moments(n, ne, nq, r_o, r_i, ops, q0, q1, s);
      const int64_t ym = (int64_t)n * m0;
      MatView yv{reinterpret_cast<const cplx*>(y) + e0 * ym, m0, ym};
      gemm(n, m0, n, ne, ONE, q0, OP_N, yv, OP_N, MutView{reinterpret_cast<cplx*>(p0) + e0 * ym, m0, ym}, s);
      gemm(n, m0, n, ne, ONE, q1, OP_N, yv, OP_N, MutView{reinterpret_cast<cplx*>(p1) + e0 * ym, m0, ym}, s);
    }
    read_info_or_throw(ctx, info, chunk * 2 * nq, s, "qtx_beyn_moments (contour operator)");
  });
}

qtx_status qtx_spectral_surface(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                                const void* a_ij, int64_t stride_ij, const void* a_ji, int64_t stride_ji,
                                const void* ws, void* vs, int32_t m0, const qtx_spectral_params* params,
                                int32_t* mask, void* x, qtx_stream stream) {
  return guarded(ctx, [&] {
    if (n < 1 || batch < 0 || m0 < 1 || !a_ii || !a_ij || !a_ji || !ws || !vs || !params || !x ||
        params->num_ref_iterations < 1)
      throw QtxError(QTX_E_INVAL, "qtx_spectral_surface: bad arguments");
    if (batch == 0) return;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int64_t nn = (int64_t)n * n, nm = (int64_t)n * m0, mm = (int64_t)m0 * m0;
    DevBuf buf(sizeof(cplx) * (size_t)(batch * (5 * nm + 2 * mm + 3 * nn)) + sizeof(int) * (size_t)(batch * (m0 + 1)),
               s);
    cplx* p = buf.as<cplx>();
    cplx* r_ji = p;
    cplx* r_ii = r_ji + batch * nm;
    cplx* r_ij = r_ii + batch * nm;
    cplx* vm = r_ij + batch * nm;
    cplx* vw = vm + batch * nm;
    cplx* g = vw + batch * nm;
    cplx* gi = g + batch * mm;
    cplx* t0 = gi + batch * mm;
    cplx* t1 = t0 + batch * nn;
    cplx* t2 = t1 + batch * nn;
    int* d_mask = reinterpret_cast<int*>(t2 + batch * nn);
    int* info = d_mask + batch * m0;
    launch_fill_int(info, batch, 0, s);
    MatView aii{reinterpret_cast<const cplx*>(a_ii), n, stride_ii};
    MatView aij{reinterpret_cast<const cplx*>(a_ij), n, stride_ij};
    MatView aji{reinterpret_cast<const cplx*>(a_ji), n, stride_ji};
    cplx* v = reinterpret_cast<cplx*>(vs);
    const cplx* w = reinterpret_cast<const cplx*>(ws);
    // unit eigenvectors (spectral.py:355-358), then the mode classification
    launch_normalize_columns(n, m0, batch, v, s);
    MatView vv{v, m0, nm};
    gemm(n, m0, n, batch, ONE, aji, OP_N, vv, OP_N, MutView{r_ji, m0, nm}, s);
    gemm(n, m0, n, batch, ONE, aii, OP_N, vv, OP_N, MutView{r_ii, m0, nm}, s);
    gemm(n, m0, n, batch, ONE, aij, OP_N, vv, OP_N, MutView{r_ij, m0, nm}, s);
    SpectralFilter f;
    f.min_decay = params->min_decay;
    f.max_decay = params->max_decay;
    f.min_propagation = params->min_propagation;
    f.residual_tolerance = params->residual_tolerance;
    f.eta_decay = params->eta_decay;
    f.residual_normalization = params->residual_normalization;
    launch_mode_filter(n, m0, batch, w, v, r_ji, r_ii, r_ij, f, d_mask, s);
    // x a_ij = V_r diag(1 / w_r) (V_r^H V_r)^-1 V_r^H over the reflected modes
    // (spectral.py:400-415): with the unselected columns zeroed and the
    // unselected block of the Gram matrix set to the identity, one batched
    // product covers every energy whatever its number of modes
    launch_masked_modes(n, m0, batch, w, v, d_mask, vm, vw, s);
    gemm(m0, m0, n, batch, ONE, MatView{vm, m0, nm}, OP_C, MatView{vm, m0, nm}, OP_N, MutView{g, m0, mm}, s);
    launch_gram_identity(m0, batch, d_mask, g, s);
    zinv(m0, batch, MatView{g, m0, mm}, MutView{gi, m0, mm}, nullptr, nullptr, s);
    // t0 (m0 x n) = G^-1 V_m^H ; t1 = V_w t0 = x a_ij
    gemm(m0, n, m0, batch, ONE, MatView{gi, m0, mm}, OP_N, MatView{vm, m0, nm}, OP_C, MutView{t0, n, nm}, s);
    gemm(n, n, m0, batch, ONE, MatView{vw, m0, nm}, OP_N, MatView{t0, n, nm}, OP_N, MutView{t1, n, nn}, s);
    // x = inv(a_ii + a_ji (x a_ij)), then num_ref_iterations fixed-point
    // steps x = inv(a_ii - a_ji x a_ij) (spectral.py:491-526)
    gemm(n, n, n, batch, ONE, aji, OP_N, MatView{t1, n, nn}, OP_N, MutView{t2, n, nn}, s, aii, ONE);
    MutView xv{reinterpret_cast<cplx*>(x), n, nn};
    zinv(n, batch, MatView{t2, n, nn}, xv, info, nullptr, s);
    for (int it = 0; it < params->num_ref_iterations; ++it) {
      gemm(n, n, n, batch, ONE, aji, OP_N, xv, OP_N, MutView{t0, n, nn}, s);
      gemm(n, n, n, batch, MONE, MatView{t0, n, nn}, OP_N, aij, OP_N, MutView{t2, n, nn}, s, aii, ONE);
      zinv(n, batch, MatView{t2, n, nn}, xv, info, nullptr, s);
    }
    if (mask) QTX_CUDA_TRY(cudaMemcpyAsync(mask, d_mask, sizeof(int) * (size_t)(batch * m0), cudaMemcpyDeviceToDevice, s));
    read_info_or_throw(ctx, info, batch, s, "qtx_spectral_surface");
  });
}

qtx_status qtx_obc_fixed_point(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                               const void* a_ij, int64_t stride_ij, const void* a_ji, int64_t stride_ji,
                               const void* x, void* x_ref, double* abs_res, double* rel_res, qtx_stream stream) {
  return guarded(ctx, [&] {
    if (n < 1 || batch < 1 || !a_ii || !a_ij || !a_ji || !x || !x_ref) throw QtxError(QTX_E_INVAL, "qtx_obc_fixed_point");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int64_t bb = (int64_t)n * n;
    DevBuf t(sizeof(cplx) * 2 * bb * batch, s);
    MutView t0{t.as<cplx>(), n, bb}, t1{t.as<cplx>() + bb * batch, n, bb};
    MatView aii{reinterpret_cast<const cplx*>(a_ii), n, stride_ii};
    MatView aij{reinterpret_cast<const cplx*>(a_ij), n, stride_ij};
    MatView aji{reinterpret_cast<const cplx*>(a_ji), n, stride_ji};
    MatView xv{reinterpret_cast<const cplx*>(x), n, bb};
    // x_ref = inv(a_ii - a_ji x a_ij)
    gemm(n, n, n, batch, ONE, aji, OP_N, xv, OP_N, t0, s);
    gemm(n, n, n, batch, MONE, t0, OP_N, aij, OP_N, t1, s, aii, ONE);
    DevBuf info(sizeof(int) * batch, s);
    launch_fill_int(info.as<int>(), batch, 0, s);
    zinv(n, batch, t1, MutView{reinterpret_cast<cplx*>(x_ref), n, bb}, info.as<int>(), nullptr, s);
    if (abs_res && rel_res)
      launch_residual_norm(n, batch, MatView{reinterpret_cast<cplx*>(x_ref), n, bb}, xv, abs_res, rel_res, s);
    read_info_or_throw(ctx, info.as<int>(), batch, s, "qtx_obc_fixed_point");
  });
}

qtx_status qtx_obc_assemble(qtx_ctx* ctx, int32_t n, int64_t batch, const void* g, const void* m_ji,
                            int64_t stride_ji, const void* m_ij, int64_t stride_ij, const double* occupancy,
                            void* sigma_r, void* sigma_l, void* sigma_g, qtx_stream stream) {
  return guarded(ctx, [&] {
    if (n < 1 || batch < 0 || !g || !m_ji || !m_ij || !sigma_r) throw QtxError(QTX_E_INVAL, "qtx_obc_assemble");
    if ((sigma_l || sigma_g) && !occupancy) throw QtxError(QTX_E_INVAL, "qtx_obc_assemble: occupancy missing");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int64_t bb = (int64_t)n * n;
    DevBuf t(sizeof(cplx) * bb * std::max<int64_t>(batch, 1), s);
    gemm(n, n, n, batch, ONE, MatView{reinterpret_cast<const cplx*>(m_ji), n, stride_ji}, OP_N,
         MatView{reinterpret_cast<const cplx*>(g), n, bb}, OP_N, MutView{t.as<cplx>(), n, bb}, s);
    gemm(n, n, n, batch, ONE, MatView{t.as<cplx>(), n, bb}, OP_N,
         MatView{reinterpret_cast<const cplx*>(m_ij), n, stride_ij}, OP_N,
         MutView{reinterpret_cast<cplx*>(sigma_r), n, bb}, s);
    if (sigma_l || sigma_g)
      launch_obc_lesser_greater(n, batch, MatView{reinterpret_cast<cplx*>(sigma_r), n, bb}, occupancy,
                                MutView{reinterpret_cast<cplx*>(sigma_l), n, bb},
                                MutView{reinterpret_cast<cplx*>(sigma_g), n, bb}, MutView{}, s);
  });
}

qtx_status qtx_transport_solve_grouped(qtx_ctx* ctx, int32_t count, const qtx_transport_problem* problems,
                                       const qtx_transport_outputs* outputs, int32_t precision, uint32_t flags,
                                       qtx_status* statuses, qtx_stream stream) {
  std::vector<int> fl;
  qtx_status st = guarded(ctx, [&] {
    if (count < 1 || !problems || !outputs) throw QtxError(QTX_E_INVAL, "qtx_transport_solve_grouped: no problems");
    if (precision != QTX_PREC_FP64)
      throw QtxError(QTX_E_UNSUPPORTED, "qtx_transport_solve_grouped: FP64 products only");
    (void)flags;
    fl = transport_grouped_impl(count, problems, outputs, reinterpret_cast<cudaStream_t>(stream));
  });
  if (st != QTX_OK) {
    if (statuses)
      for (int q = 0; q < count; ++q) statuses[q] = st;
    return st;
  }
  bool singular = false, unconverged = false;
  for (int q = 0; q < count; ++q) {
    const qtx_status s = (fl[q] & 1) ? QTX_E_SINGULAR : ((fl[q] & 2) ? QTX_E_NOT_CONVERGED : QTX_OK);
    if (statuses) statuses[q] = s;
    singular = singular || s == QTX_E_SINGULAR;
    unconverged = unconverged || s == QTX_E_NOT_CONVERGED;
  }
  if (singular) {
    ctx->last_error = "qtx_transport_solve_grouped: exactly singular diagonal block";
    return QTX_E_SINGULAR;
  }
  if (unconverged) {
    ctx->last_error = "Surface Green's function did not converge.";
    return QTX_E_NOT_CONVERGED;
  }
  return QTX_OK;
}

size_t qtx_transport_grouped_footprint(int32_t count, const int32_t* num_blocks, const int64_t* num_energies,
                                       int32_t block_size) {
  if (count < 1 || !num_blocks || !num_energies || block_size < 1 || block_size > GROUPED_MAX_B) return 0;
  int max_nb = 0;
  int64_t items = 0;
  for (int q = 0; q < count; ++q) {
    max_nb = std::max(max_nb, num_blocks[q]);
    items += std::max<int64_t>(num_energies[q], 0);
  }
  if (items == 0) return 0;
  GroupedPlan plan;
  plan.b = block_size;
  plan.max_nb = max_nb;
  plan.problems.resize(count);
  return grouped_bytes(plan, grouped_grid(block_size, items));
}

qtx_status qtx_transport_solve(qtx_ctx* ctx, const qtx_transport_problem* p, const qtx_transport_outputs* o,
                               int32_t precision, uint32_t flags, qtx_stream stream) {
  bool ok = true;
  qtx_status st = guarded(ctx, [&] {
    if (!p || !o) throw QtxError(QTX_E_INVAL, "qtx_transport_solve: null problem");
    if (p->num_blocks < 2 || p->block_size < 1 || p->num_energies < 0 || !p->h_diag || !p->h_upper ||
        (p->num_energies > 0 && !p->energies) || p->kt <= 0 || p->sr_max_iterations < 1)
      throw QtxError(QTX_E_INVAL, "qtx_transport_solve: bad problem");
    if (p->num_energies == 0) return;  // an empty energy grid: nothing to solve
    const bool use_graph = (flags & QTX_FLAG_GRAPH) != 0 &&
                           (p->max_batch_size <= 0 || p->max_batch_size >= p->num_energies);
    if (use_graph) transport_graph_impl(ctx, *p, *o, precision, reinterpret_cast<cudaStream_t>(stream), ok);
    else transport_impl(ctx, *p, *o, precision, reinterpret_cast<cudaStream_t>(stream), ok);
  });
  if (st == QTX_OK && !ok) {
    ctx->last_error = "Surface Green's function did not converge.";
    return QTX_E_NOT_CONVERGED;
  }
  return st;
}

}  // extern "C"
