// Continuous-batching transport server: the native runtime of the serving form
// (declared in include/qtx_rgf.h; no counterpart in the reference, which
// solves one request at a time).
//
// `slots` worker threads each own a library context and a non-blocking CUDA
// stream.  Requests wait in arrival order; a worker takes the oldest one as
// soon as its footprint (qtx_transport_footprint at the request's energies per
// call) fits in the memory budget next to the requests already running, runs
// qtx_transport_solve on its stream and synchronises that stream only.
// Requests admitted while others run overlap with them on the device.  With
// grouping on, a worker that admits an FP64 request of a small block size
// also takes the waiting FP64 requests of the same block size that fit the
// budget (arrival order) and solves them in one qtx_transport_solve_grouped
// launch (one persistent kernel for all their energies).  Nothing here
// synchronises the whole device.  Latency = completion - submission (steady
// clock); every completed request's latency is kept for p50/p99.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/qtx_rgf.h"

namespace {

constexpr int kMaxGroup = 256;  // requests per grouped launch

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  qtx_transport_problem p{};
  qtx_transport_outputs o{};
  int32_t precision = QTX_PREC_FP64;
  uint32_t flags = 0;
  size_t footprint = 0;
  Clock::time_point submitted;
  bool done = false;
  qtx_status status = QTX_OK;
  double latency_s = 0;
  std::string error;
};

}  // namespace

struct qtx_server {
  qtx_server_config cfg{};
  size_t budget = 0;
  std::mutex m;
  std::condition_variable cv_work;  // queue changed, memory freed, or closing
  std::condition_variable cv_done;  // a request completed
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<int64_t, std::shared_ptr<Request>> pending;  // submitted, not yet collected
  std::deque<int64_t> completed_uncollected;
  std::vector<std::thread> workers;
  std::vector<double> latencies;
  int64_t next_id = 1;
  int64_t submitted = 0, completed = 0, failed = 0, running = 0, peak_running = 0, solves = 0;
  int64_t grouped_launches = 0, grouped_requests = 0;
  size_t in_use = 0;
  bool closing = false;
  int start_errors = 0;
};

namespace {

bool groupable(const qtx_server* srv, const Request& r) {
  const int gmax = std::min(srv->cfg.group_max_block_size, 64);
  return gmax > 0 && r.precision == QTX_PREC_FP64 && r.p.block_size <= gmax;
}

size_t group_footprint(const std::vector<std::shared_ptr<Request>>& g) {
  std::vector<int32_t> nbs;
  std::vector<int64_t> nes;
  for (const auto& r : g) {
    nbs.push_back(r->p.num_blocks);
    nes.push_back(r->p.num_energies);
  }
  return qtx_transport_grouped_footprint((int32_t)g.size(), nbs.data(), nes.data(), g[0]->p.block_size);
}

// Complete one request (lock held).
void finish(qtx_server* srv, const std::shared_ptr<Request>& req, qtx_status st, const std::string& err,
            double lat) {
  req->done = true;
  req->status = st;
  req->latency_s = lat;
  if (st != QTX_OK && st != QTX_E_NOT_CONVERGED) {
    req->error = err;
    ++srv->failed;
  } else {
    if (st == QTX_E_NOT_CONVERGED) req->error = err;
    ++srv->completed;
    srv->solves += req->p.num_energies;
    srv->latencies.push_back(lat);
  }
  srv->completed_uncollected.push_back(req->id);
}

void worker_main(qtx_server* srv) {
  qtx_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;
  bool ok = cudaSetDevice(srv->cfg.device) == cudaSuccess && qtx_ctx_create(srv->cfg.device, &ctx) == QTX_OK &&
            cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    std::lock_guard<std::mutex> lk(srv->m);
    ++srv->start_errors;
  }
  for (;;) {
    std::vector<std::shared_ptr<Request>> group;
    size_t fp = 0;
    bool grouped = false;
    {
      std::unique_lock<std::mutex> lk(srv->m);
      srv->cv_work.wait(lk, [&] {
        if (srv->queue.empty()) return srv->closing;
        const auto& head = srv->queue.front();
        return srv->running == 0 || srv->in_use + head->footprint <= srv->budget;
      });
      if (srv->queue.empty()) break;  // closing and drained
      std::shared_ptr<Request> head = srv->queue.front();
      srv->queue.pop_front();
      group.push_back(head);
      fp = head->footprint;
      if (groupable(srv, *head)) {
        grouped = true;
        // the waiting requests of the same block size, in arrival order, while
        // the group's work space fits next to the running requests
        for (auto it = srv->queue.begin(); it != srv->queue.end() && (int)group.size() < kMaxGroup;) {
          const auto& r = *it;
          if (!groupable(srv, *r) || r->p.block_size != head->p.block_size) {
            ++it;
            continue;
          }
          group.push_back(r);
          const size_t need = std::max(fp, group_footprint(group));
          if (srv->in_use + need > srv->budget) {
            group.pop_back();
            break;
          }
          fp = need;
          it = srv->queue.erase(it);
        }
      }
      srv->in_use += fp;
      srv->running += (int64_t)group.size();
      srv->peak_running = std::max(srv->peak_running, srv->running);
    }
    std::vector<qtx_status> st(group.size(), QTX_E_CUDA);
    std::string err = "server worker could not create its context or stream";
    if (ok && grouped) {
      std::vector<qtx_transport_problem> ps;
      std::vector<qtx_transport_outputs> os;
      for (const auto& r : group) {
        ps.push_back(r->p);
        os.push_back(r->o);
      }
      const qtx_status s = qtx_transport_solve_grouped(ctx, (int32_t)group.size(), ps.data(), os.data(),
                                                       QTX_PREC_FP64, 0, st.data(), stream);
      if (s != QTX_OK) err = qtx_last_error(ctx);
    } else if (ok) {
      st[0] = qtx_transport_solve(ctx, &group[0]->p, &group[0]->o, group[0]->precision, group[0]->flags, stream);
      if (st[0] != QTX_OK) err = qtx_last_error(ctx);
    }
    if (ok && cudaStreamSynchronize(stream) != cudaSuccess) {
      err = cudaGetErrorString(cudaGetLastError());
      for (auto& s : st)
        if (s == QTX_OK) s = QTX_E_CUDA;
    }
    const auto now = Clock::now();
    {
      std::lock_guard<std::mutex> lk(srv->m);
      for (size_t i = 0; i < group.size(); ++i)
        finish(srv, group[i], st[i], err, std::chrono::duration<double>(now - group[i]->submitted).count());
      if (grouped && ok) {
        ++srv->grouped_launches;
        srv->grouped_requests += (int64_t)group.size();
      }
      srv->in_use -= fp;
      srv->running -= (int64_t)group.size();
    }
    srv->cv_work.notify_all();
    srv->cv_done.notify_all();
  }
  if (stream) cudaStreamDestroy(stream);
  if (ctx) qtx_ctx_destroy(ctx);
}

void copy_error(const std::string& msg, char* err, int32_t err_len) {
  if (!err || err_len <= 0) return;
  const size_t n = std::min<size_t>(msg.size(), (size_t)err_len - 1);
  memcpy(err, msg.data(), n);
  err[n] = '\0';
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  // linear interpolation between closest ranks (numpy's default)
  const double pos = q * (double)(v.size() - 1);
  const size_t lo = (size_t)pos;
  const size_t hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (pos - (double)lo) * (v[hi] - v[lo]);
}

// Collect a completed request (lock held).
qtx_status collect(qtx_server* srv, const std::shared_ptr<Request>& req, qtx_status* request_status,
                   double* latency_s, char* err, int32_t err_len) {
  if (request_status) *request_status = req->status;
  if (latency_s) *latency_s = req->latency_s;
  copy_error(req->error, err, err_len);
  srv->pending.erase(req->id);
  auto it = std::find(srv->completed_uncollected.begin(), srv->completed_uncollected.end(), req->id);
  if (it != srv->completed_uncollected.end()) srv->completed_uncollected.erase(it);
  return QTX_OK;
}

}  // namespace

extern "C" {

qtx_status qtx_server_create(const qtx_server_config* cfg, qtx_server** out) {
  if (!cfg || !out || cfg->slots < 1) return QTX_E_INVAL;
  *out = nullptr;
  if (cudaSetDevice(cfg->device) != cudaSuccess) {
    cudaGetLastError();
    return QTX_E_CUDA;
  }
  auto* srv = new qtx_server();
  srv->cfg = *cfg;
  srv->budget = cfg->memory_budget;
  if (srv->budget == 0) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      delete srv;
      return QTX_E_CUDA;
    }
    srv->budget = free_b / 2;
  }
  for (int i = 0; i < cfg->slots; ++i) srv->workers.emplace_back(worker_main, srv);
  *out = srv;
  return QTX_OK;
}

qtx_status qtx_server_destroy(qtx_server* srv) {
  if (!srv) return QTX_E_INVAL;
  {
    std::lock_guard<std::mutex> lk(srv->m);
    srv->closing = true;
  }
  srv->cv_work.notify_all();
  for (auto& t : srv->workers) t.join();
  delete srv;
  return QTX_OK;
}

qtx_status qtx_server_submit(qtx_server* srv, const qtx_transport_problem* p, const qtx_transport_outputs* o,
                             int32_t precision, uint32_t flags, int64_t* request_id) {
  if (!srv || !p || !o || !request_id) return QTX_E_INVAL;
  if (p->num_blocks < 2 || p->block_size < 1 || p->num_energies < 1 || !p->h_diag || !p->h_upper ||
      !p->energies || p->kt <= 0 || p->sr_max_iterations < 1)
    return QTX_E_INVAL;
  if (precision != QTX_PREC_FP64 && precision != QTX_PREC_MIXED) return QTX_E_INVAL;
  auto req = std::make_shared<Request>();
  req->p = *p;
  req->o = *o;
  req->precision = precision;
  // every request brings its own buffers, so a captured sweep would never be
  // replayed and its work space would escape the admission budget
  req->flags = flags & ~QTX_FLAG_GRAPH;
  const int64_t ne_call = p->max_batch_size > 0 ? std::min(p->max_batch_size, p->num_energies) : p->num_energies;
  req->footprint = qtx_transport_footprint(p->num_blocks, p->block_size, ne_call, precision);
  if (groupable(srv, *req)) {
    // solved in a grouped launch: its work space when it runs alone
    const int32_t nb = p->num_blocks;
    const int64_t ne = p->num_energies;
    req->footprint = std::max(req->footprint, qtx_transport_grouped_footprint(1, &nb, &ne, p->block_size));
  }
  std::lock_guard<std::mutex> lk(srv->m);
  if (srv->closing) return QTX_E_INVAL;
  if (req->footprint > srv->budget) return QTX_E_NOMEM;
  req->id = srv->next_id++;
  req->submitted = Clock::now();
  srv->pending[req->id] = req;
  srv->queue.push_back(req);
  ++srv->submitted;
  *request_id = req->id;
  srv->cv_work.notify_all();
  return QTX_OK;
}

qtx_status qtx_server_wait(qtx_server* srv, int64_t request_id, int64_t timeout_ms, qtx_status* request_status,
                           double* latency_s, char* err, int32_t err_len) {
  if (!srv) return QTX_E_INVAL;
  std::unique_lock<std::mutex> lk(srv->m);
  auto it = srv->pending.find(request_id);
  if (it == srv->pending.end()) return QTX_E_INVAL;
  std::shared_ptr<Request> req = it->second;
  auto ready = [&] { return req->done; };
  if (timeout_ms < 0) srv->cv_done.wait(lk, ready);
  else if (!srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return QTX_E_TIMEOUT;
  return collect(srv, req, request_status, latency_s, err, err_len);
}

qtx_status qtx_server_wait_any(qtx_server* srv, int64_t timeout_ms, int64_t* request_id, qtx_status* request_status,
                               double* latency_s, char* err, int32_t err_len) {
  if (!srv || !request_id) return QTX_E_INVAL;
  std::unique_lock<std::mutex> lk(srv->m);
  auto ready = [&] { return !srv->completed_uncollected.empty(); };
  if (timeout_ms < 0) {
    if (srv->pending.empty()) return QTX_E_INVAL;
    srv->cv_done.wait(lk, ready);
  } else if (!srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return QTX_E_TIMEOUT;
  }
  const int64_t id = srv->completed_uncollected.front();
  auto it = srv->pending.find(id);
  if (it == srv->pending.end()) {  // collected by qtx_server_wait meanwhile
    srv->completed_uncollected.pop_front();
    return QTX_E_TIMEOUT;
  }
  *request_id = id;
  std::shared_ptr<Request> req = it->second;
  return collect(srv, req, request_status, latency_s, err, err_len);
}

qtx_status qtx_server_get_stats(qtx_server* srv, qtx_server_stats* st) {
  if (!srv || !st) return QTX_E_INVAL;
  std::lock_guard<std::mutex> lk(srv->m);
  st->submitted = srv->submitted;
  st->completed = srv->completed;
  st->failed = srv->failed;
  st->queued = (int64_t)srv->queue.size();
  st->running = srv->running;
  st->peak_running = srv->peak_running;
  st->solves = srv->solves;
  st->memory_in_use = srv->in_use;
  st->p50_latency_s = percentile(srv->latencies, 0.50);
  st->p99_latency_s = percentile(srv->latencies, 0.99);
  double sum = 0;
  for (double x : srv->latencies) sum += x;
  st->mean_latency_s = srv->latencies.empty() ? 0.0 : sum / (double)srv->latencies.size();
  st->grouped_launches = srv->grouped_launches;
  st->grouped_requests = srv->grouped_requests;
  return QTX_OK;
}

}  // extern "C"
