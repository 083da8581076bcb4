// Continuous-batching transport server: the native runtime of the serving form
// (declared in include/qtx_rgf.h; no counterpart in the reference, which
// solves one request at a time).
//
// `slots` worker threads each own a library context and a non-blocking CUDA
// stream.  Requests wait in arrival order; a worker takes the oldest one as
// soon as its footprint (qtx_transport_footprint at the request's energies per
// call) fits in the memory budget next to the requests already running, runs
// qtx_transport_solve on its stream and synchronises that stream only.
// Requests admitted while others run overlap with them on the device.  Nothing
// here synchronises the whole device.  Latency = completion - submission
// (steady clock); every completed request's latency is kept for p50/p99.
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
  size_t in_use = 0;
  bool closing = false;
  int start_errors = 0;
};

namespace {

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
    std::shared_ptr<Request> req;
    {
      std::unique_lock<std::mutex> lk(srv->m);
      srv->cv_work.wait(lk, [&] {
        if (srv->queue.empty()) return srv->closing;
        const auto& head = srv->queue.front();
        return srv->running == 0 || srv->in_use + head->footprint <= srv->budget;
      });
      if (srv->queue.empty()) break;  // closing and drained
      req = srv->queue.front();
      srv->queue.pop_front();
      srv->in_use += req->footprint;
      ++srv->running;
      srv->peak_running = std::max(srv->peak_running, srv->running);
    }
    qtx_status st = QTX_E_CUDA;
    std::string err = "server worker could not create its context or stream";
    if (ok) {
      st = qtx_transport_solve(ctx, &req->p, &req->o, req->precision, req->flags, stream);
      if (st != QTX_OK) err = qtx_last_error(ctx);
      if (cudaStreamSynchronize(stream) != cudaSuccess && st == QTX_OK) {
        st = QTX_E_CUDA;
        err = cudaGetErrorString(cudaGetLastError());
      }
    }
    const double lat = std::chrono::duration<double>(Clock::now() - req->submitted).count();
    {
      std::lock_guard<std::mutex> lk(srv->m);
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
      srv->in_use -= req->footprint;
      --srv->running;
      srv->completed_uncollected.push_back(req->id);
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
  return QTX_OK;
}

}  // extern "C"
