// Serving loop: asynchronous :gradepro requests with continuous batching on one GPU.
//
// Requests queue on the context.  Each lane is a worker thread with its own context
// (device buffers), its own non-blocking stream and its own waves: when a lane is free
// it takes the queued requests in arrival order while their estimated device footprint
// fits the lane's memory budget (always at least one), and runs them as one
// pkde_gradepro_estimate_batch call.  Lanes run side by side, so a wave that starts
// while another lane's wave is on the GPU overlaps with it on the device.  The state of
// a request (samples, spectra, convergence state, outputs) stays in the lane's device
// buffers from binning to the last bandwidth step.  No counterpart in the reference.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>

#include "pkde_internal.cuh"

namespace pkde {
namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Pending {
  uint64_t ticket;
  pkde_request req;
  size_t footprint;
  double t_submit;
};

std::mutex g_start_mu;  // serialises the lazy start of a context's server

struct Server {
  pkde_ctx *owner = nullptr;
  size_t lane_bytes = 0;
  std::vector<pkde_ctx *> lane_ctx;
  std::vector<cudaStream_t> lane_stream;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Pending> queue;
  std::unordered_map<uint64_t, pkde_result> done;
  std::unordered_set<uint64_t> open;  // submitted and not yet collected by pkde_wait
  uint64_t next_ticket = 1;
  bool stop = false;
};

// Upper bound of the device memory one request needs inside a wave: samples, indices,
// outputs, paired spectra, convergence state, factor tables, binning scratch, 1-D
// per-step arrays and the step engine's ring slots and counters.
size_t footprint(const pkde_gradepro_params *p, int64_t n, bool has_idx) {
  const int N = p->grid.ndim;
  int64_t G = 1, axes = 0;
  for (int j = 0; j < N; ++j) {
    G *= p->grid.dims[j];
    axes += p->grid.dims[j];
  }
  const int64_t B = p->n_bootstraps, P = (B + 1) / 2;
  const int64_t S = p->n_steps > 0 ? (int64_t)p->n_steps + 1 : 1001;  // bw_step ladders: a generous bound
  const int64_t nc = int64_t(1) << N;
  size_t b = 0;
  b += sizeof(double) * N * n + (has_idx ? sizeof(int32_t) * n * B : 0) + 12 * (size_t)G;  // in/out
  b += sizeof(double2) * (2 * P + 1) * G;                                                 // spectra
  b += 64 * (size_t)G;                                                                    // state
  b += sizeof(double) * 2 * S * axes;                                                     // tables
  b += 4 * n + 8 * N * n + 32 * nc * n + 4 * (B + 1) * G;                                 // binning
  b += sizeof(double2) * (2 * P + 1) * G;  // low parts of the fixed-point sums
  b += 4 * B * n + 8 * n + 8 * (size_t)G;  // draws per sample, cell order, cell starts
  if (N == 1) b += sizeof(double) * 2 * S * G;                                            // 1-D steps
  const size_t slot = std::max<size_t>(32u << 20, sizeof(double2) * 2 * (size_t)G);
  b += 8 * slot + 32 * (size_t)G + sizeof(int) * (size_t)S * (P + 1) * (N + G / 16 + 1);  // engine
  return b + (4u << 20);
}

void lane_main(Server *S, int li) {
  cudaSetDevice(S->owner->device);
  pkde_ctx *ctx = S->lane_ctx[li];
  cudaStream_t st = S->lane_stream[li];
  for (;;) {
    std::vector<Pending> wave;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
      if (S->queue.empty()) return;  // stopping and drained
      size_t sum = 0;
      while (!S->queue.empty() && wave.size() < 65535) {
        const Pending &p = S->queue.front();
        if (!wave.empty() && sum + p.footprint > S->lane_bytes) break;
        sum += p.footprint;
        wave.push_back(p);
        S->queue.pop_front();
      }
    }
    const double t_start = now_ms();
    const int count = (int)wave.size();
    std::vector<pkde_gradepro_params> params(count);
    std::vector<const double *> data(count);
    std::vector<int64_t> n(count);
    std::vector<const int32_t *> idx(count);
    std::vector<uint64_t> seeds(count);
    std::vector<double *> dens(count);
    std::vector<int32_t *> sel(count);
    for (int e = 0; e < count; ++e) {
      const pkde_request &r = wave[e].req;
      params[e] = r.params;
      data[e] = r.data;
      n[e] = r.n;
      idx[e] = r.boot_idx;
      seeds[e] = r.seed;
      dens[e] = r.density_out;
      sel[e] = r.selected_out;
    }
    std::vector<int> status(count, PKDE_OK);
    std::vector<std::string> msg(count);
    int rc = pkde_gradepro_estimate_batch(ctx, count, params.data(), data.data(), n.data(), idx.data(), seeds.data(),
                                          dens.data(), sel.data(), 0, st);
    if (rc != PKDE_OK && count > 1) {
      // attribute the failure: run every request of the wave alone
      for (int e = 0; e < count; ++e) {
        status[e] = pkde_gradepro_estimate(ctx, &params[e], data[e], n[e], idx[e], seeds[e], dens[e], sel[e], 0, st);
        if (status[e] != PKDE_OK) msg[e] = pkde_last_error(ctx);
      }
    } else if (rc != PKDE_OK) {
      status[0] = rc;
      msg[0] = pkde_last_error(ctx);
    }
    const double t_end = now_ms();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (int e = 0; e < count; ++e) {
        pkde_result res{};
        res.status = status[e];
        res.batch_size = count;
        res.queue_ms = t_start - wave[e].t_submit;
        res.run_ms = t_end - t_start;
        res.total_ms = t_end - wave[e].t_submit;
        std::strncpy(res.message, msg[e].c_str(), sizeof(res.message) - 1);
        S->done[wave[e].ticket] = res;
      }
    }
    S->cv_done.notify_all();
  }
}

Server *start_server(pkde_ctx *ctx) {
  Server *S = new Server();
  S->owner = ctx;
  const int lanes = ctx->serve_lanes;
  size_t freeb = 0, totalb = 0;
  PKDE_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
  S->lane_bytes = ctx->serve_lane_bytes > 0 ? (size_t)ctx->serve_lane_bytes : (size_t)(0.8 * (double)freeb / lanes);
  for (int i = 0; i < lanes; ++i) {
    pkde_ctx *c = nullptr;
    cudaStream_t s = nullptr;
    if (pkde_create(&c, ctx->device) != PKDE_OK || cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      if (c) pkde_destroy(c);
      for (size_t k = 0; k < S->lane_ctx.size(); ++k) {
        cudaStreamDestroy(S->lane_stream[k]);
        pkde_destroy(S->lane_ctx[k]);
      }
      delete S;
      throw Error{PKDE_ECUDA, "serving: cannot create a lane context or stream"};
    }
    c->tune_wide = false;  // the lane's memory budget assumes narrow ring slots
    S->lane_ctx.push_back(c);
    S->lane_stream.push_back(s);
  }
  for (int i = 0; i < lanes; ++i) S->threads.emplace_back(lane_main, S, i);
  return S;
}

}  // namespace

void stop_server(pkde_ctx *ctx) {
  Server *S = (Server *)ctx->server;
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (auto &t : S->threads) t.join();
  for (size_t i = 0; i < S->lane_ctx.size(); ++i) {
    cudaStreamDestroy(S->lane_stream[i]);
    pkde_destroy(S->lane_ctx[i]);
  }
  delete S;
  ctx->server = nullptr;
}

}  // namespace pkde

extern "C" {

int pkde_serve_config(pkde_ctx *ctx, int32_t lanes, int64_t lane_memory_bytes) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    std::lock_guard<std::mutex> lk(g_start_mu);
    if (ctx->server) throw invalid("pkde_serve_config must come before the first pkde_submit");
    if (lanes < 1 || lanes > 8) throw invalid("lanes must be in 1..8 (got %d)", lanes);
    if (lane_memory_bytes < 0) throw invalid("lane memory budget must be >= 0");
    ctx->serve_lanes = lanes;
    ctx->serve_lane_bytes = lane_memory_bytes;
  });
}

int pkde_submit(pkde_ctx *ctx, const pkde_request *req, uint64_t *ticket) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    if (!req || !ticket) throw invalid("request and ticket are required");
    validate_gradepro_params(&req->params, req->n);
    if (!req->data || !req->density_out) throw invalid("data and density_out are required");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    {
      std::lock_guard<std::mutex> lk(g_start_mu);
      if (!ctx->server) ctx->server = start_server(ctx);
    }
    Server *S = (Server *)ctx->server;
    Pending p{0, *req, footprint(&req->params, req->n, req->boot_idx != nullptr), now_ms()};
    {
      std::lock_guard<std::mutex> lk(S->mu);
      p.ticket = S->next_ticket++;
      S->open.insert(p.ticket);
      S->queue.push_back(p);
      *ticket = p.ticket;
    }
    S->cv_work.notify_one();
  });
}

int pkde_wait(pkde_ctx *ctx, uint64_t ticket, int32_t timeout_ms, pkde_result *out) {
  if (!ctx || !out) return PKDE_EINVAL;
  pkde::Server *S;
  {
    std::lock_guard<std::mutex> lk(pkde::g_start_mu);
    S = (pkde::Server *)ctx->server;
  }
  if (!S) {
    pkde::thread_error(ctx) = "unknown ticket";
    return PKDE_EINVAL;
  }
  std::unique_lock<std::mutex> lk(S->mu);
  if (!S->open.count(ticket)) {
    pkde::thread_error(ctx) = "unknown ticket";
    return PKDE_EINVAL;
  }
  auto ready = [&] { return S->done.count(ticket) > 0; };
  if (timeout_ms < 0) {
    S->cv_done.wait(lk, ready);
  } else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return PKDE_ETIMEDOUT;
  }
  *out = S->done[ticket];
  S->done.erase(ticket);
  S->open.erase(ticket);
  return PKDE_OK;
}

}  // extern "C"
