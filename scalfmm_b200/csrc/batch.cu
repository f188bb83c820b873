// Batches of independent FMM problems of uneven size (the batch workload: many problems, orders and heights
// per problem).  The problems are spread over a few worker streams, each driven by its own host thread, so
// that one problem's tree build (which synchronises its stream once) overlaps other problems' passes on the
// GPU.  Each worker keeps one handle per (order, height, box) it has met, so operators are computed once and
// device buffers are reused across calls.  Problems are taken largest first.
#include "common.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

struct b200fmm_batch_context {
  int kernel = 0, precision = 0, device = 0, nstreams = 1;
  struct Worker {
    cudaStream_t stream = nullptr;
    std::map<std::tuple<int, int, double, double, double, double>, b200fmm_handle> handles;
  };
  std::vector<Worker> workers;
  double last_ms = 0.0;
};

namespace {

b200fmm_status run_problem(b200fmm_batch_context &b, b200fmm_batch_context::Worker &w, const b200fmm_problem &p) {
  const auto key = std::make_tuple(p.order, p.height, p.box_width, p.center[0], p.center[1], p.center[2]);
  auto it = w.handles.find(key);
  if (it == w.handles.end()) {
    b200fmm_config cfg{};
    cfg.kernel = b.kernel;
    cfg.order = p.order;
    cfg.height = p.height;
    cfg.nrhs = 1;
    cfg.precision = b.precision;
    cfg.box_width = p.box_width;
    for (int d = 0; d < 3; ++d) cfg.center[d] = p.center[d];
    cfg.epsilon = -1.0;
    cfg.stream = w.stream;
    cfg.device = b.device;
    b200fmm_handle h = nullptr;
    const b200fmm_status st = b200fmm_create(&cfg, &h);
    if (st != B200FMM_OK) return st;
    it = w.handles.emplace(key, h).first;
  }
  b200fmm_handle h = it->second;
  b200fmm_status st = b200fmm_set_particles(h, p.n, p.x, p.y, p.z, p.q, 0);
  if (st == B200FMM_OK) st = b200fmm_execute(h, B200FMM_ALL);
  if (st == B200FMM_OK) st = b200fmm_get_results(h, p.phi, p.fx, p.fy, p.fz, 0);
  return st;
}

}  // namespace

extern "C" {

b200fmm_status b200fmm_batch_create(int kernel, int precision, int nstreams, int device, b200fmm_batch *out) {
  using namespace b200;
  if (!out) return fail(B200FMM_ERR_INVALID, "batch_create: null output");
  *out = nullptr;
  if (kernel < B200FMM_CHEB_SYM || kernel > B200FMM_LAGRANGE) return fail(B200FMM_ERR_INVALID, "batch_create: kernel");
  if (precision != B200FMM_FP64 && precision != B200FMM_MIXED)
    return fail(B200FMM_ERR_INVALID, "batch_create: precision");
  if (nstreams < 1 || nstreams > 64) return fail(B200FMM_ERR_INVALID, "batch_create: nstreams must be in [1, 64]");
  if (device < 0) B200_CUDA(cudaGetDevice(&device));
  B200_CUDA(cudaSetDevice(device));
  auto *b = new (std::nothrow) b200fmm_batch_context;
  if (!b) return fail(B200FMM_ERR_OOM, "batch_create: host allocation");
  b->kernel = kernel;
  b->precision = precision;
  b->device = device;
  b->nstreams = nstreams;
  b->workers.resize(nstreams);
  for (auto &w : b->workers) {
    if (cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      b200fmm_batch_destroy(b);
      return fail(B200FMM_ERR_CUDA, "batch_create: stream creation failed");
    }
  }
  *out = b;
  return B200FMM_OK;
}

b200fmm_status b200fmm_batch_destroy(b200fmm_batch b) {
  if (!b) return B200FMM_OK;
  cudaSetDevice(b->device);
  for (auto &w : b->workers) {
    for (auto &kv : w.handles) b200fmm_destroy(kv.second);
    if (w.stream) cudaStreamDestroy(w.stream);
  }
  delete b;
  return B200FMM_OK;
}

b200fmm_status b200fmm_batch_execute(b200fmm_batch b, int nproblems, const b200fmm_problem *problems) {
  using namespace b200;
  if (!b) return fail(B200FMM_ERR_INVALID, "batch_execute: null batch");
  if (nproblems < 0 || (nproblems > 0 && !problems)) return fail(B200FMM_ERR_INVALID, "batch_execute: problems");
  for (int i = 0; i < nproblems; ++i) {
    const b200fmm_problem &p = problems[i];
    if (p.n < 1 || !p.x || !p.y || !p.z || !p.q || !p.phi || !p.fx || !p.fy || !p.fz)
      return fail(B200FMM_ERR_INVALID, "batch_execute: problem " + std::to_string(i) + " has a bad size or pointer");
  }
  // largest first, so that the last problems to start are the small ones
  std::vector<int> order(nproblems);
  for (int i = 0; i < nproblems; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return problems[a].n > problems[c].n; });
  std::atomic<int> next{0};
  std::atomic<bool> failed{false};
  std::mutex mu;
  b200fmm_status first = B200FMM_OK;
  std::string first_msg;
  const auto t0 = std::chrono::steady_clock::now();
  auto work = [&](int wi) {
    cudaSetDevice(b->device);
    for (;;) {
      if (failed.load()) return;
      const int k = next.fetch_add(1);
      if (k >= nproblems) return;
      const b200fmm_status st = run_problem(*b, b->workers[wi], problems[order[k]]);
      if (st != B200FMM_OK) {
        std::lock_guard<std::mutex> g(mu);
        if (first == B200FMM_OK) {
          first = st;
          first_msg = "batch_execute: problem " + std::to_string(order[k]) + ": " + b200fmm_last_error();
        }
        failed.store(true);
        return;
      }
    }
  };
  const int nw = std::min(b->nstreams, std::max(nproblems, 1));
  std::vector<std::thread> threads;
  for (int wi = 1; wi < nw; ++wi) threads.emplace_back(work, wi);
  work(0);
  for (auto &t : threads) t.join();
  b->last_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (first != B200FMM_OK) return fail(first, first_msg);
  return B200FMM_OK;
}

b200fmm_status b200fmm_batch_last_time(b200fmm_batch b, double *ms) {
  using namespace b200;
  if (!b || !ms) return fail(B200FMM_ERR_INVALID, "batch_last_time: null argument");
  *ms = b->last_ms;
  return B200FMM_OK;
}

}  // extern "C"
