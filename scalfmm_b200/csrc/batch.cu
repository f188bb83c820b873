// Batches of independent FMM problems of uneven size (the batch workload: many problems, orders and heights
// per problem).  The problems are spread over a few worker streams, each driven by its own host thread, so
// that one problem's tree build (which synchronises its stream once) overlaps other problems' passes on the
// GPU.  Each worker keeps one handle per (order, height, box) it has met, so operators are computed once and
// device buffers are reused across calls.
//
// The schedule is static: the problems are dealt to the workers by estimated cost, largest first, each to
// the least loaded worker (LPT), and each worker runs its own in that order.  The same problem list therefore
// gives every worker the same problems on every call, so a second call finds all its handles created and all
// their buffers large enough: no handle creation (operator precomputation) and no device allocation, both of
// which synchronise the device, happen inside it.  (A shared queue would hand a problem to whichever worker is
// free, which differs from call to call and made the batch time vary by several times.)
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
  cudaEvent_t ev_start = nullptr;          // recorded before any worker starts
  std::vector<cudaEvent_t> ev_end;         // after each worker's last problem
  double last_ms = 0.0, last_device_ms = 0.0;
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
  b->ev_end.assign(nstreams, nullptr);
  bool ev_ok = cudaEventCreate(&b->ev_start) == cudaSuccess;
  for (auto &e : b->ev_end) ev_ok = ev_ok && cudaEventCreate(&e) == cudaSuccess;
  if (!ev_ok) {
    cudaGetLastError();
    b200fmm_batch_destroy(b);
    return fail(B200FMM_ERR_CUDA, "batch_create: event creation failed");
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
  if (b->ev_start) cudaEventDestroy(b->ev_start);
  for (auto e : b->ev_end)
    if (e) cudaEventDestroy(e);
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
  // static LPT schedule over an estimated cost: the near field and the per-particle operators grow with n,
  // the far field with the cells (about n / 30) times p^3; a fixed part stands for a problem's launches and
  // host synchronisations
  const int nw = std::min(b->nstreams, std::max(nproblems, 1));
  auto cost = [&](int i) {
    const double p3 = (double)problems[i].order * problems[i].order * problems[i].order;
    return (double)problems[i].n * (1.0 + p3 / 125.0) + 1.0e5;
  };
  std::vector<int> order(nproblems);
  for (int i = 0; i < nproblems; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return cost(a) > cost(c); });
  std::vector<std::vector<int>> plan(nw);
  std::vector<double> load(nw, 0.0);
  for (int i : order) {
    const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    plan[w].push_back(i);
    load[w] += cost(i);
  }
  std::atomic<bool> failed{false};
  std::mutex mu;
  b200fmm_status first = B200FMM_OK;
  std::string first_msg;
  const auto t0 = std::chrono::steady_clock::now();
  B200_CUDA(cudaSetDevice(b->device));
  B200_CUDA(cudaEventRecord(b->ev_start, b->workers[0].stream));
  auto work = [&](int wi) {
    cudaSetDevice(b->device);
    for (int i : plan[wi]) {
      if (failed.load()) break;
      const b200fmm_status st = run_problem(*b, b->workers[wi], problems[i]);
      if (st != B200FMM_OK) {
        std::lock_guard<std::mutex> g(mu);
        if (first == B200FMM_OK) {
          first = st;
          first_msg = "batch_execute: problem " + std::to_string(i) + ": " + b200fmm_last_error();
        }
        failed.store(true);
        break;
      }
    }
    cudaEventRecord(b->ev_end[wi], b->workers[wi].stream);
  };
  std::vector<std::thread> threads;
  for (int wi = 1; wi < nw; ++wi) threads.emplace_back(work, wi);
  work(0);
  for (auto &t : threads) t.join();
  b->last_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  // device span: from the start event to the last worker's end event
  double dev = 0.0;
  for (int wi = 0; wi < nw; ++wi) {
    float t = 0.f;
    if (cudaEventSynchronize(b->ev_end[wi]) == cudaSuccess &&
        cudaEventElapsedTime(&t, b->ev_start, b->ev_end[wi]) == cudaSuccess)
      dev = std::max(dev, (double)t);
  }
  cudaGetLastError();
  b->last_device_ms = dev;
  if (first != B200FMM_OK) return fail(first, first_msg);
  return B200FMM_OK;
}

b200fmm_status b200fmm_batch_last_time(b200fmm_batch b, double *ms) {
  using namespace b200;
  if (!b || !ms) return fail(B200FMM_ERR_INVALID, "batch_last_time: null argument");
  *ms = b->last_ms;
  return B200FMM_OK;
}

b200fmm_status b200fmm_batch_last_device_time(b200fmm_batch b, double *ms) {
  using namespace b200;
  if (!b || !ms) return fail(B200FMM_ERR_INVALID, "batch_last_device_time: null argument");
  *ms = b->last_device_ms;
  return B200FMM_OK;
}

}  // extern "C"
