// The C ABI of include/b200fmm.h: handle lifecycle, particle insertion, the algorithm driver and the
// level-batched operators.  The driver follows FFmmAlgorithmThread::executeCore
// (Src/Core/FFmmAlgorithmThread.hpp:118-159): bottom pass (P2M), upward pass (M2M, levels height-2..2),
// transfer pass (M2L, levels 2..height-1), downward pass (L2L, parents at levels 2..height-2), direct
// pass (L2P + P2P).
#include "common.cuh"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

namespace b200 {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

b200fmm_status fail(b200fmm_status st, const std::string &msg) {
  g_last_error = msg;
  return st;
}

b200fmm_status ensure_scratch(Context &c, size_t bytes) {
  if (c.scratch_bytes >= bytes) return B200FMM_OK;
  if (c.d_scratch) cudaFree(c.d_scratch);
  c.d_scratch = nullptr;
  c.scratch_bytes = 0;
  B200_CUDA(cudaMalloc(&c.d_scratch, bytes));
  c.scratch_bytes = bytes;
  return B200FMM_OK;
}

b200fmm_status check_status(Context &c) {
  int st[4] = {0, 0, 0, 0};
  B200_CUDA(cudaMemcpyAsync(st, c.d_status, sizeof(st), cudaMemcpyDeviceToHost, c.stream));
  B200_CUDA(cudaStreamSynchronize(c.stream));
  if (st[0] || st[1] || st[2] || st[3]) {
    cudaMemsetAsync(c.d_status, 0, sizeof(st), c.stream);
    return fail(B200FMM_ERR_CUDA, std::string("a device wait ran out of its iteration budget (") +
                                      (st[0] ? "P2P" : st[1] ? "M2L" : "kernel") + ")");
  }
  return B200FMM_OK;
}

namespace {

// counts: [0] M2L pairs (existing interaction-list entries), [1] ordered P2P pairs
__global__ void count_m2l_pairs(long long ncells, const int *__restrict__ ilist, unsigned long long *__restrict__ out) {
  unsigned long long n = 0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ncells * 189;
       e += (long long)gridDim.x * blockDim.x)
    n += ilist[e] >= 0;
  atomicAdd(out, n);
}
// Sum over the interaction pairs of the rank of their slot (rank_of[child type][entry]) and the number of cells
// of each child type.
struct RankTable {
  int r[8][189];
};
__global__ void count_m2l_ranks(long long ncells, const long long *__restrict__ keys, const int *__restrict__ ilist,
                                const __grid_constant__ RankTable T, unsigned long long *__restrict__ out) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= ncells) return;
  const int ct = (int)(keys[cell] & 7);
  unsigned long long s = 0;
  for (int e = 0; e < 189; ++e) s += ilist[cell * 189 + e] >= 0 ? (unsigned long long)T.r[ct][e] : 0ull;
  atomicAdd(out, s);
  atomicAdd(out + 1 + ct, 1ull);
}
__global__ void count_p2p_pairs(long long nleaves, const long long *__restrict__ start, const int *__restrict__ nbr,
                                unsigned long long *__restrict__ out) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= nleaves) return;
  const long long nt = start[c + 1] - start[c];
  long long ns = 0;
  for (int e = 0; e < 27; ++e) {
    const int s = nbr[c * 27 + e];
    if (s >= 0) ns += start[s + 1] - start[s];
  }
  atomicAdd(out + 1, (unsigned long long)(nt * ns - nt));
}

__global__ void scatter_to_original(long long n, int R, const long long *__restrict__ perm,
                                    const double *__restrict__ a, const double *__restrict__ b,
                                    const double *__restrict__ c, const double *__restrict__ d, double *__restrict__ oa,
                                    double *__restrict__ ob, double *__restrict__ oc, double *__restrict__ od) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long j = perm[i];
  for (int r = 0; r < R; ++r) {
    const long long s = (long long)r * n + i, t = (long long)r * n + j;
    if (oa) oa[t] = a[s];
    if (ob) ob[t] = b[s];
    if (oc) oc[t] = c[s];
    if (od) od[t] = d[s];
  }
}

b200fmm_status check_handle(b200fmm_handle h) {
  if (!h) return fail(B200FMM_ERR_INVALID, "null handle");
  return B200FMM_OK;
}

b200fmm_status set_device(Context &c) {
  B200_CUDA(cudaSetDevice(c.device));
  return B200FMM_OK;
}

b200fmm_status need_particles(Context &c) {
  if (!c.has_particles) return fail(B200FMM_ERR_STATE, "no particles: call b200fmm_set_particles first");
  return B200FMM_OK;
}

b200fmm_status zero_state(Context &c) {
  for (int l = 2; l < c.H; ++l) {
    const size_t bytes = sizeof(double) * (size_t)c.lv[l].n * c.R * c.nn;
    if (bytes) {
      B200_CUDA(cudaMemsetAsync(c.lv[l].M, 0, bytes, c.stream));
      B200_CUDA(cudaMemsetAsync(c.lv[l].L, 0, bytes, c.stream));
    }
  }
  const size_t pb = sizeof(double) * (size_t)c.N * c.R;
  for (double *p : {c.d_phi, c.d_fx, c.d_fy, c.d_fz}) B200_CUDA(cudaMemsetAsync(p, 0, pb, c.stream));
  return B200FMM_OK;
}

b200fmm_status record(Context &c, int k) {
  B200_CUDA(record_event(c, k));
  return B200FMM_OK;
}

void drop_graph(Context &c) {
  if (c.graph) cudaGraphExecDestroy(c.graph);
  c.graph = nullptr;
  c.graph_serial = -1;
}

b200fmm_status run_m2l(Context &c, int level) {
  if (c.cfg.precision == B200FMM_MIXED) return run_m2l_tc(c, level);
  B200_CHECK(build_ilists(c));  // built with the tree in FP64: a no-op
  return run_m2l_fp64(c, level);
}

void destroy_context(b200fmm_context *c) {
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->stream_out) cudaStreamSynchronize(c->stream_out);
  if (c->stream_in) cudaStreamSynchronize(c->stream_in);
  drop_graph(*c);
  free_tree(*c);
  tc_free(*c);
  sym64_free(*c);
  for (void *p : {(void *)c->d_roots, (void *)c->d_S, (void *)c->d_pindices, (void *)c->d_pvec,
                  (void *)c->d_symU, (void *)c->d_symV, (void *)c->d_symoff, (void *)c->d_symrank,
                  (void *)c->d_dense, (void *)c->d_itab, (void *)c->d_class_order, (void *)c->d_cls_bounds,
                  (void *)c->d_cls_slots, (void *)c->d_status, (void *)c->d_mmax, (void *)c->d_Ut, (void *)c->d_Vt,
                  (void *)c->d_toff, (void *)c->d_trank, c->d_scratch, (void *)c->d_out, (void *)c->d_shard})
    if (p) cudaFree(p);
  if (c->events_ready)
    for (auto &e : c->ev) cudaEventDestroy(e);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  if (c->stream2) cudaStreamDestroy(c->stream2);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->stream_out) cudaStreamDestroy(c->stream_out);
  if (c->ev_scat) cudaEventDestroy(c->ev_scat);
  if (c->ev_out) cudaEventDestroy(c->ev_out);
  if (c->stream_in) cudaStreamDestroy(c->stream_in);
  for (cudaEvent_t e : {c->ev_in_xyz, c->ev_in_q, c->ev_stage_free})
    if (e) cudaEventDestroy(e);
  delete c;
}

}  // namespace
}  // namespace b200

using namespace b200;

extern "C" {

const char *b200fmm_last_error(void) { return g_last_error.c_str(); }

const char *b200fmm_version(void) { return "b200fmm 0.1 (sm_100a)"; }

b200fmm_status b200fmm_create(const b200fmm_config *cfg, b200fmm_handle *out) {
  if (!cfg || !out) return fail(B200FMM_ERR_INVALID, "null argument");
  *out = nullptr;
  if (cfg->kernel < 0 || cfg->kernel > 2) return fail(B200FMM_ERR_INVALID, "unknown kernel");
  if (cfg->order < 3 || cfg->order > kMaxOrder) return fail(B200FMM_ERR_INVALID, "order must be in [3, 8]");
  if (cfg->height < 3 || cfg->height > kMaxHeight) return fail(B200FMM_ERR_INVALID, "height must be in [3, 12]");
  if (cfg->nrhs < 1 || cfg->nrhs > kMaxNrhs) return fail(B200FMM_ERR_INVALID, "nrhs must be in [1, 32]");
  if (cfg->precision != B200FMM_FP64 && cfg->precision != B200FMM_MIXED)
    return fail(B200FMM_ERR_INVALID, "unknown precision");
  if (!(cfg->box_width > 0) || !std::isfinite(cfg->box_width)) return fail(B200FMM_ERR_INVALID, "bad box width");
  for (int d = 0; d < 3; ++d)
    if (!std::isfinite(cfg->center[d])) return fail(B200FMM_ERR_INVALID, "bad box centre");
  b200fmm_context *c = new (std::nothrow) b200fmm_context();
  if (!c) return fail(B200FMM_ERR_OOM, "host allocation failed");
  c->cfg = *cfg;
  c->p = cfg->order;
  c->nn = c->p * c->p * c->p;
  c->H = cfg->height;
  c->R = cfg->nrhs;
  if (cfg->device >= 0) {
    c->device = cfg->device;
  } else if (cudaGetDevice(&c->device) != cudaSuccess) {
    delete c;
    return fail(B200FMM_ERR_CUDA, "no CUDA device");
  }
  b200fmm_status st = set_device(*c);
  if (st == B200FMM_OK) {
    if (cfg->stream) {
      c->stream = (cudaStream_t)cfg->stream;
    } else {
      if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        st = fail(B200FMM_ERR_CUDA, "stream creation failed");
      c->own_stream = true;
    }
  }
  if (st == B200FMM_OK) {
    if (cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream_out, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_scat, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_out, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream_in, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_in_xyz, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_in_q, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_stage_free, cudaEventDisableTiming) != cudaSuccess)
      st = fail(B200FMM_ERR_CUDA, "stream creation failed");
  }
  if (st == B200FMM_OK) {
    bool ok = true;
    for (auto &e : c->ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
    c->events_ready = ok;
    if (!ok) st = fail(B200FMM_ERR_CUDA, "event creation failed");
  }
  if (st == B200FMM_OK) {
    if (cudaMalloc(&c->d_status, 16 * sizeof(int)) != cudaSuccess ||
        cudaMemset(c->d_status, 0, 16 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->d_shard, sizeof(long long) * (2 + 2 * kMaxHeight)) != cudaSuccess ||
        cudaMalloc(&c->d_mmax, sizeof(unsigned long long) * kMaxHeight * kMmaxSlots) != cudaSuccess)
      st = fail(B200FMM_ERR_OOM, "status allocation failed");
  }
  if (st == B200FMM_OK) st = build_tables(*c);
  if (st == B200FMM_OK && cfg->kernel == B200FMM_CHEB_SYM) {
    // the compressed operators: applied in FP64, or in their low-rank tensor-core form (MIXED)
    st = compress_sym_operators(*c);
    if (st == B200FMM_OK && cfg->precision == B200FMM_FP64) st = upload_sym_operators(*c);
  }
  if (st == B200FMM_OK && cfg->kernel != B200FMM_CHEB_SYM && cfg->precision == B200FMM_FP64)
    st = build_dense_operators(*c);
  if (st == B200FMM_OK && cfg->precision == B200FMM_MIXED) st = tc_init(*c);
  if (st != B200FMM_OK) {
    destroy_context(c);
    return st;
  }
  *out = c;
  return B200FMM_OK;
}

b200fmm_status b200fmm_destroy(b200fmm_handle h) {
  if (!h) return B200FMM_OK;
  destroy_context(h);
  return B200FMM_OK;
}

b200fmm_status b200fmm_set_sym_operators(b200fmm_handle h, const int *ranks, const double *uv, long long uv_len) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  if (c.cfg.kernel != B200FMM_CHEB_SYM || c.cfg.precision != B200FMM_FP64)
    return fail(B200FMM_ERR_STATE, "symmetric operators apply to the FP64 CHEB_SYM kernel only");
  drop_graph(c);  // a captured execute() holds the old operator buffers
  c.eager_serial = -1;
  if (!ranks || !uv) return fail(B200FMM_ERR_INVALID, "null argument");
  long long need = 0;
  int nclass = 0;
  for (int t = 0; t < 343; ++t) {
    if (ranks[t] < 0 || ranks[t] > c.nn) return fail(B200FMM_ERR_INVALID, "rank out of range");
    if (ranks[t] > 0) ++nclass;
    need += 2LL * ranks[t] * c.nn;
  }
  if (nclass != 16) return fail(B200FMM_ERR_INVALID, "expected operators for exactly 16 class slots");
  if (uv_len != need) return fail(B200FMM_ERR_INVALID, "uv length does not match the ranks");
  B200_CHECK(set_device(c));
  c.sym_ranks.assign(ranks, ranks + 343);
  c.sym_uv.assign(uv, uv + need);
  return upload_sym_operators(c);
}

b200fmm_status b200fmm_get_sym_operators(b200fmm_handle h, int *ranks, double *uv, long long uv_cap,
                                         long long *uv_len) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  if (c.sym_ranks.empty()) return fail(B200FMM_ERR_STATE, "this handle has no symmetric operators");
  if (uv_len) *uv_len = (long long)c.sym_uv.size();
  if (ranks) std::memcpy(ranks, c.sym_ranks.data(), sizeof(int) * 343);
  if (uv) {
    if (uv_cap < (long long)c.sym_uv.size()) return fail(B200FMM_ERR_INVALID, "uv buffer too small");
    std::memcpy(uv, c.sym_uv.data(), sizeof(double) * c.sym_uv.size());
  }
  return B200FMM_OK;
}

b200fmm_status b200fmm_set_particles(b200fmm_handle h, long long n, const double *x, const double *y,
                                     const double *z, const double *q, int on_device) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  if (n < 1 || n > 2000000000LL) return fail(B200FMM_ERR_INVALID, "particle count must be in [1, 2e9]");
  if (!x || !y || !z || !q) return fail(B200FMM_ERR_INVALID, "null particle array");
  B200_CHECK(set_device(c));
  c.has_particles = false;
  c.N = n;
  ++c.tree_serial;
  drop_graph(c);
  B200_CUDA(cudaEventRecord(c.ev[14], c.stream));
  b200fmm_status st = build_tree(c, x, y, z, q, on_device != 0);
  if (st != B200FMM_OK) return st;
  B200_CHECK(zero_state(c));  // a new tree starts from zero expansions and results
  c.state_zero = true;
  B200_CUDA(cudaEventRecord(c.ev[15], c.stream));
  B200_CUDA(cudaEventSynchronize(c.ev[15]));
  float ms = 0;
  cudaEventElapsedTime(&ms, c.ev[14], c.ev[15]);
  c.ms[0] = ms;
  c.has_particles = true;
  return B200FMM_OK;
}

b200fmm_status b200fmm_set_charges(b200fmm_handle h, const double *q, int on_device) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  if (!q) return fail(B200FMM_ERR_INVALID, "null charges");
  B200_CHECK(set_device(c));
  return upload_charges(c, q, on_device != 0);
}

b200fmm_status b200fmm_reset_expansions(b200fmm_handle h) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  B200_CHECK(set_device(c));
  B200_CHECK(zero_state(c));
  c.state_zero = true;
  return B200FMM_OK;
}

b200fmm_status b200fmm_zero_results(b200fmm_handle h) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  B200_CHECK(set_device(c));
  const size_t pb = sizeof(double) * (size_t)c.N * c.R;
  for (double *p : {c.d_phi, c.d_fx, c.d_fy, c.d_fz}) B200_CUDA(cudaMemsetAsync(p, 0, pb, c.stream));
  return B200FMM_OK;
}

// The passes of execute(), in the reference's order (FFmmAlgorithmThread::executeCore).
static b200fmm_status execute_body(Context &c, unsigned ops) {
  // per-tree tables (the shard's ranges, the tensor-core M2L's tables, which take a host synchronisation) are
  // built by an eager evaluation, never inside a capture: a capture that finds them pending gives up before it
  // changes any state, and the caller's evaluation runs eagerly
  if (c.capturing && ((c.shard_count > 1 && c.shard_serial != c.tree_serial) ||
                      (c.cfg.precision == B200FMM_MIXED && (ops & B200FMM_M2L) && tc_tables_pending(c))))
    return fail(B200FMM_ERR_STATE, "per-tree tables pending: the evaluation is not captured");
  c.launches = 0;
  const int LL = c.H - 1;
  B200_CHECK(record(c, 0));
  // skipped right after set_particles, which zeroed them; always part of a captured graph
  if (!c.state_zero || c.capturing) B200_CHECK(zero_state(c));
  c.state_zero = false;
  // MIXED records the multipole maxima during a full upward pass for the tensor-core M2L
  c.mmax_out = nullptr;
  c.mmax_ready = false;
  const bool fuse_max = c.cfg.precision == B200FMM_MIXED && (ops & B200FMM_P2M) && (ops & B200FMM_M2M) &&
                        (ops & B200FMM_M2L);
  if (fuse_max) {
    B200_CUDA(cudaMemsetAsync(c.d_mmax, 0, sizeof(unsigned long long) * kMaxHeight * kMmaxSlots, c.stream));
    c.mmax_out = c.d_mmax;
  }
  B200_CHECK(record(c, 1));
  // a target shard: the leaf and cell ranges of this tree, read by the near field, L2P and the M2L's units
  const long long *shard = nullptr;
  if (c.shard_count > 1) {
    if (c.shard_serial != c.tree_serial) B200_CHECK(shard_ranges(c));
    shard = c.d_shard;
  }
  // The near field needs only the tree: it runs on the second stream beside P2M and M2M and joins before the
  // M2L (a persistent kernel that wants every SM) and before L2P adds into the same results.
  const bool overlap = (ops & B200FMM_P2P) && (ops & (B200FMM_P2M | B200FMM_M2M));
  c.p2p_overlapped = overlap;
  if (overlap) {
    B200_CUDA(cudaEventRecord(c.ev_fork, c.stream));
    B200_CUDA(cudaStreamWaitEvent(c.stream2, c.ev_fork, 0));
    cudaStream_t main = c.stream;
    c.stream = c.stream2;
    b200fmm_status st = record(c, 12);
    if (st == B200FMM_OK) st = run_p2p(c, 0, shard);
    if (st == B200FMM_OK) st = record(c, 13);
    if (st == B200FMM_OK && cudaEventRecord(c.ev_join, c.stream2) != cudaSuccess)
      st = fail(B200FMM_ERR_CUDA, "event record failed");
    c.stream = main;
    B200_CHECK(st);
  }
  // the tensor-core M2L's per-tree tables (one host synchronisation on compacted levels) while the near field
  // runs on the second stream
  if (c.cfg.precision == B200FMM_MIXED && (ops & B200FMM_M2L)) B200_CHECK(tc_tree_setup(c));
  if (ops & B200FMM_P2M) B200_CHECK(run_p2m(c));
  B200_CHECK(record(c, 2));
  if (ops & B200FMM_M2M)
    for (int l = LL - 1; l >= 2; --l) B200_CHECK(run_m2m(c, l));
  c.mmax_out = nullptr;
  c.mmax_ready = fuse_max;
  B200_CHECK(record(c, 16));
  if (overlap) B200_CUDA(cudaStreamWaitEvent(c.stream, c.ev_join, 0));
  B200_CHECK(record(c, 3));
  if (ops & B200FMM_M2L) {
    b200fmm_status st = B200FMM_OK;
    if (c.cfg.precision == B200FMM_MIXED)
      st = run_m2l_tc(c, -1);  // one launch for every level
    else
      for (int l = 2; l <= LL && st == B200FMM_OK; ++l) st = run_m2l_fp64(c, l);
    c.mmax_ready = false;
    B200_CHECK(st);
  }
  c.mmax_ready = false;
  B200_CHECK(record(c, 4));
  if (ops & B200FMM_L2L)
    for (int l = 2; l <= LL - 1; ++l) B200_CHECK(run_l2l(c, l));
  B200_CHECK(record(c, 5));
  if (ops & B200FMM_L2P) B200_CHECK(run_l2p(c, shard));
  B200_CHECK(record(c, 6));
  if ((ops & B200FMM_P2P) && !overlap) B200_CHECK(run_p2p(c, 0, shard));
  B200_CHECK(record(c, 7));
  return B200FMM_OK;
}

static bool graphs_enabled() {
  const char *e = std::getenv("B200FMM_GRAPHS");
  return !(e && e[0] == '0');
}

// Capture execute_body into c.graph.  On any failure the capture is discarded, the error cleared and the
// tree stays on the eager path.
static void capture_graph(Context &c, unsigned ops) {
  drop_graph(c);
  c.packed32 = false;  // the graph repacks the FP32 near-field copies, which carry the charges
  if (cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    c.eager_ops = ~0u;
    return;
  }
  c.capturing = true;
  const b200fmm_status st = execute_body(c, ops);
  c.capturing = false;
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c.stream, &g);
  cudaGraphExec_t x = nullptr;
  if (st == B200FMM_OK && e == cudaSuccess && g && cudaGraphInstantiate(&x, g, 0) == cudaSuccess) {
    c.graph = x;
    c.graph_serial = c.tree_serial;
    c.graph_ops = ops;
    c.graph_launches = c.launches;
  } else {
    c.eager_ops = ~0u;  // not again for this tree
  }
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
}

b200fmm_status b200fmm_execute(b200fmm_handle h, unsigned ops) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  B200_CHECK(set_device(c));
  // a caller that is itself capturing this stream gets the plain launches in its own graph
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  B200_CUDA(cudaStreamIsCapturing(c.stream, &cs));
  if (graphs_enabled() && cs == cudaStreamCaptureStatusNone && c.eager_serial == c.tree_serial &&
      c.eager_ops == ops) {
    if (!c.graph || c.graph_serial != c.tree_serial || c.graph_ops != ops) capture_graph(c, ops);
    if (c.graph) {
      B200_CUDA(cudaEventRecord(c.ev[0], c.stream));
      B200_CUDA(cudaGraphLaunch(c.graph, c.stream));
      B200_CUDA(cudaEventRecord(c.ev[7], c.stream));
      c.packed32 = true;
      c.state_zero = false;
      c.last_was_graph = true;
      c.launches = c.graph_launches;
      return B200FMM_OK;
    }
  }
  c.last_was_graph = false;
  B200_CHECK(execute_body(c, ops));
  if (c.eager_ops != ~0u || c.eager_serial != c.tree_serial) {
    c.eager_serial = c.tree_serial;
    c.eager_ops = ops;
  }
  return B200FMM_OK;
}

b200fmm_status b200fmm_autotune(b200fmm_handle h, int *splits, double *ms) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  B200_CHECK(set_device(c));
  if (splits) *splits = 0;
  if (ms) *ms = 0;
  if (c.cfg.precision != B200FMM_MIXED || !c.tc) return B200FMM_OK;  // nothing to tune
  drop_graph(c);
  c.eager_serial = -1;
  const int cand[] = {1, 2, 3, 4};  // work ranges per CTA (pair) of the tensor-core M2L
  int best = 0;
  float best_ms = 0.f;
  for (int k : cand) {
    tc_set_splits(c, k);
    float t = 0.f;
    for (int rep = 0; rep < 2; ++rep) {  // the first run rebuilds the work units
      B200_CHECK(execute_body(c, B200FMM_P2M | B200FMM_M2M | B200FMM_M2L));
      B200_CUDA(cudaEventSynchronize(c.ev[7]));
      B200_CHECK(check_status(c));
      if (cudaEventElapsedTime(&t, c.ev[8], c.ev[9]) != cudaSuccess) {
        cudaGetLastError();
        t = 1e30f;
      }
    }
    if (best == 0 || t < best_ms) {
      best = k;
      best_ms = t;
    }
  }
  tc_set_splits(c, best);
  // the near field's work items: the largest leaf taken whole and the size of the pieces of larger leaves,
  // timed on the current tree (the item table is rebuilt with each rule)
  const int rules[][2] = {{64, 32}, {32, 32}, {128, 32}, {64, 16}, {128, 64}, {32, 16}};
  int bw = c.p2p_whole, bi = c.p2p_item;
  float bt = 0.f;
  bool have = false;
  for (const auto &rule : rules) {
    c.p2p_whole = rule[0];
    c.p2p_item = rule[1];
    c.column_serial = -1;
    c.packed32 = false;
    float t = 0.f;
    for (int rep = 0; rep < 2; ++rep) {  // the first run rebuilds the item table
      B200_CHECK(run_p2p(c, 0));
      B200_CUDA(cudaEventSynchronize(c.ev[11]));
      B200_CHECK(check_status(c));
      if (cudaEventElapsedTime(&t, c.ev[10], c.ev[11]) != cudaSuccess) {
        cudaGetLastError();
        t = 1e30f;
      }
    }
    if (!have || t < bt) {
      have = true;
      bt = t;
      bw = rule[0];
      bi = rule[1];
    }
  }
  c.p2p_whole = bw;
  c.p2p_item = bi;
  c.column_serial = -1;
  c.packed32 = false;
  c.state_zero = false;
  if (splits) *splits = best;
  if (ms) *ms = best_ms;
  return B200FMM_OK;
}

b200fmm_status b200fmm_get_tuning(b200fmm_handle h, int *values) {
  B200_CHECK(check_handle(h));
  if (!values) return fail(B200FMM_ERR_INVALID, "null argument");
  Context &c = *h;
  values[0] = c.tc ? tc_splits_used(c) : 0;
  values[1] = c.p2p_whole;
  values[2] = c.p2p_item;
  return B200FMM_OK;
}

b200fmm_status b200fmm_p2m(b200fmm_handle h) {
  B200_CHECK(check_handle(h));
  h->state_zero = false;
  B200_CHECK(need_particles(*h));
  B200_CHECK(set_device(*h));
  return run_p2m(*h);
}

b200fmm_status b200fmm_m2m(b200fmm_handle h, int level) {
  B200_CHECK(check_handle(h));
  h->state_zero = false;
  B200_CHECK(need_particles(*h));
  B200_CHECK(set_device(*h));
  return run_m2m(*h, level);
}

b200fmm_status b200fmm_m2l(b200fmm_handle h, int level) {
  B200_CHECK(check_handle(h));
  h->state_zero = false;
  B200_CHECK(need_particles(*h));
  B200_CHECK(set_device(*h));
  if (level < 2 || level > h->H - 1) return fail(B200FMM_ERR_INVALID, "m2l: level must be in [2, height-1]");
  return run_m2l(*h, level);
}

b200fmm_status b200fmm_l2l(b200fmm_handle h, int level) {
  B200_CHECK(check_handle(h));
  h->state_zero = false;
  B200_CHECK(need_particles(*h));
  B200_CHECK(set_device(*h));
  return run_l2l(*h, level);
}

b200fmm_status b200fmm_l2p(b200fmm_handle h) {
  B200_CHECK(check_handle(h));
  h->state_zero = false;
  B200_CHECK(need_particles(*h));
  B200_CHECK(set_device(*h));
  return run_l2p(*h);
}

b200fmm_status b200fmm_p2p(b200fmm_handle h, int variant) {
  B200_CHECK(check_handle(h));
  h->state_zero = false;
  B200_CHECK(need_particles(*h));
  if (variant != 0 && variant != 1) return fail(B200FMM_ERR_INVALID, "p2p variant must be 0 or 1");
  B200_CHECK(set_device(*h));
  return run_p2p(*h, variant);
}

b200fmm_status b200fmm_get_results(b200fmm_handle h, double *phi, double *fx, double *fy, double *fz,
                                   int on_device) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  B200_CHECK(set_device(c));
  const long long n = c.N;
  const size_t bytes = sizeof(double) * n * c.R;
  if (on_device) {
    scatter_to_original<<<grid_for(n, 256), 256, 0, c.stream>>>(n, c.R, c.d_perm, c.d_phi, c.d_fx, c.d_fy, c.d_fz, phi,
                                                                fx, fy, fz);
    B200_CUDA(cudaGetLastError());
    return B200FMM_OK;
  }
  B200_CHECK(ensure_scratch(c, 4 * bytes + 4096));
  double *o = (double *)((char *)c.d_scratch + 4096);
  scatter_to_original<<<grid_for(n, 256), 256, 0, c.stream>>>(n, c.R, c.d_perm, c.d_phi, c.d_fx, c.d_fy, c.d_fz, o,
                                                              o + n * c.R, o + 2 * n * c.R, o + 3 * n * c.R);
  B200_CUDA(cudaGetLastError());
  double *dst[4] = {phi, fx, fy, fz};
  for (int k = 0; k < 4; ++k)
    if (dst[k]) B200_CUDA(cudaMemcpyAsync(dst[k], o + k * n * c.R, bytes, cudaMemcpyDeviceToHost, c.stream));
  B200_CUDA(cudaStreamSynchronize(c.stream));
  return check_status(c);
}

// Results to the host without waiting: staged in the caller's order on the handle's stream, then copied on a
// stream of their own, so that the copies overlap whatever the caller queues next (the next tree's upload and
// build, in a time-stepping loop).  The staging buffer is rewritten only after the previous copies have read it.
b200fmm_status b200fmm_get_results_async(b200fmm_handle h, double *phi, double *fx, double *fy, double *fz) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  B200_CHECK(set_device(c));
  const long long n = c.N;
  const size_t bytes = sizeof(double) * n * c.R;
  if (c.out_cap < 4 * bytes) {
    B200_CUDA(cudaStreamSynchronize(c.stream_out));
    if (c.d_out) cudaFree(c.d_out);
    c.d_out = nullptr;
    c.out_cap = 0;
    B200_CUDA(cudaMalloc(&c.d_out, 4 * bytes));
    c.out_cap = 4 * bytes;
  }
  double *o = c.d_out;
  B200_CUDA(cudaStreamWaitEvent(c.stream, c.ev_out, 0));
  scatter_to_original<<<grid_for(n, 256), 256, 0, c.stream>>>(n, c.R, c.d_perm, c.d_phi, c.d_fx, c.d_fy, c.d_fz, o,
                                                              o + n * c.R, o + 2 * n * c.R, o + 3 * n * c.R);
  B200_CUDA(cudaGetLastError());
  B200_CUDA(cudaEventRecord(c.ev_scat, c.stream));
  B200_CUDA(cudaStreamWaitEvent(c.stream_out, c.ev_scat, 0));
  double *dst[4] = {phi, fx, fy, fz};
  for (int k = 0; k < 4; ++k)
    if (dst[k]) B200_CUDA(cudaMemcpyAsync(dst[k], o + k * n * c.R, bytes, cudaMemcpyDeviceToHost, c.stream_out));
  B200_CUDA(cudaEventRecord(c.ev_out, c.stream_out));
  return B200FMM_OK;
}

b200fmm_status b200fmm_join_results(b200fmm_handle h) {
  B200_CHECK(check_handle(h));
  B200_CHECK(set_device(*h));
  B200_CUDA(cudaStreamWaitEvent(h->stream, h->ev_out, 0));
  return B200FMM_OK;
}

b200fmm_status b200fmm_set_shard(b200fmm_handle h, int rank, int count) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  if (count < 1 || rank < 0 || rank >= count) return fail(B200FMM_ERR_INVALID, "set_shard: need 0 <= rank < count");
  B200_CHECK(set_device(c));
  if (rank == c.shard_rank && count == c.shard_count) return B200FMM_OK;
  c.shard_rank = count > 1 ? rank : 0;
  c.shard_count = count;
  c.shard_serial = -1;
  drop_graph(c);         // a captured evaluation holds the earlier ranges
  c.eager_serial = -1;   // the next evaluation runs eagerly and rebuilds the per-tree tables
  tc_invalidate_units(c);  // the M2L's units are weighted by the shard
  return B200FMM_OK;
}

b200fmm_status b200fmm_synchronize(b200fmm_handle h) {
  B200_CHECK(check_handle(h));
  B200_CHECK(set_device(*h));
  B200_CUDA(cudaStreamSynchronize(h->stream));
  B200_CUDA(cudaStreamSynchronize(h->stream_out));
  return check_status(*h);
}

b200fmm_status b200fmm_tree_info(b200fmm_handle h, long long *ncells, long long *nparticles) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  if (ncells)
    for (int l = 0; l < c.H; ++l) ncells[l] = c.lv[l].n;
  if (nparticles) *nparticles = c.N;
  return B200FMM_OK;
}

b200fmm_status b200fmm_get_cells(b200fmm_handle h, int level, long long *keys, double *multipoles, double *locals) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  if (level < 0 || level >= c.H) return fail(B200FMM_ERR_INVALID, "level out of range");
  B200_CHECK(set_device(c));
  const Level &L = c.lv[level];
  if (keys) B200_CUDA(cudaMemcpyAsync(keys, L.keys, sizeof(long long) * L.n, cudaMemcpyDeviceToHost, c.stream));
  const size_t bytes = sizeof(double) * (size_t)L.n * c.R * c.nn;
  if (multipoles) {
    if (!L.M) return fail(B200FMM_ERR_INVALID, "no expansions above level 2");
    B200_CUDA(cudaMemcpyAsync(multipoles, L.M, bytes, cudaMemcpyDeviceToHost, c.stream));
  }
  if (locals) {
    if (!L.L) return fail(B200FMM_ERR_INVALID, "no expansions above level 2");
    B200_CUDA(cudaMemcpyAsync(locals, L.L, bytes, cudaMemcpyDeviceToHost, c.stream));
  }
  B200_CUDA(cudaStreamSynchronize(c.stream));
  return B200FMM_OK;
}

b200fmm_status b200fmm_get_permutation(b200fmm_handle h, long long *perm) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  if (!perm) return fail(B200FMM_ERR_INVALID, "null argument");
  B200_CHECK(set_device(c));
  B200_CUDA(cudaMemcpyAsync(perm, c.d_perm, sizeof(long long) * c.N, cudaMemcpyDeviceToHost, c.stream));
  B200_CUDA(cudaStreamSynchronize(c.stream));
  return B200FMM_OK;
}

b200fmm_status b200fmm_get_leaf_neighbors(b200fmm_handle h, int *nbr) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  if (!nbr) return fail(B200FMM_ERR_INVALID, "null argument");
  B200_CHECK(set_device(c));
  const Level &L = c.lv[c.H - 1];
  B200_CUDA(cudaMemcpyAsync(nbr, c.d_leaf_nbr, sizeof(int) * 27 * (size_t)L.n, cudaMemcpyDeviceToHost, c.stream));
  B200_CUDA(cudaStreamSynchronize(c.stream));
  return B200FMM_OK;
}

b200fmm_status b200fmm_get_leaf_ranges(b200fmm_handle h, long long *start) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  if (!start) return fail(B200FMM_ERR_INVALID, "null argument");
  B200_CHECK(set_device(c));
  const Level &L = c.lv[c.H - 1];
  B200_CUDA(cudaMemcpyAsync(start, c.d_leaf_start, sizeof(long long) * ((size_t)L.n + 1), cudaMemcpyDeviceToHost,
                            c.stream));
  B200_CUDA(cudaStreamSynchronize(c.stream));
  return B200FMM_OK;
}

b200fmm_status b200fmm_get_interaction_lists(b200fmm_handle h, int level, int *src, int *pos) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  if (level < 2 || level > c.H - 1) return fail(B200FMM_ERR_INVALID, "level must be in [2, height-1]");
  if (!src && !pos) return fail(B200FMM_ERR_INVALID, "null argument");
  B200_CHECK(set_device(c));
  B200_CHECK(build_ilists(c));  // MIXED builds them on demand only
  const Level &L = c.lv[level];
  std::vector<int> s((size_t)L.n * 189);
  std::vector<long long> keys((size_t)L.n);
  if (L.n) {
    B200_CUDA(cudaMemcpyAsync(s.data(), L.ilist, sizeof(int) * s.size(), cudaMemcpyDeviceToHost, c.stream));
    B200_CUDA(cudaMemcpyAsync(keys.data(), L.keys, sizeof(long long) * keys.size(), cudaMemcpyDeviceToHost,
                              c.stream));
  }
  B200_CUDA(cudaStreamSynchronize(c.stream));
  // entry e of a cell with Morton child index ct sits at position itab.slot[ct][e]
  for (long long i = 0; i < L.n; ++i)
    for (int e = 0; e < 189; ++e) {
      const size_t k = (size_t)i * 189 + e;
      if (src) src[k] = s[k];
      if (pos) pos[k] = s[k] >= 0 ? c.itab.slot[keys[i] & 7][e] : -1;
    }
  return B200FMM_OK;
}

b200fmm_status b200fmm_last_timings(b200fmm_handle h, double *ms8) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  if (!ms8) return fail(B200FMM_ERR_INVALID, "null argument");
  B200_CHECK(set_device(c));
  B200_CUDA(cudaEventSynchronize(c.ev[7]));
  ms8[0] = c.ms[0];
  for (int k = 1; k <= 6; ++k) {
    float t = 0;
    // the concurrent near field has its own events; M2M ends before the main stream waits for it
    const int a = (k == 6 && c.p2p_overlapped) ? 12 : k;
    const int b = (k == 6 && c.p2p_overlapped) ? 13 : k == 2 ? 16 : k + 1;
    if (c.last_was_graph || cudaEventElapsedTime(&t, c.ev[a], c.ev[b]) != cudaSuccess) t = 0;
    ms8[k] = t;
  }
  float tot = 0;
  if (cudaEventElapsedTime(&tot, c.ev[0], c.ev[7]) != cudaSuccess) tot = 0;
  ms8[7] = tot;
  return B200FMM_OK;
}

b200fmm_status b200fmm_last_kernel_times(b200fmm_handle h, double *ms4) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  if (!ms4) return fail(B200FMM_ERR_INVALID, "null argument");
  B200_CHECK(set_device(c));
  B200_CUDA(cudaEventSynchronize(c.ev[7]));
  if (c.last_was_graph) {
    for (int k = 0; k < 4; ++k) ms4[k] = 0;
    return B200FMM_OK;
  }
  float t = 0;
  if (c.cfg.precision == B200FMM_MIXED && cudaEventElapsedTime(&t, c.ev[8], c.ev[9]) == cudaSuccess)
    ms4[0] = t;
  else
    ms4[0] = (cudaEventElapsedTime(&t, c.ev[3], c.ev[4]) == cudaSuccess) ? t : 0;
  ms4[1] = (cudaEventElapsedTime(&t, c.ev[10], c.ev[11]) == cudaSuccess) ? t : 0;
  ms4[2] = (cudaEventElapsedTime(&t, c.ev[1], c.ev[2]) == cudaSuccess) ? t : 0;
  ms4[3] = (cudaEventElapsedTime(&t, c.ev[5], c.ev[6]) == cudaSuccess) ? t : 0;
  cudaGetLastError();
  return B200FMM_OK;
}

b200fmm_status b200fmm_tree_stats(b200fmm_handle h, long long *m2l_pairs, long long *p2p_pairs) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  B200_CHECK(need_particles(c));
  B200_CHECK(set_device(c));
  B200_CHECK(build_ilists(c));
  B200_CHECK(ensure_scratch(c, 4096));
  unsigned long long *d = (unsigned long long *)((char *)c.d_scratch + 2048);
  B200_CUDA(cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), c.stream));
  for (int l = 2; l < c.H; ++l)
    if (c.lv[l].n)
      count_m2l_pairs<<<grid_for(c.lv[l].n * 189, 256) < 1024 ? grid_for(c.lv[l].n * 189, 256) : 1024, 256, 0,
                        c.stream>>>(c.lv[l].n, c.lv[l].ilist, d);
  const Level &lf = c.lv[c.H - 1];
  count_p2p_pairs<<<grid_for(lf.n, 256), 256, 0, c.stream>>>(lf.n, c.d_leaf_start, c.d_leaf_nbr, d);
  B200_CUDA(cudaGetLastError());
  unsigned long long hv[2];
  B200_CUDA(cudaMemcpyAsync(hv, d, sizeof(hv), cudaMemcpyDeviceToHost, c.stream));
  B200_CUDA(cudaStreamSynchronize(c.stream));
  if (m2l_pairs) *m2l_pairs = (long long)hv[0];
  if (p2p_pairs) *p2p_pairs = (long long)hv[1];
  return B200FMM_OK;
}

b200fmm_status b200fmm_m2l_flops(b200fmm_handle h, double *flops) {
  B200_CHECK(check_handle(h));
  Context &c = *h;
  if (!flops) return fail(B200FMM_ERR_INVALID, "null argument");
  B200_CHECK(need_particles(c));
  B200_CHECK(set_device(c));
  int rank[343];
  double fed[8];
  const bool lr = c.cfg.precision == B200FMM_MIXED && tc_lowrank_info(c, rank, fed);
  const bool sym64 = c.cfg.precision == B200FMM_FP64 && c.cfg.kernel == B200FMM_CHEB_SYM;
  // the FP64 symmetric M2L runs as two GEMMs: V^T M per source cell over the slots its parity feeds, then U Y
  // per pair -- the same work as the low-rank tensor-core form
  const bool two_gemm = sym64 && sym64_fed_ranks(c, fed);
  if (!lr && !sym64) {
    long long pairs = 0;
    B200_CHECK(b200fmm_tree_stats(h, &pairs, nullptr));
    *flops = 2.0 * c.nn * (double)c.nn * (double)pairs * c.R;
    return B200FMM_OK;
  }
  if (sym64) {
    for (int t = 0; t < 343; ++t) rank[t] = 0;
    std::vector<int> pind, pvec;
    slot_symmetry_tables(c.p, pind, pvec);
    for (int t = 0; t < 343; ++t) rank[t] = c.sym_ranks[pind[t]];
  }
  B200_CHECK(build_ilists(c));
  RankTable T;
  for (int ct = 0; ct < 8; ++ct)
    for (int e = 0; e < 189; ++e) T.r[ct][e] = rank[c.itab.slot[ct][e]];
  B200_CHECK(ensure_scratch(c, 4096));
  unsigned long long *d = (unsigned long long *)((char *)c.d_scratch + 2048);
  B200_CUDA(cudaMemsetAsync(d, 0, 9 * sizeof(unsigned long long), c.stream));
  for (int l = 2; l < c.H; ++l)
    if (c.lv[l].n)
      count_m2l_ranks<<<grid_for(c.lv[l].n, 256), 256, 0, c.stream>>>(c.lv[l].n, c.lv[l].keys, c.lv[l].ilist, T, d);
  B200_CUDA(cudaGetLastError());
  unsigned long long hv[9];
  B200_CUDA(cudaMemcpyAsync(hv, d, sizeof(hv), cudaMemcpyDeviceToHost, c.stream));
  B200_CUDA(cudaStreamSynchronize(c.stream));
  if (sym64 && !two_gemm) {
    // per pair: Y = V^T M and U Y, each 2 p^3 r
    *flops = 4.0 * c.nn * (double)hv[0] * c.R;
  } else {
    // second product per pair (2 p^3 r), first product per cell over the slots its parity feeds
    double first = 0;
    for (int ct = 0; ct < 8; ++ct) first += (double)hv[1 + ct] * fed[ct];
    *flops = 2.0 * c.nn * ((double)hv[0] + first) * c.R;
  }
  return B200FMM_OK;
}

b200fmm_status b200fmm_last_launch_count(b200fmm_handle h, long long *count) {
  B200_CHECK(check_handle(h));
  if (!count) return fail(B200FMM_ERR_INVALID, "null argument");
  *count = h->launches + h->tree_launches;
  return B200FMM_OK;
}

b200fmm_status b200fmm_direct(long long n, const double *x, const double *y, const double *z, const double *q,
                              long long ntargets, const long long *targets, double *phi, double *fx, double *fy,
                              double *fz) {
  if (n < 1 || !x || !y || !z || !q || !phi || !fx || !fy || !fz) return fail(B200FMM_ERR_INVALID, "bad argument");
  const long long nt = ntargets < 0 ? n : ntargets;
  if (ntargets >= 0 && !targets) return fail(B200FMM_ERR_INVALID, "null target list");
  for (long long k = 0; ntargets >= 0 && k < nt; ++k)
    if (targets[k] < 0 || targets[k] >= n) return fail(B200FMM_ERR_INVALID, "target index out of range");
  cudaStream_t s;
  B200_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  double *d = nullptr;
  long long *dt = nullptr;
  const size_t in_bytes = sizeof(double) * n * 4, out_bytes = sizeof(double) * nt * 4;
  cudaError_t e = cudaMallocAsync(&d, in_bytes + out_bytes, s);
  if (e == cudaSuccess && ntargets >= 0) e = cudaMallocAsync(&dt, sizeof(long long) * nt, s);
  if (e != cudaSuccess) {
    cudaStreamDestroy(s);
    return fail(B200FMM_ERR_OOM, "device allocation failed");
  }
  cudaMemcpyAsync(d, x, sizeof(double) * n, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d + n, y, sizeof(double) * n, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d + 2 * n, z, sizeof(double) * n, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d + 3 * n, q, sizeof(double) * n, cudaMemcpyHostToDevice, s);
  if (dt) cudaMemcpyAsync(dt, targets, sizeof(long long) * nt, cudaMemcpyHostToDevice, s);
  double *o = d + 4 * n;
  b200fmm_status st = run_direct(n, d, d + n, d + 2 * n, d + 3 * n, nt, dt, o, o + nt, o + 2 * nt, o + 3 * nt, s);
  if (st == B200FMM_OK) {
    double *dst[4] = {phi, fx, fy, fz};
    for (int k = 0; k < 4; ++k) cudaMemcpyAsync(dst[k], o + k * nt, sizeof(double) * nt, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = fail(B200FMM_ERR_CUDA, cudaGetErrorString(e));
  }
  cudaFreeAsync(d, s);
  if (dt) cudaFreeAsync(dt, s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return st;
}

}  // extern "C"
