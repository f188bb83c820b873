// Shared definitions of the b200fmm library: the handle (context), the per-level tree storage,
// error plumbing and small device helpers.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/b200fmm.h"

namespace b200 {

constexpr int kMaxOrder = 8;
constexpr int kMaxHeight = 12;
// slots per level of the multipole maxima that P2M and M2M record (spread to keep atomics uncontended)
constexpr int kMmaxSlots = 64;
constexpr int kMaxNrhs = 32;
// work items of the FP32 near field (one warp each): a leaf of at most `whole` targets is one item, a larger leaf
// is cut into items of `item` targets, so that dense leaves spread over many warps.  Defaults 64 / 32;
// b200fmm_autotune picks them per handle.
constexpr int kP2PWholeLeaf = 64;
constexpr int kP2PItemTargets = 32;
__host__ __device__ inline long long p2p_leaf_items(long long n, int whole, int item) {
  return n <= whole ? 1 : (n + item - 1) / item;
}

// Error reporting: the last message per host thread.
void set_error(const std::string &msg);
b200fmm_status fail(b200fmm_status st, const std::string &msg);

#define B200_CUDA(call)                                                                                   \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess)                                                                                \
      return ::b200::fail(e_ == cudaErrorMemoryAllocation ? B200FMM_ERR_OOM : B200FMM_ERR_CUDA,          \
                          std::string(#call) + ": " + cudaGetErrorString(e_));                          \
  } while (0)

#define B200_CHECK(st)                  \
  do {                                  \
    b200fmm_status s_ = (st);           \
    if (s_ != B200FMM_OK) return s_;    \
  } while (0)

// One level of the octree.  Cells are the non-empty cells of the level in Morton order.
struct Level {
  long long n = 0;
  size_t cap = 0;             // allocated cells (grow-only)
  bool grid_ready = false;
  long long *keys = nullptr;  // [n] Morton keys (device)
  int *parent = nullptr;      // [n] index of the parent cell at level-1 (device)
  int *child = nullptr;       // [n][8] index of child cells at level+1, -1 if empty (device)
  int *ilist = nullptr;       // [n][189] source cell of each interaction-list entry, -1 if empty (device)
  double *M = nullptr;        // [n][nrhs][p^3] multipole expansions (device)
  double *L = nullptr;        // [n][nrhs][p^3] local expansions (device)
  int *grid = nullptr;        // [side^3] cell index by (x,y,z) grid position, -1 if empty (device, MIXED)
};

// Interaction-list candidates of a target with Morton child index c (0..7): the children of the
// parent's 26 neighbours that are not adjacent to the target (FTreeCoordinate.hpp:219-264).
struct IListTable {
  int n[8];                  // 189 for every child type
  signed char off[8][189][3];
  short slot[8][189];        // ((dx+3)*7+(dy+3))*7+(dz+3)
};

struct DenseTC;  // tensor-core M2L state (m2l_tc.cu)
struct Sym64;    // two-GEMM FP64 symmetric M2L state (m2l_sym64.cu)

struct Context {
  b200fmm_config cfg{};
  int p = 0, nn = 0, H = 0, R = 1;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaStream_t stream2 = nullptr;              // the near field, concurrent with the upward pass
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // asynchronous results: the caller-order results are staged in d_out and copied to the host on stream_out
  cudaStream_t stream_out = nullptr;
  cudaEvent_t ev_scat = nullptr, ev_out = nullptr;  // staged on the main stream / copies done on stream_out
  // host inputs of set_particles: uploaded on stream_in, so that the upload overlaps work still queued on the
  // main stream; ev_stage_free follows the last main-stream reader of the staging buffer
  cudaStream_t stream_in = nullptr;
  cudaEvent_t ev_in_xyz = nullptr, ev_in_q = nullptr, ev_stage_free = nullptr;
  double *d_out = nullptr;
  size_t out_cap = 0;                          // bytes of d_out
  bool p2p_overlapped = false;                 // the last execute() ran P2P on stream2
  // target shard of execute(): the particles of a Morton range of leaves holding about N / shard_count of them
  // (shard_rank of shard_count); shard_count 1 evaluates every particle
  int shard_rank = 0, shard_count = 1;
  long long *d_shard = nullptr;                // [2 + 2 * kMaxHeight]: leaf range, then each level's cell range
  long long shard_serial = -1;                 // tree d_shard was computed for
  int device = 0;

  // interpolation tables (device)
  double *d_roots = nullptr;     // [p]
  double *d_S = nullptr;         // [8][3][p][p] child->parent 1-D interpolators

  // symmetric compressed operators (host copy + device)
  std::vector<int> sym_ranks;        // [343]
  std::vector<double> sym_uv;        // reference layout
  int *d_pindices = nullptr;         // [343]
  int *d_pvec = nullptr;             // [343][nn]
  double *d_symU = nullptr;          // per class slot: U^T stored [r][nn] (= the reference's column-major U)
  double *d_symV = nullptr;          // per class slot: V^T stored [r][nn]
  long long *d_symoff = nullptr;     // [343] element offset of slot's U/V in d_symU/d_symV, -1 if none
  int *d_symrank = nullptr;          // [343]
  int max_rank = 0;
  // the same operators expanded per transfer-vector slot t through its permutation:
  // Ut[t][n][a] = U_c[pvec_t[n]][a], Vt[t][m][a] = V_c[pvec_t[m]][a] (both row-major p^3 x r)
  double *d_Ut = nullptr, *d_Vt = nullptr;
  long long *d_toff = nullptr;       // [343] element offset of slot t's Ut / Vt, -1 for near slots
  int *d_trank = nullptr;            // [343] rank of slot t (its class's rank)

  // dense FP64 operators (CHEB_DENSE / LAGRANGE in FP64): [343][nn][nn], zero for near slots
  double *d_dense = nullptr;

  IListTable itab{};
  IListTable *d_itab = nullptr;
  int *d_class_order = nullptr;  // [8][189] list entries of child type c ordered by symmetry class
  int *d_cls_bounds = nullptr;   // [8][17] start of each class's run in d_class_order (16 classes + end)
  std::vector<int> cls_slots;    // the 16 class slots in increasing order
  int *d_cls_slots = nullptr;    // same, on the device

  // particles (sorted by Morton key, stable)
  long long N = 0;
  double *d_x = nullptr, *d_y = nullptr, *d_z = nullptr;  // sorted positions
  double *d_q = nullptr;                                  // [R][N] sorted charges
  long long *d_perm = nullptr;                            // sorted -> original
  long long *d_leaf_start = nullptr;                      // [nleaves+1]
  int *d_leaf_nbr = nullptr;                              // [nleaves][27] (13 = self), -1 if empty
  float4 *d_pq32 = nullptr;                               // FP32 near-field copies (MIXED), see p2p.cu
  int *d_leaf_rank = nullptr;      // [nleaves] position of each leaf in the column-major record order (MIXED P2P)
  long long *d_rec_base = nullptr; // [nleaves+1] first source record of each leaf, in that order
  // [nleaves+1] first work item of each leaf in the FP32 near field (p2p_leaf_items per leaf,
  // each a work item of its own (the last entry is the item count), so that dense leaves spread over many warps
  long long *d_chunk_base = nullptr;
  int p2p_whole = kP2PWholeLeaf, p2p_item = kP2PItemTargets;  // the work-item rule d_chunk_base was built with
  double *d_phi = nullptr, *d_fx = nullptr, *d_fy = nullptr, *d_fz = nullptr;  // [R][N] sorted results
  Level lv[kMaxHeight];
  bool has_particles = false;
  bool packed32 = false;      // d_pq32 holds the current particles
  bool state_zero = false;    // expansions and results are all zero (nothing ran since they were reset)
  // CUDA graph of execute(): captured on the second execute() of one tree with the same operations and
  // replayed from then on (set_charges() keeps the tree; set_particles() starts a new one)
  long long tree_serial = 0;              // bumped by every set_particles()
  long long ilist_serial = -1;            // tree whose interaction lists are built (MIXED builds them on demand)
  long long column_serial = -1;           // tree whose leaves are in the FP32 P2P column order
  long long eager_serial = -1, graph_serial = -1;
  unsigned eager_ops = 0, graph_ops = 0;
  cudaGraphExec_t graph = nullptr;
  long long graph_launches = 0;           // kernels in the graph
  bool capturing = false;                 // inside the capture: no timing events
  bool last_was_graph = false;            // the last execute() replayed the graph (only its total is timed)

  // grow-only buffers of the tree build (capacities in elements)
  size_t cap_N = 0, cap_leaf = 0, cap_sort = 0, cap_cnt = 0, cap_stage = 0, cap_scan = 0;
  unsigned long long *d_sortk = nullptr;  // [2N] radix-sort keys (ping-pong)
  int *d_sortv = nullptr;                 // [2N] radix-sort values
  long long *d_flags = nullptr;           // [2(N+1)] head flags and their scan
  unsigned *d_cnt = nullptr;              // radix histograms and offsets
  double *d_stage = nullptr;              // host input staged on the device
  long long *d_scan = nullptr;            // scan block sums
  int *d_err = nullptr;                   // domain error flag; from byte 16 the cell count of each level
  long long *h_pinned = nullptr;          // small pinned host buffer for counts
  int tree_gen = 0;                       // bumped whenever a tree buffer moves

  // device status words set by kernels whose bounded waits ran out (0 = fine); checked by the host at
  // every synchronising call
  int *d_status = nullptr;
  // max |M| of every level as P2M and M2M write it, [kMaxHeight][kMmaxSlots] bit patterns of non-negative
  // doubles (which order like the doubles).  execute() points mmax_out at it for its upward pass; after a
  // complete upward pass from zeroed expansions mmax_ready tells the tensor-core M2L that the maxima of the
  // current multipoles are there, so that it needs no pass of its own over them.
  unsigned long long *d_mmax = nullptr;
  unsigned long long *mmax_out = nullptr;
  bool mmax_ready = false;

  // scratch
  void *d_scratch = nullptr;
  size_t scratch_bytes = 0;

  DenseTC *tc = nullptr;
  Sym64 *s64 = nullptr;

  // timings / counters
  cudaEvent_t ev[17];  // [16]: the end of M2M, before the wait for a concurrent near field
  bool events_ready = false;
  double ms[8] = {0};
  long long launches = 0;       // kernel launches of the last execute()
  long long tree_launches = 0;  // kernel launches of the last set_particles()
};

b200fmm_status ensure_scratch(Context &c, size_t bytes);
b200fmm_status check_status(Context &c);

// ---- module entry points -------------------------------------------------------------------------
// precompute.cu
b200fmm_status build_tables(Context &c);
b200fmm_status compress_sym_operators(Context &c);
// ACA + QR + SVD compression of ncls weighted class matrices (device, row-major nn x nn each) with node
// weights dw: ranks per class and the factors in the reference layout (per class: U rows, then V rows)
b200fmm_status compress_classes(Context &c, int ncls, const double *dA, const double *dw, double eps,
                                std::vector<int> &ranks, std::vector<double> &uv);
b200fmm_status upload_sym_operators(Context &c);
bool tc_lowrank_info(const Context &c, int *rank_of_slot, double *rank_fed);
void slot_symmetry_tables(int p, std::vector<int> &pind, std::vector<int> &pvec);
b200fmm_status sym_slot_factors(const Context &c, std::vector<double> &Ut, std::vector<double> &Vt,
                                std::vector<long long> &toff, std::vector<int> &trank);
b200fmm_status build_dense_operators(Context &c);
// tree.cu
b200fmm_status build_ilists(Context &c);
b200fmm_status build_tree(Context &c, const double *x, const double *y, const double *z, const double *q,
                          bool on_device);
b200fmm_status upload_charges(Context &c, const double *q, bool on_device);
void free_tree(Context &c);
// interp.cu
// the interpolation nodes and Chebyshev values of the handle's order into the device's constant tables
b200fmm_status upload_basis_constants(const Context &c, const double *roots, const double *Tr);
b200fmm_status run_p2m(Context &c);
b200fmm_status run_m2m(Context &c, int level);
b200fmm_status run_l2l(Context &c, int level);
// shard: [first leaf, end leaf) in device memory, or null for every leaf
b200fmm_status run_l2p(Context &c, const long long *shard = nullptr);
// p2p.cu
b200fmm_status run_p2p(Context &c, int variant, const long long *shard = nullptr);
// Orders the leaves by (x, y) column, z within a column (stable from Morton order), into d_leaf_rank, and
// lays out the FP32 source records in that order (d_rec_base).  Uses the free tree-build scratch.
b200fmm_status leaf_column_order(Context &c);
// m2l_fp64.cu
b200fmm_status run_m2l_fp64(Context &c, int level);
// m2l_sym64.cu: the FP64 symmetric M2L as two GEMMs per level (stacked V_t^T, then concatenated U_t)
b200fmm_status sym64_prepare(Context &c, const double *d_Ut, const double *d_Vt, const std::vector<long long> &toff,
                             const std::vector<int> &trank);
void sym64_free(Context &c);
b200fmm_status run_m2l_sym64(Context &c, int level);
// rows of the stacked V of each source parity (the ranks of the slots that parity feeds)
bool sym64_fed_ranks(const Context &c, double *fed);
// m2l_tc.cu
b200fmm_status tc_init(Context &c);
void tc_free(Context &c);
b200fmm_status run_m2l_tc(Context &c, int level);
b200fmm_status tc_tree_setup(Context &c);
void tc_invalidate_units(Context &c);  // the work units are recomputed at the next M2L (shard change)
bool tc_tables_pending(const Context &c);  // the current tree's tables are not built yet
b200fmm_status shard_ranges(Context &c);  // d_shard for the current tree
void tc_set_splits(Context &c, int splits);
int tc_splits_used(const Context &c);
// direct.cu
b200fmm_status run_direct(long long n, const double *x, const double *y, const double *z, const double *q,
                          long long nt, const long long *targets, double *phi, double *fx, double *fy, double *fz,
                          cudaStream_t s);

// ---- device helpers --------------------------------------------------------------------------------
__host__ __device__ inline long long morton_encode3(int ix, int iy, int iz) {
  long long key = 0;
#pragma unroll
  for (int b = 0; b < 21; ++b) {
    key |= (long long)((iz >> b) & 1) << (3 * b);
    key |= (long long)((iy >> b) & 1) << (3 * b + 1);
    key |= (long long)((ix >> b) & 1) << (3 * b + 2);
  }
  return key;
}

__host__ __device__ inline void morton_decode3(long long key, int &ix, int &iy, int &iz) {
  int x = 0, y = 0, z = 0;
#pragma unroll
  for (int b = 0; b < 21; ++b) {
    z |= (int)((key >> (3 * b)) & 1) << b;
    y |= (int)((key >> (3 * b + 1)) & 1) << b;
    x |= (int)((key >> (3 * b + 2)) & 1) << b;
  }
  ix = x;
  iy = y;
  iz = z;
}

// Index of key in sorted keys[0..n), or -1.
__device__ inline int find_key(const long long *keys, long long n, long long key) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (keys[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < n && keys[lo] == key) ? (int)lo : -1;
}

// Timing event k on the handle's stream, except while execute() is being captured into a CUDA graph.
inline cudaError_t record_event(Context &c, int k) {
  return c.capturing ? cudaSuccess : cudaEventRecord(c.ev[k], c.stream);
}

inline unsigned grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 2147483647LL) g = 2147483647LL;
  return (unsigned)g;
}

}  // namespace b200

// The opaque handle type of the C ABI is the context itself.
struct b200fmm_context : public b200::Context {};
