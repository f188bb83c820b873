// Tree construction on the GPU -- integer work, bit-exact with the reference's rules:
//   leaf coordinate  FCoordinateComputer::GetTreeCoordinate (Src/Containers/FCoordinateComputer.hpp:16-40)
//   Morton key       FTreeCoordinate::getMortonIndex (Src/Containers/FTreeCoordinate.hpp:91-113)
//   leaf order       FOctree::insert appends in input order -> a stable sort by key
//   leaf neighbours  FTreeCoordinate::getNeighborsIndexes (FTreeCoordinate.hpp:189-216)
//   interaction list FTreeCoordinate::getInteractionNeighbors (FTreeCoordinate.hpp:219-264)
//
// The particle sort is a stable LSD radix sort with 8-bit digits (histogram / scan / scatter per digit,
// ranks within a warp by __match_any_sync); keys have 3*(height-1) significant bits, two passes at height 6.
// The leaf sort of sparse trees uses 4-bit digits.
#include "common.cuh"

#include <algorithm>

namespace b200 {

namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_BINS = 16;
constexpr int RS8_BINS = 256;  // 8-bit digits: each warp of a tile owns 256 consecutive items (8 rounds of 32)
static_assert(RS_THREADS == RS8_BINS && RS_ITEMS == 8, "one thread per digit; 8 rounds of 32 items per warp");

// --------------------------------------------------------------------------------------------------
// keys
// --------------------------------------------------------------------------------------------------
__global__ void keys_kernel(long long n, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, double cx, double cy, double cz, double box_width,
                            double leaf_width, int height, unsigned long long *__restrict__ keys,
                            int *__restrict__ vals, int *__restrict__ err) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double r[3] = {x[i] - cx, y[i] - cy, z[i] - cz};
  int c[3];
  const int last = (1 << (height - 1)) - 1;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (!(r[d] >= 0.0 && r[d] <= box_width)) {  // also rejects NaN
      atomicExch(err, 1);
      c[d] = 0;
    } else if (r[d] == box_width) {
      c[d] = last;
    } else {
      c[d] = (int)(r[d] / leaf_width);
      if (c[d] > last) c[d] = last;  // unreachable for in-box input; keeps the key in range
    }
  }
  keys[i] = (unsigned long long)morton_encode3(c[0], c[1], c[2]);
  vals[i] = (int)i;
}

// --------------------------------------------------------------------------------------------------
// radix sort
// --------------------------------------------------------------------------------------------------
__global__ void rs_hist(const unsigned long long *__restrict__ keys, long long n, int shift, int nblocks,
                        unsigned *__restrict__ counts) {
  __shared__ unsigned h[RS_BINS];
  if (threadIdx.x < RS_BINS) h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * RS_TILE;
#pragma unroll
  for (int k = 0; k < RS_ITEMS; ++k) {
    const long long i = base + k * RS_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & (RS_BINS - 1)], 1u);
  }
  __syncthreads();
  if (threadIdx.x < RS_BINS) counts[(long long)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// 8-bit digits.  Histogram of one tile: counts[d * nblocks + block].
__global__ void rs8_hist(const unsigned long long *__restrict__ keys, long long n, int shift, int nblocks,
                         unsigned *__restrict__ counts) {
  __shared__ unsigned h[RS8_BINS];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * RS_TILE;
#pragma unroll
  for (int k = 0; k < RS_ITEMS; ++k) {
    const long long i = base + k * RS_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & (RS8_BINS - 1)], 1u);
  }
  __syncthreads();
  counts[(long long)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile.  Warp w owns the tile's items [256 w, 256 w + 256), taken in 8 rounds of 32
// consecutive items; within a round the lanes with the same digit find each other (__match_any_sync) and
// rank by lane, and per-warp running counts carry the ranks across rounds.  An item's position is the
// tile's global offset for its digit, plus the items of that digit in the tile's earlier warps, plus its
// rank in its own warp: input order is kept within every digit.
__global__ void __launch_bounds__(RS_THREADS) rs8_scatter(const unsigned long long *__restrict__ kin,
                                                          const int *__restrict__ vin,
                                                          unsigned long long *__restrict__ kout,
                                                          int *__restrict__ vout, long long n, int shift, int nblocks,
                                                          const unsigned *__restrict__ offsets) {
  constexpr int W = RS_THREADS / 32;
  __shared__ unsigned wc[W][RS8_BINS];  // per-warp counts, then the counts of the warps before
  __shared__ unsigned boff[RS8_BINS];
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
#pragma unroll
  for (int k = 0; k < W; ++k) wc[k][t] = 0;
  boff[t] = offsets[(long long)t * nblocks + blockIdx.x];
  __syncthreads();
  const long long base = (long long)blockIdx.x * RS_TILE + (long long)w * (32 * RS_ITEMS);
  const unsigned lt = (1u << lane) - 1u;
  unsigned long long k[RS_ITEMS];
  int v[RS_ITEMS], dg[RS_ITEMS];
  unsigned rank[RS_ITEMS];
#pragma unroll
  for (int j = 0; j < RS_ITEMS; ++j) {
    const long long i = base + j * 32 + lane;
    const bool ok = i < n;
    k[j] = ok ? kin[i] : 0ull;
    v[j] = ok ? vin[i] : 0;
    dg[j] = ok ? (int)((k[j] >> shift) & (RS8_BINS - 1)) : RS8_BINS;
    const unsigned peers = __match_any_sync(0xffffffffu, dg[j]);
    const unsigned before = ok ? wc[w][dg[j]] : 0u;
    rank[j] = before + __popc(peers & lt);
    __syncwarp();
    if (ok && (peers & lt) == 0) wc[w][dg[j]] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    // thread t: digit t, exclusive prefix over the warps
    unsigned run = 0;
#pragma unroll
    for (int q = 0; q < W; ++q) {
      const unsigned c = wc[q][t];
      wc[q][t] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RS_ITEMS; ++j) {
    if (dg[j] >= RS8_BINS) continue;
    const unsigned pos = boff[dg[j]] + wc[w][dg[j]] + rank[j];
    kout[pos] = k[j];
    vout[pos] = v[j];
  }
}

// Exclusive scan of an unsigned array in tiles of 1024 (one block per tile), block sums out.
__global__ void scan_tiles_u32(const unsigned *__restrict__ in, unsigned *__restrict__ out, long long n,
                               unsigned *__restrict__ sums) {
  __shared__ unsigned wsum[32];
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  const unsigned v = i < n ? in[i] : 0u;
  // warp inclusive scan
  unsigned x = v;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned y = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += t;
    }
    wsum[lane] = y;
  }
  __syncthreads();
  const unsigned incl = x + (w > 0 ? wsum[w - 1] : 0u);
  if (i < n) out[i] = incl - v;
  if (threadIdx.x == 1023 && sums) sums[blockIdx.x] = incl;
}

__global__ void add_tile_offsets_u32(unsigned *__restrict__ out, long long n, const unsigned *__restrict__ offs) {
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += offs[blockIdx.x];
}

// Same for long long.
__global__ void scan_tiles_i64(const long long *__restrict__ in, long long *__restrict__ out, long long n,
                               long long *__restrict__ sums) {
  __shared__ long long wsum[32];
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  const long long v = i < n ? in[i] : 0;
  long long x = v;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    long long y = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += t;
    }
    wsum[lane] = y;
  }
  __syncthreads();
  const long long incl = x + (w > 0 ? wsum[w - 1] : 0);
  if (i < n) out[i] = incl - v;
  if (threadIdx.x == 1023 && sums) sums[blockIdx.x] = incl;
}

__global__ void add_tile_offsets_i64(long long *__restrict__ out, long long n, const long long *__restrict__ offs) {
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += offs[blockIdx.x];
}

__global__ void rs_scatter(const unsigned long long *__restrict__ kin, const int *__restrict__ vin,
                           unsigned long long *__restrict__ kout, int *__restrict__ vout, long long n, int shift,
                           int nblocks, const unsigned *__restrict__ offsets) {
  __shared__ unsigned cnt[RS_BINS][RS_THREADS + 1];
  __shared__ unsigned base_off[RS_BINS];
  const int t = threadIdx.x;
  const long long base = (long long)blockIdx.x * RS_TILE + (long long)t * RS_ITEMS;  // blocked: items in order
  unsigned long long k[RS_ITEMS];
  int v[RS_ITEMS];
  int dg[RS_ITEMS];
  unsigned rank[RS_ITEMS];
  unsigned c[RS_BINS];
#pragma unroll
  for (int b = 0; b < RS_BINS; ++b) c[b] = 0;
#pragma unroll
  for (int j = 0; j < RS_ITEMS; ++j) {
    const long long i = base + j;
    if (i < n) {
      k[j] = kin[i];
      v[j] = vin[i];
      dg[j] = (int)((k[j] >> shift) & (RS_BINS - 1));
    } else {
      dg[j] = -1;
    }
    rank[j] = 0;
#pragma unroll
    for (int b = 0; b < RS_BINS; ++b)
      if (dg[j] == b) rank[j] = c[b]++;
  }
#pragma unroll
  for (int b = 0; b < RS_BINS; ++b) cnt[b][t] = c[b];
  if (t < RS_BINS) base_off[t] = offsets[(long long)t * nblocks + blockIdx.x];
  __syncthreads();
  // exclusive scan over threads of each digit's counts: warp w scans digits 2w and 2w+1
  {
    const int lane = t & 31, w = t >> 5;
    for (int b = 2 * w; b < 2 * w + 2; ++b) {
      unsigned loc[RS_THREADS / 32];
      unsigned s = 0;
#pragma unroll
      for (int e = 0; e < RS_THREADS / 32; ++e) {
        loc[e] = cnt[b][lane * (RS_THREADS / 32) + e];
        s += loc[e];
      }
      unsigned x = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      unsigned run = x - s;
#pragma unroll
      for (int e = 0; e < RS_THREADS / 32; ++e) {
        cnt[b][lane * (RS_THREADS / 32) + e] = run;
        run += loc[e];
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RS_ITEMS; ++j) {
    if (dg[j] < 0) continue;
    const unsigned pos = base_off[dg[j]] + cnt[dg[j]][t] + rank[j];
    kout[pos] = k[j];
    vout[pos] = v[j];
  }
}

// --------------------------------------------------------------------------------------------------
// tree arrays
// --------------------------------------------------------------------------------------------------
__global__ void gather_particles(long long n, int R, const int *__restrict__ perm, const double *__restrict__ x,
                                 const double *__restrict__ y, const double *__restrict__ z,
                                 const double *__restrict__ q, double *__restrict__ xs, double *__restrict__ ys,
                                 double *__restrict__ zs, double *__restrict__ qs, long long *__restrict__ perm64) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long j = perm[i];
  xs[i] = x[j];
  ys[i] = y[j];
  zs[i] = z[j];
  for (int r = 0; r < R; ++r) qs[(long long)r * n + i] = q[(long long)r * n + j];
  perm64[i] = j;
}

__global__ void gather_charges(long long n, int R, const long long *__restrict__ perm, const double *__restrict__ q,
                               double *__restrict__ qs) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long j = perm[i];
  for (int r = 0; r < R; ++r) qs[(long long)r * n + i] = q[(long long)r * n + j];
}

// cells of every level 0..LL: one per change of the sorted particle key above that level's bits, counted
// per warp (ballot), then per block in shared memory, then one atomic per block and level; the leaf level's
// changes are also written as flags[i] for the leaf compaction
__global__ void level_counts_kernel(long long n, const unsigned long long *__restrict__ keys, int LL,
                                    long long *__restrict__ flags, unsigned long long *__restrict__ counts) {
  __shared__ unsigned bc[kMaxHeight];
  if (threadIdx.x < kMaxHeight) bc[threadIdx.x] = 0;
  __syncthreads();
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const unsigned long long k = i < n ? keys[i] : 0ull, kp = (i > 0 && i < n) ? keys[i - 1] : 0ull;
  for (int l = 0; l <= LL; ++l) {
    const int shift = 3 * (LL - l);
    const bool head = i < n && (i == 0 || (k >> shift) != (kp >> shift));
    if (l == LL && i < n) flags[i] = head ? 1 : 0;
    const unsigned m = __ballot_sync(0xffffffffu, head);
    if (lane == 0 && m) atomicAdd(&bc[l], (unsigned)__popc(m));
  }
  __syncthreads();
  if (threadIdx.x <= LL && bc[threadIdx.x]) atomicAdd(counts + threadIdx.x, (unsigned long long)bc[threadIdx.x]);
}

__global__ void compact_leaves(long long n, const unsigned long long *__restrict__ keys,
                               const long long *__restrict__ flags, const long long *__restrict__ idx,
                               long long *__restrict__ leaf_keys, long long *__restrict__ leaf_start) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (flags[i]) {
    leaf_keys[idx[i]] = (long long)keys[i];
    leaf_start[idx[i]] = i;
  }
}

// ---- upper levels of the tree, all at once from the sorted leaf keys ---------------------------------
// Cell c of level l < LL starts at the first leaf whose key >> 3(LL - l) differs from its predecessor's;
// a leaf's cell index at level l is the number of such starts up to it, minus one.  Three launches for
// all levels: per-block start counts, their exclusive scans, then keys and parent/child links.
constexpr int ML_T = 1024;
struct LevelLinks {
  long long *keys[kMaxHeight];
  int *parent[kMaxHeight];
  int *child[kMaxHeight];
};

__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned *ws, unsigned &total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned t = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0u, u = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, u, o);
      if (lane >= o) u += y;
    }
    ws[lane] = u - t;
    if (lane == 31) ws[32] = u;
  }
  __syncthreads();
  const unsigned r = ws[w] + x - v;
  total = ws[32];
  __syncthreads();
  return r;
}

__global__ void ml_count_kernel(long long nl, const long long *__restrict__ K, int LL, unsigned *__restrict__ bcount,
                                int nblk) {
  __shared__ unsigned ws[33];
  const long long i = (long long)blockIdx.x * ML_T + threadIdx.x;
  const long long k = i < nl ? K[i] : 0, kp = (i > 0 && i < nl) ? K[i - 1] : 0;
  for (int l = 0; l < LL; ++l) {
    const int sh = 3 * (LL - l);
    const bool head = i < nl && (i == 0 || (k >> sh) != (kp >> sh));
    unsigned total;
    block_exclusive_scan(head ? 1u : 0u, ws, total);
    if (threadIdx.x == 0) bcount[(long long)l * nblk + blockIdx.x] = total;
  }
}

__global__ void ml_scan_kernel(unsigned *__restrict__ bcount, int nblk) {
  __shared__ unsigned ws[33];
  unsigned *b = bcount + (long long)blockIdx.x * nblk;
  unsigned carry = 0;
  for (int base = 0; base < nblk; base += ML_T) {
    const int j = base + threadIdx.x;
    const unsigned v = j < nblk ? b[j] : 0u;
    unsigned total;
    const unsigned ex = block_exclusive_scan(v, ws, total);
    if (j < nblk) b[j] = carry + ex;
    carry += total;
  }
}

__global__ void ml_build_kernel(long long nl, const long long *__restrict__ K, int LL,
                                const unsigned *__restrict__ boff, int nblk, LevelLinks P) {
  __shared__ unsigned ws[33];
  const long long i = (long long)blockIdx.x * ML_T + threadIdx.x;
  const long long k = i < nl ? K[i] : 0, kp = (i > 0 && i < nl) ? K[i - 1] : 0;
  int idx_next = (int)i;  // this leaf's cell at level l + 1 (at LL: the leaf itself)
  bool head_next = true;  // the leaf starts that cell
  for (int l = LL - 1; l >= 0; --l) {
    const int sh = 3 * (LL - l);
    const bool head = i < nl && (i == 0 || (k >> sh) != (kp >> sh));
    unsigned total;
    const unsigned ex = block_exclusive_scan(head ? 1u : 0u, ws, total);
    const int idx = (int)(boff[(long long)l * nblk + blockIdx.x] + ex) + (head ? 1 : 0) - 1;
    if (i < nl) {
      if (head) P.keys[l][idx] = k >> sh;
      if (head_next) {
        P.parent[l + 1][idx_next] = idx;
        P.child[l][(long long)idx * 8 + ((k >> (sh - 3)) & 7)] = idx_next;
      }
    }
    idx_next = idx;
    head_next = head;
  }
}

// interaction lists and dense grids of every level in one launch each: block b serves cell b of the
// concatenated levels 2..LL
struct LevelCellsT {
  const long long *keys[kMaxHeight];
  int *ilist[kMaxHeight];
  int *grid[kMaxHeight];
  long long start[kMaxHeight + 1];
  int l0, l1;
};

__device__ __forceinline__ int level_at(const LevelCellsT &C, long long g) {
  int l = C.l0;
  while (l < C.l1 && g >= C.start[l + 1]) ++l;
  return l;
}

// One thread per (leaf, neighbour position).  In a full leaf level (every cell a leaf) leaf i has Morton key
// i, so the neighbour's index is its key; otherwise it is found by binary search.
__global__ void leaf_neighbors_kernel(long long nleaves, const long long *__restrict__ keys, int height, int full,
                                      int *__restrict__ nbr) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= nleaves * 27) return;
  const long long c = g / 27;
  const int p = (int)(g % 27);
  int ix, iy, iz;
  morton_decode3(keys[c], ix, iy, iz);
  const int lim = 1 << (height - 1);
  const int dx = p / 9 - 1, dy = (p / 3) % 3 - 1, dz = p % 3 - 1;
  int v = -1;
  if (p == 13) {
    v = (int)c;
  } else if (ix + dx >= 0 && ix + dx < lim && iy + dy >= 0 && iy + dy < lim && iz + dz >= 0 && iz + dz < lim) {
    const long long key = morton_encode3(ix + dx, iy + dy, iz + dz);
    v = full ? (int)key : find_key(keys, nleaves, key);
  }
  nbr[g] = v;
}

__global__ void ilist_kernel(const __grid_constant__ LevelCellsT C, const IListTable *__restrict__ tab) {
  const int level = level_at(C, blockIdx.x);
  const long long c = blockIdx.x - C.start[level];
  const long long ncells = C.start[level + 1] - C.start[level];
  const long long *__restrict__ keys = C.keys[level];
  int *__restrict__ ilist = C.ilist[level];
  int ix, iy, iz;
  const long long key = keys[c];
  morton_decode3(key, ix, iy, iz);
  const int ct = (int)(key & 7);
  const int lim = 1 << level;
  for (int e = threadIdx.x; e < 189; e += blockDim.x) {
    const int sx = ix + tab->off[ct][e][0], sy = iy + tab->off[ct][e][1], sz = iz + tab->off[ct][e][2];
    int v = -1;
    if (sx >= 0 && sx < lim && sy >= 0 && sy < lim && sz >= 0 && sz < lim)
      v = find_key(keys, ncells, morton_encode3(sx, sy, sz));
    ilist[c * 189 + e] = v;
  }
}

__global__ void grid_index_kernel(const __grid_constant__ LevelCellsT C) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= C.start[C.l1 + 1]) return;
  const int level = level_at(C, g);
  const long long c = g - C.start[level];
  const long long *__restrict__ keys = C.keys[level];
  int *__restrict__ grid = C.grid[level];
  int ix, iy, iz;
  morton_decode3(keys[c], ix, iy, iz);
  const long long side = 1LL << level;
  grid[((long long)iz * side + iy) * side + ix] = (int)c;
}

// column key of a leaf: (x, y) of its cell; a stable sort by it from Morton order (monotone in z inside a
// column) puts the three z-neighbours of every column next to each other
__global__ void leaf_column_keys(long long nleaves, const long long *__restrict__ keys, int LL,
                                 unsigned long long *__restrict__ k, int *__restrict__ v) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nleaves) return;
  int ix, iy, iz;
  morton_decode3(keys[i], ix, iy, iz);
  k[i] = ((unsigned long long)ix << LL) | (unsigned long long)iy;
  v[i] = (int)i;
}

// The same order for a full leaf level (every cell a leaf, so leaf i has Morton key i): the leaf at column
// position r = (x * side + y) * side + z is the cell (x, y, z).
__global__ void full_column_order(long long nleaves, int LL, int *__restrict__ order) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= nleaves) return;
  const long long side = 1LL << LL;
  const int ix = (int)(r / (side * side)), iy = (int)((r / side) % side), iz = (int)(r % side);
  order[r] = (int)morton_encode3(ix, iy, iz);
}

__global__ void leaf_rank_kernel(long long nleaves, const int *__restrict__ order,
                                 const long long *__restrict__ leaf_start, int *__restrict__ rank_of,
                                 long long *__restrict__ nrec) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= nleaves) return;
  const int leaf = order[r];
  rank_of[leaf] = (int)r;
  nrec[r] = (leaf_start[leaf + 1] - leaf_start[leaf] + 1) >> 1;  // two particles per record
}

__global__ void rec_total_kernel(long long nleaves, const long long *__restrict__ nrec, long long *__restrict__ base) {
  base[nleaves] = base[nleaves - 1] + nrec[nleaves - 1];
}

// work items of the near field per leaf (p2p_leaf_items)
__global__ void leaf_chunks_kernel(long long nleaves, const long long *__restrict__ leaf_start, int whole, int item,
                                   long long *__restrict__ nch) {
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (l >= nleaves) return;
  nch[l] = p2p_leaf_items(leaf_start[l + 1] - leaf_start[l], whole, item);
}

// grow-only device buffer: reallocates (and bumps the tree generation) only when n exceeds the capacity
template <class T>
b200fmm_status grow(Context &c, T *&p, size_t &cap, size_t n) {
  if (p && n <= cap) return B200FMM_OK;
  if (p) cudaFree(p);
  p = nullptr;
  const size_t nc = std::max<size_t>(n, cap + cap / 4);
  B200_CUDA(cudaMalloc((void **)&p, sizeof(T) * std::max<size_t>(nc, 1)));
  cap = nc;
  ++c.tree_gen;
  return B200FMM_OK;
}

// exclusive scans (host driver over tiles of 1024, block sums in a persistent buffer)
template <class T>
size_t scan_tmp_elems(long long n) {
  size_t tot = 0;
  long long tiles = (n + 1023) / 1024;
  while (tiles > 1) {
    tot += 2 * tiles;
    tiles = (tiles + 1023) / 1024;
  }
  return tot + 2;
}

b200fmm_status scan_u32(Context &c, const unsigned *in, unsigned *out, long long n, unsigned *tmp) {
  const long long tiles = (n + 1023) / 1024;
  c.tree_launches += tiles > 1 ? 2 : 1;
  scan_tiles_u32<<<(unsigned)tiles, 1024, 0, c.stream>>>(in, out, n, tiles > 1 ? tmp : nullptr);
  if (tiles > 1) {
    B200_CHECK(scan_u32(c, tmp, tmp + tiles, tiles, tmp + 2 * tiles));
    add_tile_offsets_u32<<<(unsigned)tiles, 1024, 0, c.stream>>>(out, n, tmp + tiles);
  }
  return B200FMM_OK;
}

b200fmm_status scan_i64(Context &c, const long long *in, long long *out, long long n, long long *tmp) {
  const long long tiles = (n + 1023) / 1024;
  c.tree_launches += tiles > 1 ? 2 : 1;
  scan_tiles_i64<<<(unsigned)tiles, 1024, 0, c.stream>>>(in, out, n, tiles > 1 ? tmp : nullptr);
  if (tiles > 1) {
    B200_CHECK(scan_i64(c, tmp, tmp + tiles, tiles, tmp + 2 * tiles));
    add_tile_offsets_i64<<<(unsigned)tiles, 1024, 0, c.stream>>>(out, n, tmp + tiles);
  }
  return B200FMM_OK;
}

template <class T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace

void free_tree(Context &c) {
  dfree(c.d_x);
  dfree(c.d_y);
  dfree(c.d_z);
  dfree(c.d_q);
  dfree(c.d_perm);
  dfree(c.d_leaf_start);
  dfree(c.d_leaf_nbr);
  dfree(c.d_leaf_rank);
  dfree(c.d_rec_base);
  dfree(c.d_chunk_base);
  dfree(c.d_pq32);
  dfree(c.d_phi);
  dfree(c.d_fx);
  dfree(c.d_fy);
  dfree(c.d_fz);
  dfree(c.d_sortk);
  dfree(c.d_sortv);
  dfree(c.d_flags);
  dfree(c.d_cnt);
  dfree(c.d_stage);
  dfree(c.d_scan);
  dfree(c.d_err);
  if (c.h_pinned) cudaFreeHost(c.h_pinned);
  c.h_pinned = nullptr;
  for (int l = 0; l < kMaxHeight; ++l) {
    Level &L = c.lv[l];
    dfree(L.keys);
    dfree(L.parent);
    dfree(L.child);
    dfree(L.ilist);
    dfree(L.M);
    dfree(L.L);
    dfree(L.grid);
    L.n = 0;
    L.cap = 0;
    L.grid_ready = false;
  }
  c.cap_N = c.cap_leaf = c.cap_sort = c.cap_cnt = c.cap_stage = c.cap_scan = 0;
  c.N = 0;
  c.has_particles = false;
  c.packed32 = false;
  ++c.tree_gen;
}

b200fmm_status upload_charges(Context &c, const double *q, bool on_device) {
  const long long n = c.N;
  if (!on_device) {
    B200_CHECK(grow(c, c.d_stage, c.cap_stage, (size_t)n * (3 + c.R)));
    B200_CUDA(cudaMemcpyAsync(c.d_stage, q, sizeof(double) * n * c.R, cudaMemcpyHostToDevice, c.stream));
    q = c.d_stage;
  }
  gather_charges<<<grid_for(n, 256), 256, 0, c.stream>>>(n, c.R, c.d_perm, q, c.d_q);
  B200_CUDA(cudaGetLastError());
  B200_CUDA(cudaEventRecord(c.ev_stage_free, c.stream));  // the staging buffer's last reader
  c.packed32 = false;
  return B200FMM_OK;
}

// Level storage for n cells (grow-only; M and L are zeroed by execute / reset_expansions).
static b200fmm_status level_storage(Context &c, Level &L, long long n) {
  L.n = n;
  if (L.keys && (size_t)n <= L.cap) return B200FMM_OK;
  size_t cap = L.cap, tmp;
  B200_CHECK(grow(c, L.keys, cap, (size_t)n));
  tmp = L.cap;
  B200_CHECK(grow(c, L.parent, tmp, cap));
  tmp = 8 * L.cap;
  B200_CHECK(grow(c, L.child, tmp, 8 * cap));
  tmp = 189 * L.cap;
  B200_CHECK(grow(c, L.ilist, tmp, 189 * cap));
  tmp = (size_t)c.R * c.nn * L.cap;
  B200_CHECK(grow(c, L.M, tmp, (size_t)c.R * c.nn * cap));
  tmp = (size_t)c.R * c.nn * L.cap;
  B200_CHECK(grow(c, L.L, tmp, (size_t)c.R * c.nn * cap));
  L.cap = cap;
  return B200FMM_OK;
}

b200fmm_status build_tree(Context &c, const double *x, const double *y, const double *z, const double *q,
                          bool on_device) {
  const long long n = c.N;
  const int H = c.H, LL = H - 1;
  cudaStream_t s = c.stream;
  c.tree_launches = 0;
  c.packed32 = false;
  if (!c.h_pinned) B200_CUDA(cudaMallocHost((void **)&c.h_pinned, sizeof(long long) * 64));
  // particle-sized buffers
  size_t cap;
  cap = c.cap_N;
  B200_CHECK(grow(c, c.d_x, cap, (size_t)n));
  cap = c.cap_N;
  B200_CHECK(grow(c, c.d_y, cap, (size_t)n));
  cap = c.cap_N;
  B200_CHECK(grow(c, c.d_z, cap, (size_t)n));
  cap = c.cap_N;
  B200_CHECK(grow(c, c.d_perm, cap, (size_t)n));
  for (double **p : {&c.d_q, &c.d_phi, &c.d_fx, &c.d_fy, &c.d_fz}) {
    size_t cr = c.cap_N * c.R;
    B200_CHECK(grow(c, *p, cr, (size_t)n * c.R));
  }
  {
    // FP32 P2P copies: target hi [R][N], target lo [N], pair-packed sources [R][N+2][4]
    size_t cp = c.cap_N * (c.R + 1) + 4 * c.R * (c.cap_N + 2);
    B200_CHECK(grow(c, c.d_pq32, cp, (size_t)n * (c.R + 1) + 4 * (size_t)c.R * (n + 2)));
  }
  c.cap_N = std::max(c.cap_N, (size_t)n);
  {
    // the three sort buffers share one capacity: each compares against the old value
    size_t cs = c.cap_sort;
    B200_CHECK(grow(c, c.d_sortk, cs, (size_t)2 * (n + 1)));
    cs = c.cap_sort;
    B200_CHECK(grow(c, c.d_sortv, cs, (size_t)2 * (n + 1)));
    cs = c.cap_sort;
    B200_CHECK(grow(c, c.d_flags, cs, (size_t)2 * (n + 1)));
    c.cap_sort = std::max(c.cap_sort, (size_t)(2 * (n + 1)));
  }
  const long long nb = (n + RS_TILE - 1) / RS_TILE;
  B200_CHECK(grow(c, c.d_cnt, c.cap_cnt, (size_t)2 * RS8_BINS * nb));
  B200_CHECK(grow(c, c.d_scan, c.cap_scan,
                  std::max(scan_tmp_elems<long long>(n + 1), scan_tmp_elems<unsigned>(RS8_BINS * nb))));
  // the domain error flag (int) followed, 16 bytes in, by the per-level cell counts
  if (!c.d_err) B200_CUDA(cudaMalloc(&c.d_err, 32 + sizeof(unsigned long long) * kMaxHeight));
  // inputs on the device
  const double *dx = x, *dy = y, *dz = z, *dq = q;
  if (!on_device) {
    B200_CHECK(grow(c, c.d_stage, c.cap_stage, (size_t)n * (3 + c.R)));
    // The inputs travel on a copy stream of their own: in a time-stepping loop this upload runs while the
    // previous evaluation is still executing on the main stream.  The staging buffer is rewritten only after
    // its last main-stream reader (the previous build's gather, or set_charges' gather) has run.  The keys wait
    // for the coordinates; the charges, first read by the gather after the sort, arrive meanwhile.
    B200_CUDA(cudaStreamWaitEvent(c.stream_in, c.ev_stage_free, 0));
    B200_CUDA(cudaMemcpyAsync(c.d_stage, x, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream_in));
    B200_CUDA(cudaMemcpyAsync(c.d_stage + n, y, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream_in));
    B200_CUDA(cudaMemcpyAsync(c.d_stage + 2 * n, z, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream_in));
    B200_CUDA(cudaEventRecord(c.ev_in_xyz, c.stream_in));
    B200_CUDA(cudaMemcpyAsync(c.d_stage + 3 * n, q, sizeof(double) * n * c.R, cudaMemcpyHostToDevice, c.stream_in));
    B200_CUDA(cudaEventRecord(c.ev_in_q, c.stream_in));
    B200_CUDA(cudaStreamWaitEvent(s, c.ev_in_xyz, 0));
    dx = c.d_stage;
    dy = c.d_stage + n;
    dz = c.d_stage + 2 * n;
    dq = c.d_stage + 3 * n;
  }
  unsigned long long *k0 = c.d_sortk, *k1 = c.d_sortk + n;
  int *v0 = c.d_sortv, *v1 = c.d_sortv + n;
  unsigned *cnt = c.d_cnt, *off = c.d_cnt + RS8_BINS * nb;
  long long *flags = c.d_flags, *idx = c.d_flags + (n + 1);
  B200_CUDA(cudaMemsetAsync(c.d_err, 0, sizeof(int), s));
  const double W = c.cfg.box_width;
  const double leaf_w = W / (double)(1 << LL);
  keys_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, dx, dy, dz, c.cfg.center[0] - W / 2, c.cfg.center[1] - W / 2,
                                               c.cfg.center[2] - W / 2, W, leaf_w, H, k0, v0, c.d_err);
  ++c.tree_launches;
  // stable LSD radix sort of (key, original index)
  const int bits = 3 * LL;
  for (int sh = 0; sh < bits; sh += 8) {
    rs8_hist<<<(unsigned)nb, RS_THREADS, 0, s>>>(k0, n, sh, (int)nb, cnt);
    B200_CHECK(scan_u32(c, cnt, off, RS8_BINS * nb, (unsigned *)c.d_scan));
    rs8_scatter<<<(unsigned)nb, RS_THREADS, 0, s>>>(k0, v0, k1, v1, n, sh, (int)nb, off);
    c.tree_launches += 2;
    std::swap(k0, k1);
    std::swap(v0, v1);
  }
  if (!on_device) B200_CUDA(cudaStreamWaitEvent(s, c.ev_in_q, 0));
  gather_particles<<<grid_for(n, 256), 256, 0, s>>>(n, c.R, v0, dx, dy, dz, dq, c.d_x, c.d_y, c.d_z, c.d_q, c.d_perm);
  B200_CUDA(cudaEventRecord(c.ev_stage_free, s));  // the last reader of the staging buffer
  // the cell count of every level at once (and the leaf heads), then the build's one synchronisation
  unsigned long long *counts = (unsigned long long *)(c.d_err + 4);
  B200_CUDA(cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * kMaxHeight, s));
  level_counts_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, k0, LL, flags, counts);
  c.tree_launches += 2;
  B200_CHECK(scan_i64(c, flags, idx, n, (long long *)c.d_scan));
  B200_CUDA(cudaMemcpyAsync(c.h_pinned + 2, c.d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  B200_CUDA(cudaMemcpyAsync(c.h_pinned + 8, counts, sizeof(long long) * (LL + 1), cudaMemcpyDeviceToHost, s));
  B200_CUDA(cudaStreamSynchronize(s));
  if ((int)c.h_pinned[2]) return fail(B200FMM_ERR_DOMAIN, "a particle lies outside the box or has a non-finite coordinate");
  const long long nleaves = c.h_pinned[8 + LL];
  Level &leaf = c.lv[LL];
  B200_CHECK(level_storage(c, leaf, nleaves));
  {
    size_t cl = c.cap_leaf;
    B200_CHECK(grow(c, c.d_leaf_start, cl, (size_t)nleaves + 1));
    cl = c.cap_leaf * 27;
    B200_CHECK(grow(c, c.d_leaf_nbr, cl, (size_t)(nleaves + 1) * 27));
    cl = c.cap_leaf;
    B200_CHECK(grow(c, c.d_leaf_rank, cl, (size_t)nleaves + 1));
    cl = c.cap_leaf;
    B200_CHECK(grow(c, c.d_rec_base, cl, (size_t)nleaves + 1));
    cl = c.cap_leaf;
    B200_CHECK(grow(c, c.d_chunk_base, cl, (size_t)nleaves + 1));
    c.cap_leaf = std::max(c.cap_leaf, (size_t)nleaves + 1);
  }
  compact_leaves<<<grid_for(n, 256), 256, 0, s>>>(n, k0, flags, idx, leaf.keys, c.d_leaf_start);
  ++c.tree_launches;
  c.h_pinned[3] = c.N;
  B200_CUDA(cudaMemcpyAsync(c.d_leaf_start + nleaves, c.h_pinned + 3, sizeof(long long), cudaMemcpyHostToDevice, s));
  // upper levels: storage from the counts taken before the synchronisation, then keys and links of every
  // level from the leaf keys in three launches
  LevelLinks links{};
  for (int l = LL - 1; l >= 0; --l) {
    Level &pa = c.lv[l];
    B200_CHECK(level_storage(c, pa, c.h_pinned[8 + l]));
    B200_CUDA(cudaMemsetAsync(pa.child, 0xFF, sizeof(int) * 8 * (size_t)pa.n, s));  // -1: no child
    links.keys[l] = pa.keys;
    links.parent[l] = pa.parent;
    links.child[l] = pa.child;
  }
  links.parent[LL] = leaf.parent;
  if (LL > 0) {
    const int nblk = (int)((nleaves + ML_T - 1) / ML_T);
    unsigned *bcount = (unsigned *)c.d_flags;  // LL * nblk entries; the flag scratch is free now
    ml_count_kernel<<<nblk, ML_T, 0, s>>>(nleaves, leaf.keys, LL, bcount, nblk);
    ml_scan_kernel<<<LL, ML_T, 0, s>>>(bcount, nblk);
    ml_build_kernel<<<nblk, ML_T, 0, s>>>(nleaves, leaf.keys, LL, bcount, nblk, links);
    c.tree_launches += 3;
  }
  // neighbour and interaction lists, dense grids
  leaf_neighbors_kernel<<<grid_for(nleaves * 27, 256), 256, 0, s>>>(nleaves, leaf.keys, H,
                                                                    nleaves == (1LL << (3 * LL)) ? 1 : 0, c.d_leaf_nbr);
  ++c.tree_launches;
  if (LL >= 2) {
    LevelCellsT C{};
    C.l0 = 2;
    C.l1 = LL;
    C.start[2] = 0;
    for (int l = 2; l <= LL; ++l) {
      Level &L = c.lv[l];
      C.keys[l] = L.keys;
      C.ilist[l] = L.ilist;
      C.start[l + 1] = C.start[l] + L.n;
      if (c.cfg.precision == B200FMM_MIXED) {
        const long long side = 1LL << l;
        if (!L.grid) {
          B200_CUDA(cudaMalloc(&L.grid, sizeof(int) * side * side * side));
          ++c.tree_gen;
        }
        B200_CUDA(cudaMemsetAsync(L.grid, 0xFF, sizeof(int) * side * side * side, s));  // -1: empty
        C.grid[l] = L.grid;
      }
    }
    const long long total = C.start[LL + 1];
    if (total > 0) {
      // the interaction lists feed the FP64 M2L; the tensor-core M2L works from the cell grids, and MIXED
      // builds the lists only when asked for work counts (build_ilists)
      if (c.cfg.precision == B200FMM_FP64) {
        ilist_kernel<<<(unsigned)total, 192, 0, s>>>(C, c.d_itab);
        ++c.tree_launches;
        c.ilist_serial = c.tree_serial;
      } else {
        grid_index_kernel<<<grid_for(total, 256), 256, 0, s>>>(C);
        ++c.tree_launches;
      }
    }
  }
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

// The target shard of execute(): leaves [lo, hi), the Morton range whose particles are those of ranks
// [rank * N / count, (rank + 1) * N / count) of the sorted order rounded to whole leaves, and at every level the
// cells [a, b) that are ancestors of those leaves (contiguous in Morton order).  One thread.
struct ShardLinks {
  const int *parent[kMaxHeight];
  int LL;
};
__global__ void shard_range_kernel(const long long *__restrict__ leaf_start, long long nleaves, long long N, int rank,
                                   int count, const __grid_constant__ ShardLinks S, long long *__restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  // the first leaf that starts at or after particle t
  auto first_leaf = [&](long long t) {
    long long a = 0, b = nleaves;
    while (a < b) {
      const long long m = (a + b) >> 1;
      if (leaf_start[m] < t) a = m + 1; else b = m;
    }
    return a;
  };
  const long long lo = rank == 0 ? 0 : first_leaf(N * rank / count);
  const long long hi = rank == count - 1 ? nleaves : first_leaf(N * (rank + 1) / count);
  out[0] = lo;
  out[1] = hi;
  for (int l = 0; l < kMaxHeight; ++l) out[2 + 2 * l] = out[3 + 2 * l] = 0;
  if (hi <= lo) return;
  long long a = lo, b = hi - 1;
  for (int l = S.LL; l >= 0; --l) {
    out[2 + 2 * l] = a;
    out[3 + 2 * l] = b + 1;
    if (l > 0) {
      a = S.parent[l][a];
      b = S.parent[l][b];
    }
  }
}

b200fmm_status shard_ranges(Context &c) {
  const int LL = c.H - 1;
  ShardLinks S{};
  S.LL = LL;
  for (int l = 0; l <= LL; ++l) S.parent[l] = c.lv[l].parent;
  shard_range_kernel<<<1, 32, 0, c.stream>>>(c.d_leaf_start, c.lv[LL].n, c.N, c.shard_rank, c.shard_count, S,
                                             c.d_shard);
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  c.shard_serial = c.tree_serial;
  return B200FMM_OK;
}

// Interaction lists of levels 2..height-1 of the current tree, if not built yet.
b200fmm_status build_ilists(Context &c) {
  const int LL = c.H - 1;
  if (LL < 2 || c.ilist_serial == c.tree_serial) return B200FMM_OK;
  LevelCellsT C{};
  C.l0 = 2;
  C.l1 = LL;
  C.start[2] = 0;
  for (int l = 2; l <= LL; ++l) {
    C.keys[l] = c.lv[l].keys;
    C.ilist[l] = c.lv[l].ilist;
    C.start[l + 1] = C.start[l] + c.lv[l].n;
  }
  const long long total = C.start[LL + 1];
  if (total > 0) ilist_kernel<<<(unsigned)total, 192, 0, c.stream>>>(C, c.d_itab);
  B200_CUDA(cudaGetLastError());
  c.ilist_serial = c.tree_serial;
  return B200FMM_OK;
}

}  // namespace b200

namespace b200 {

b200fmm_status leaf_column_order(Context &c) {
  const int LL = c.H - 1;
  const long long nl = c.lv[LL].n;
  cudaStream_t s = c.stream;
  // the particle sort's buffers are free after the tree build and hold 2(N+1) >= 2 nleaves entries
  unsigned long long *k0 = c.d_sortk, *k1 = c.d_sortk + nl;
  int *v0 = c.d_sortv, *v1 = c.d_sortv + nl;
  const long long nb = (nl + RS_TILE - 1) / RS_TILE;
  unsigned *cnt = c.d_cnt, *off = c.d_cnt + RS_BINS * nb;
  if (nl == (1LL << (3 * LL))) {
    // a full leaf level (uniform trees): the order follows from the cell coordinates
    full_column_order<<<grid_for(nl, 256), 256, 0, s>>>(nl, LL, v0);
    ++c.launches;
  } else {
    leaf_column_keys<<<grid_for(nl, 256), 256, 0, s>>>(nl, c.lv[LL].keys, LL, k0, v0);
    ++c.launches;
    for (int sh = 0; sh < 2 * LL; sh += 4) {
      rs_hist<<<(unsigned)nb, RS_THREADS, 0, s>>>(k0, nl, sh, (int)nb, cnt);
      B200_CHECK(scan_u32(c, cnt, off, RS_BINS * nb, (unsigned *)c.d_scan));
      rs_scatter<<<(unsigned)nb, RS_THREADS, 0, s>>>(k0, v0, k1, v1, nl, sh, (int)nb, off);
      c.launches += 2;
      std::swap(k0, k1);
      std::swap(v0, v1);
    }
  }
  long long *nrec = c.d_flags;
  leaf_rank_kernel<<<grid_for(nl, 256), 256, 0, s>>>(nl, v0, c.d_leaf_start, c.d_leaf_rank, nrec);
  B200_CHECK(scan_i64(c, nrec, c.d_rec_base, nl, (long long *)c.d_scan));
  rec_total_kernel<<<1, 1, 0, s>>>(nl, nrec, c.d_rec_base);
  // the near field's work items, leaf by leaf (nrec is free again)
  leaf_chunks_kernel<<<grid_for(nl, 256), 256, 0, s>>>(nl, c.d_leaf_start, c.p2p_whole, c.p2p_item, nrec);
  B200_CHECK(scan_i64(c, nrec, c.d_chunk_base, nl, (long long *)c.d_scan));
  rec_total_kernel<<<1, 1, 0, s>>>(nl, nrec, c.d_chunk_base);
  c.launches += 4;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

}  // namespace b200
