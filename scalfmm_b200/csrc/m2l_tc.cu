// Tensor-core M2L (MIXED precision) on tcgen05 / TMEM, fed by TMA.
//
// The transfer pass of FFmmAlgorithmThread (Src/Core/FFmmAlgorithmThread.hpp:271-322) applies, for every
// target cell and every source of its interaction list, L_target += scale * K_t M_source with K_t the dense
// p^3 x p^3 operator of transfer vector t (FChebDenseM2LHandler.hpp:178-215; FUnifM2LHandler applies the same
// operator for the Lagrange basis).  Here this is recast as GEMMs:
//
//   * Cells of a level are stored as a dense grid split by parity (the Morton child index c of the cell):
//     A[rhs*8 + c][z/2][y/2][x/2][node].  All targets of parity c share the same 189 transfer vectors, and
//     for a fixed (c, t) every source lies in parity c' = c + t (mod 2) at a constant half-grid shift, so a
//     tile of 8x4x4 targets maps to a tile of 8x4x4 sources that one 5-D TMA box load fetches (out-of-range
//     boxes are zero-filled by the TMA unit, which supplies the domain boundary).
//   * One work item = (level, rhs, parity, 128-target tile, a range of the 189 transfer vectors).  The
//     accumulator D (128 targets x p^3 nodes, FP32) lives in TMEM; per transfer vector and 32-node K chunk
//     the MMA warp issues D += A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T (split FP16: a = hi + lo carries
//     22 significant bits; operands are pre-scaled by powers of two so that lo stays normal).
//   * The MMA accumulator is reset at the start of every segment of a transfer vector's K chunks (a
//     segment is NK / nseg chunks): the tensor-core FP32 accumulation loses about a third of an ulp of the
//     running value per instruction, always in the same direction, so its error grows linearly with the
//     chain length.  After each segment the epilogue warps read D with tcgen05.ld and add it to running
//     sums held in registers with ordinary IEEE FP32 adds; at the end of a work item they add
//     scale * 2^-(sA+sB) * sum into the FP64 locals (atomic adds: several items of the same tile contribute).
//
// Roles, by warpgroup: warpgroup 0 holds the TMA producer (warp 0, one elected thread), the MMA issuer and
// TMEM owner (warp 1), the issuer of the second column half at order 7 (warp 2) and a spare warp;
// warpgroups 1 and 2 (warps 4..11) are the epilogue (TMEM lane quarter = warp % 4, column part =
// (warp - 4) / 4).  Kernels whose epilogue holds many running sums move registers from warpgroup 0 to the
// epilogue with setmaxnreg.  Shared memory: STAGES x {A_hi, A_lo, B_hi, B_lo} K-chunks with the 64-byte
// swizzle the UMMA descriptors describe, then the transfer-vector records.  Every mbarrier wait is bounded; a wait
// that runs out sets a device status word, the CTA abandons its work, frees its TMEM and returns.
#include "common.cuh"

#include <cuda.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <utility>

namespace b200 {

namespace {

constexpr int TC_THREADS = 384;  // 12 warps: TMA, MMA, second MMA issuer, spare, 8 epilogue
// Register split of the kernels with large epilogues: launched at TC_REGS per thread, warpgroup 0 gives
// registers up (setmaxnreg.dec to REG_LOW) and the two epilogue warpgroups take them (setmaxnreg.inc to
// REG_HIGH).  The split must add up to what the block was launched with, or the increase never completes;
// the host checks the compiled register count before the first launch.
constexpr int TC_REGS = 168, REG_LOW = 56, REG_HIGH = 224;
static_assert(128 * REG_LOW + 256 * REG_HIGH == TC_THREADS * TC_REGS, "register split must match the launch");
constexpr int TILE_X = 8, TILE_Y = 4, TILE_Z = 4;  // 128 targets
constexpr int KCHUNK = 32;                          // fp16 elements per 64-byte swizzle row
constexpr int SB = 15;                              // operator pre-scale 2^15
constexpr int MAX_STAGES = 8;         // stage barriers allocated
constexpr int MAX_STAGES_SINGLE = 4;  // stages used by single CTAs
constexpr long long WAIT_LIMIT = 1LL << 22;

// A work unit: one target tile (CTA pairs: the z-adjacent tiles bz, bz + 1) of one level and right-hand side,
// with the 189 transfer vectors of its parity.  Its work is the number of those whose source box is occupied.
// On a compacted level a unit is instead one block of 128 cells of one parity (CTA pairs: blocks blk, blk + 1).
struct TcItem {
  int level, rhs, parity;
  int bx, by, bz;
  int blk;  // compacted block, or -1 for a grid tile
};

struct TcLevel {
  int HX, HY, HZ;      // padded half-grid extents
  int side;            // real grid side 2^level
  int *grid;           // [side^3] cell index or -1
  double *L;           // locals of the level
  double *scale_out;   // device scalar: scale_l * 2^-(sA + SB)
  const int *sat;      // [8][HZ+1][HY+1][HX+1] occupied cells of each parity grid below (x, y, z), exclusive
  int tile0;           // first tile of this level in the busy masks
  int unit0, nunits;   // work units of this level: [unit0, unit0 + nunits), ordered rhs, parity, z, y, x
  int TZu;             // units along z: tiles, or pairs of tiles
  // compacted targets (sparse levels): the units are blocks of 128 cells of one parity, whose A rows are
  // gathered row by row from the source grid (ghi / glo: Y in the low-rank form, else the packed multipoles)
  int cmode;           // 1: this level's units are compacted blocks
  int cblk0[9];        // first block of each parity (an even count per parity for CTA pairs)
  int cb0;             // first block of the level in the compacted busy masks
  const int *crow;     // [blocks * 128]: (parity << 28) | position in the parity grid, or -1
  const int *ccell;    // [blocks * 128]: cell index, or -1
  const __half *ghi, *glo;
  long long plane;     // positions of one parity grid: HX * HY * HZ
  // low-rank form: ypr > 0 when Y of this level is stored by compacted row ([R * ycht][ypr][16], rows counted
  // from each parity's first block); rowmap[parity * plane + position] gives a cell's row, -1 where none is
  int ypr;
  const int *rowmap;
};

// Occupied cells of parity grid `par` in the box [x0, x0+nx) x [y0, y0+ny) x [z0, z0+nz) (clipped).
__device__ __forceinline__ int box_count(const TcLevel &L, int par, int x0, int y0, int z0, int nx, int ny, int nz) {
  const int x1 = min(x0 + nx, L.HX), y1 = min(y0 + ny, L.HY), z1 = min(z0 + nz, L.HZ);
  x0 = max(x0, 0);
  y0 = max(y0, 0);
  z0 = max(z0, 0);
  if (x0 >= x1 || y0 >= y1 || z0 >= z1) return 0;
  const int SX = L.HX + 1, SY = L.HY + 1;
  const int *s = L.sat + (size_t)par * SX * SY * (L.HZ + 1);
  auto at = [&](int x, int y, int z) { return s[((size_t)z * SY + y) * SX + x]; };
  return at(x1, y1, z1) - at(x0, y1, z1) - at(x1, y0, z1) - at(x1, y1, z0) + at(x0, y0, z1) + at(x0, y1, z0) +
         at(x1, y0, z0) - at(x0, y0, z0);
}

struct __align__(64) TcParams {
  CUtensorMap mapA_hi[kMaxHeight];
  CUtensorMap mapA_lo[kMaxHeight];
  CUtensorMap mapB_hi;
  CUtensorMap mapB_lo;
  TcLevel lv[kMaxHeight];
  // exclusive prefix sums of the work of all units (finest level first); this launch runs the units
  // [u_begin, u_end), split into ranges of equal work: CTA (pair) g takes ranges g, g + G, ... of G * nranges
  const int *prefix;
  int u_begin, u_end, ranges_per_cta;
  int l0, l1;  // levels of the units [u_begin, u_end)
  int pair;    // units are pairs of z-adjacent tiles
  int R, nn, KP, NP, NH, NHALF, NK, stages, ncols;
  int nseg;  // accumulator resets per transfer vector (the K chunks are split into nseg segments)
  int nbuf;  // TMEM accumulators: 2 (alternating per segment) when 2 * NP columns fit, else 1
  int stage_bytes;
  signed char off[8][189][3];
  short slot[8][189];
  int *status;
  // per tile (level, parity, bz, by, bx): 6 words, bit e set when transfer vector e has an occupied source
  // box; bit 31 of word 5 set when the tile has an occupied target cell
  const unsigned *busy;
  // per target parity c and transfer vector e (8 x 189 records, copied to shared memory by every CTA)
  const struct TvRec *tv;
  // low-rank form (symmetric Chebyshev operators K_t = U_t V_t^T): A is Y = V_t^T M, one row of 16-rank
  // chunks per source cell, and B is U_t, both in 16-wide K chunks
  int lr_seglen;  // K chunks per accumulator segment of a fragment's chunk stream
  int ycht;       // Y chunks per right-hand side (all parities)
  // compacted target blocks: 6 mask words per block as for tiles; gather = some level of the launch is
  // compacted; growlen = fp16 per gathered grid row (16 for Y chunks, KP for multipoles)
  const unsigned *cbusy;
  int gather, growlen;
  // target shard (or null): [2 + 2 l, 3 + 2 l] hold level l's owned cells [a, b); units without one do no work
  const long long *shard;
};
// What the producer and the MMA issuers need of transfer vector e of target parity c: the A box's
// coordinates (offset of the source tile in half-grid cells; outer coordinate ya + rhs * (ycht or 8)), the B
// box's outer coordinate ub, and in the low-rank form the slot's 16-wide rank chunks nk.  Dense: ya = source
// parity, ub = operator slot.  Low rank: ya = the slot's first Y chunk in the source parity's rows, ub = its
// first U chunk.
struct TvRec {
  short ya, ub;
  unsigned char nk;
  signed char ox, oy, oz;
};
static_assert(sizeof(TvRec) == 8, "8-byte records");
constexpr int TV_BYTES = 8 * 189 * (int)sizeof(TvRec);

// ---- PTX helpers ----------------------------------------------------------------------------------
__device__ __forceinline__ unsigned su32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity) {
  for (long long it = 0; it < WAIT_LIMIT; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// The same wait taken by all 32 lanes of an epilogue warp: the warp agrees on the outcome, so that no lane
// reaches the warp-collective TMEM loads (.sync.aligned) after another lane has given up.
__device__ __forceinline__ bool mbar_wait_warp(unsigned long long *b, unsigned parity) {
  return __all_sync(0xffffffffu, mbar_wait(b, parity));
}
// the same with cluster-scope acquire: for phases completed by a release arrival from the other CTA of a pair
__device__ __forceinline__ bool mbar_wait_cluster(unsigned long long *b, unsigned parity) {
  for (long long it = 0; it < WAIT_LIMIT; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// n arrivals at once (a gathering warp that has nothing to copy for a stage)
__device__ __forceinline__ void mbar_arrive_n(unsigned bar, unsigned n) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(n) : "memory");
}
// arrival on the other CTA's barrier that publishes this CTA's shared-memory writes to it
__device__ __forceinline__ void mbar_arrive_cluster_release(unsigned cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
// 16-byte copy global -> shared through L2; src_bytes = 0 writes 16 zero bytes and reads nothing
__device__ __forceinline__ void cp_async16(unsigned dst, const void *src, unsigned src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
// one arrival on the barrier once every cp.async that this thread has issued so far has landed
__device__ __forceinline__ void cp_async_arrive_noinc(unsigned bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, unsigned long long *bar, int c0, int c1,
                                            int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6, %7}], "
      "[%2];" ::"r"(su32(dst)),
      "l"(map), "r"(su32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, unsigned long long *bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(
          su32(dst)),
      "l"(map), "r"(su32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, unsigned long long *bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          su32(dst)),
      "l"(map), "r"(su32(bar)), "r"(c0), "r"(c1)
      : "memory");
}
// UMMA shared-memory descriptor: K-major, 64-byte swizzle, rows of 64 B in 8-row groups 512 B apart.
__device__ __forceinline__ unsigned long long sdesc(const void *p) {
  const unsigned long long a = su32(p);
  return ((a >> 4) & 0x3FFFull) | (1ull << 16) | (32ull << 32) | (1ull << 46) | (4ull << 61);
}
// the same for rows of 32 B (16 fp16) with the 32-byte swizzle: 8-row groups 256 B apart, layout type 6
__device__ __forceinline__ unsigned long long sdesc32(const void *p) {
  const unsigned long long a = su32(p);
  return ((a >> 4) & 0x3FFFull) | (1ull << 16) | (16ull << 32) | (1ull << 46) | (6ull << 61);
}
__device__ __forceinline__ void mma_f16(unsigned d_tmem, unsigned long long da, unsigned long long db, unsigned idesc,
                                        unsigned accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}
// ---- CTA-pair forms (cta_group::2): the even CTA of a cluster pair issues M = 256 MMAs whose A rows
// 0..127 and B columns [0, N/2) come from its own shared memory and A rows 128..255 and B columns [N/2, N)
// from its peer's, at the same offsets; each CTA's TMEM receives its own 128 rows of D.
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// shared::cluster address of the variable at shared::cta address `a` in cluster CTA `rank`
__device__ __forceinline__ unsigned mapa_shared(unsigned a, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// arrive on a barrier of another CTA of the cluster.  The only data handed over this way is TMEM, which the
// arriving warp has finished reading (tcgen05.wait::ld) before it arrives, so CTA-scope release suffices.
__device__ __forceinline__ void mbar_arrive_cluster(unsigned cluster_addr) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
// tile loads into this CTA's shared memory whose completion is counted on the even CTA's barrier
__device__ __forceinline__ void tma_load_5d_pair(void *dst, const CUtensorMap *map, unsigned bar_cluster, int c0, int c1,
                                                 int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
      "%5, %6, %7}], [%2];" ::"r"(su32(dst)),
      "l"(map), "r"(bar_cluster), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d_pair(void *dst, const CUtensorMap *map, unsigned bar_cluster, int c0, int c1,
                                                 int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
      "%5}], [%2];" ::"r"(su32(dst)),
      "l"(map), "r"(bar_cluster), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *map, unsigned bar_cluster, int c0,
                                                 int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
      "[%2];" ::"r"(su32(dst)),
      "l"(map), "r"(bar_cluster), "r"(c0), "r"(c1)
      : "memory");
}
__device__ __forceinline__ void mma_f16_pair(unsigned d_tmem, unsigned long long da, unsigned long long db,
                                             unsigned idesc, unsigned accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}
// arrive on the barrier at this shared::cta offset in both CTAs of the pair once the issued MMAs complete
__device__ __forceinline__ void mma_commit_pair_both(unsigned long long *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          su32(bar)),
      "h"((unsigned short)3)
      : "memory");
}
__device__ __forceinline__ void mma_commit_pair_local(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(unsigned taddr, unsigned *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// add N accumulator columns starting at TMEM address taddr (a multiple of 16 columns) into acc[0..N):
// BATCH loads of 16 columns in flight per wait
template <int N, int BATCH = 1>
__device__ __forceinline__ void drain_cols(unsigned taddr, float *acc) {
  static_assert(N % 16 == 0, "drained in groups of 16 columns");
#pragma unroll
  for (int c0 = 0; c0 < N; c0 += 16 * BATCH) {
    unsigned r[16 * BATCH];
#pragma unroll
    for (int b = 0; b < BATCH; ++b)
      if (c0 + 16 * b < N) tmem_ld16(taddr + c0 + 16 * b, r + 16 * b);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int b = 0; b < BATCH; ++b)
      if (c0 + 16 * b < N) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          // the loaded registers are read only after the wait
          asm volatile("" : "+r"(r[16 * b + i]));
          acc[c0 + 16 * b + i] += __uint_as_float(r[16 * b + i]);
        }
      }
  }
}

// atomically add sc * acc[I0, I1) to dst[0, I1 - I0), the first lim of them (the nodes that exist).  Each
// addition is one instruction group on the base address plus a constant offset, so that neither the
// 64-bit addresses nor the FP64 products of a whole run are held in registers at once.
template <int K>
__device__ __forceinline__ void red_add_f64(double *dst, float v, double sc, int lim) {
  if (K < lim)
    asm volatile("{\n .reg .f64 t;\n cvt.f64.f32 t, %1;\n mul.rn.f64 t, t, %2;\n red.global.add.f64 [%0+%3], t;\n}\n" ::"l"(
                     dst),
                 "f"(v), "d"(sc), "n"(8 * K)
                 : "memory");
}
template <int I0, int... K>
__device__ __forceinline__ void flush_seq(const float *acc, double *dst, int lim, double sc,
                                          std::integer_sequence<int, K...>) {
  (red_add_f64<K>(dst, acc[I0 + K], sc, lim), ...);
}
template <int I0, int I1>
__device__ __forceinline__ void flush_cols(const float *acc, double *dst, int lim, double sc) {
  flush_seq<I0>(acc, dst, lim, sc, std::make_integer_sequence<int, I1 - I0>{});
}

// registers move from warpgroup 0 (producer and MMA issuers) to the epilogue warpgroups; each call sits at
// the top of its warpgroup's branch, so that the compiler allocates each role within its own limit
template <bool SPLIT>
__device__ __forceinline__ void give_registers() {
  if constexpr (SPLIT) asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REG_LOW));
}
template <bool SPLIT>
__device__ __forceinline__ void take_registers() {
  if constexpr (SPLIT) asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(REG_HIGH));
}

// The source box of transfer vector e for an item: parity grid sp, half-grid origin (ox, oy, oz), operator
// slot.  Every warp role derives the same box, and skips the transfer vectors whose source box is empty
// (those A tiles are all zero) and the items whose target tile is empty, so that sparse trees (surface or
// clustered distributions) cost only their occupied tiles.
struct SrcBox {
  int sp, ox, oy, oz, slot;
};
// bz: the target tile's z index (an item's tile, or in CTA pairs the item's tile + the CTA's rank)
__device__ __forceinline__ SrcBox src_box(const TcParams &P, const TcItem &w, int bz, int e) {
  const int c = w.parity;
  const int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;
  const int dx = P.off[c][e][0], dy = P.off[c][e][1], dz = P.off[c][e][2];
  SrcBox b;
  b.sp = (((cx + dx) & 1) << 2) | (((cy + dy) & 1) << 1) | ((cz + dz) & 1);
  b.ox = w.bx * TILE_X + ((cx + dx) >> 1);
  b.oy = w.by * TILE_Y + ((cy + dy) >> 1);
  b.oz = bz * TILE_Z + ((cz + dz) >> 1);
  b.slot = P.slot[c][e];
  return b;
}
__device__ __forceinline__ long long tile_id(const TcParams &P, int level, int parity, int bx, int by, int bz) {
  const TcLevel &L = P.lv[level];
  const int TX = L.HX / TILE_X, TY = L.HY / TILE_Y, TZ = L.HZ / TILE_Z;
  return L.tile0 + (((long long)parity * TZ + bz) * TY + by) * TX + bx;
}
// the busy mask of an item's tile, read once per item by every role
struct BusyMask {
  unsigned w[6];
  __device__ __forceinline__ bool tile() const { return (w[5] >> 31) & 1u; }
  __device__ __forceinline__ unsigned word(int k) const {
    return k == 0 ? w[0] : k == 1 ? w[1] : k == 2 ? w[2] : k == 3 ? w[3] : k == 4 ? w[4] : w[5];
  }
  __device__ __forceinline__ bool src(int e) const { return (word(e >> 5) >> (e & 31)) & 1u; }
};
// G: the launch may hold compacted blocks (kernels without them compile the tile form alone)
template <bool G = true>
__device__ __forceinline__ BusyMask busy_mask(const TcParams &P, const TcItem &w) {
  const unsigned *m = (G && w.blk >= 0) ? P.cbusy + 6LL * (P.lv[w.level].cb0 + w.blk)
                                 : P.busy + 6 * tile_id(P, w.level, w.parity, w.bx, w.by, w.bz);
  BusyMask b;
#pragma unroll
  for (int k = 0; k < 6; ++k) b.w[k] = m[k];
  return b;
}
// CTA pairs work on the z-adjacent tiles bz and bz + 1 (bz even) with the same transfer vectors: a pair skips
// a transfer vector (or the item) only when it is idle for both tiles.  A level with an odd number of z tiles
// has no tile bz + 1 in its last pair; that tile's A boxes lie outside the grid (zero-filled loads) and its
// rows map to no cell.
template <bool G = true>
__device__ __forceinline__ BusyMask busy_mask_pair(const TcParams &P, const TcItem &w) {
  BusyMask b = busy_mask<G>(P, w);
  if (G && w.blk >= 0) {
    // compacted blocks come in pairs of one parity: block blk + 1 always exists (possibly without cells)
    const unsigned *m = P.cbusy + 6LL * (P.lv[w.level].cb0 + w.blk + 1);
#pragma unroll
    for (int k = 0; k < 6; ++k) b.w[k] |= m[k];
  } else if (w.bz + 1 < P.lv[w.level].HZ / TILE_Z) {
    const unsigned *m = P.busy + 6 * tile_id(P, w.level, w.parity, w.bx, w.by, w.bz + 1);
#pragma unroll
    for (int k = 0; k < 6; ++k) b.w[k] |= m[k];
  }
  return b;
}

template <bool G = true>
__device__ __forceinline__ TcItem decode_unit(const TcParams &P, int u) {
  int level = P.l1;
  while (level > P.l0 && u >= P.lv[level].unit0 + P.lv[level].nunits) --level;
  const TcLevel &L = P.lv[level];
  const int TX = L.HX / TILE_X, TY = L.HY / TILE_Y;
  int r = u - L.unit0;
  TcItem w;
  w.level = level;
  if (G && L.cmode) {
    // one right-hand side; blocks of parity p are [cblk0[p], cblk0[p + 1])
    w.rhs = 0;
    w.bx = w.by = w.bz = 0;
    w.blk = r * (P.pair ? 2 : 1);
    int p = 0;
#pragma unroll
    for (int q = 1; q < 8; ++q) p += w.blk >= L.cblk0[q] ? 1 : 0;
    w.parity = p;
    return w;
  }
  w.blk = -1;
  w.bx = r % TX;
  r /= TX;
  w.by = r % TY;
  r /= TY;
  w.bz = (r % L.TZu) * (P.pair ? 2 : 1);
  r /= L.TZu;
  w.parity = r & 7;
  w.rhs = r >> 3;
  return w;
}
// Every role walks the same sequence of unit fragments; f(w, r0, r1) handles the busy transfer vectors of
// ranks [r0, r1) of unit w and returns false to stop.
//   * Dense launches (every unit has all 189 transfer vectors busy, as in uniform trees): waves of whole
//     units, unit u_begin + g + m G for CTA (pair) g, so that all CTAs stream the same transfer vector's
//     operator at about the same time and share it through L2; the units left over after the last whole wave
//     are split into G ranges of equal work, one per CTA.
//   * Otherwise: the work of all units is split into G * ranges_per_cta ranges of equal work; CTA g takes
//     ranges g, g + G, ...
template <bool G, class F>
__device__ __forceinline__ bool range_fragments(const TcParams &P, long long lo, long long hi, int u_from, F &f) {
  if (lo >= hi) return true;
  int a = u_from, b = P.u_end;  // the largest unit whose work starts at or before lo
  while (b - a > 1) {
    const int m = (a + b) >> 1;
    if (P.prefix[m] <= lo) a = m; else b = m;
  }
  for (int u = a; u < P.u_end; ++u) {
    const long long p0 = P.prefix[u], p1 = P.prefix[u + 1];
    if (p0 >= hi) break;
    const int r0 = (int)(max(lo, p0) - p0), r1 = (int)(min(hi, p1) - p0);
    if (r1 <= r0) continue;
    if (!f(decode_unit<G>(P, u), r0, r1)) return false;
  }
  return true;
}
template <bool GA, class F>
__device__ __forceinline__ void for_each_fragment(const TcParams &P, int g, int G, F &&f) {
  const int U = P.u_end - P.u_begin;
  const long long base = P.prefix[P.u_begin], W = (long long)P.prefix[P.u_end] - base;
  if (W == 189LL * U) {
    const int nwave = U / G;
    for (int m = 0; m < nwave; ++m)
      if (!f(decode_unit<GA>(P, P.u_begin + g + m * G), 0, 189)) return;
    const int ut = P.u_begin + nwave * G;
    const long long tb = P.prefix[ut], tw = (long long)P.prefix[P.u_end] - tb;
    range_fragments<GA>(P, tb + tw * g / G, tb + tw * (g + 1) / G, ut, f);
    return;
  }
  const int nr = G * P.ranges_per_cta;
  for (int m = 0; m < P.ranges_per_cta; ++m) {
    const int j = g + m * G;
    if (!range_fragments<GA>(P, base + W * j / nr, base + W * (j + 1) / nr, P.u_begin, f)) return;
  }
}

// ---- the kernel -------------------------------------------------------------------------------------
// CW: accumulator columns owned by one epilogue thread (NP / 2) and NHALF: MMA column halves, compile-time
// constants so that the running sums stay in registers.  With one half a thread owns the columns
// [ch*CW, (ch+1)*CW).  With two halves of NH = CW columns each, split at SPLIT = 16 * ceil(CW / 32) so that
// every TMEM load starts on a multiple of 16 columns, the part-0 warps own [0, SPLIT) of half 0 and
// [0, CW - SPLIT) of half 1, the part-1 warps [SPLIT, CW) of half 0 and [CW - SPLIT, CW) of half 1
// (columns counted from the start of each half).
//
// Overlap of the segment drains with the MMAs: with two TMEM accumulators (orders <= 6) the MMA of segment
// s+1 runs in the other accumulator while segment s drains.  With one (order 7: 352 of 512 columns) the
// epilogue drains half 0 first and releases it, and the first chunk of the next segment issues all its
// half-0 MMAs before waiting for half 1.
//
// PAIR: clusters of two CTAs on the z-adjacent tiles (bz, bz + 1) of an item share each operator chunk
// through cta_group::2 MMAs (M = 256).  Each CTA loads its own A tile and half of the chunk's B rows, so a
// CTA reads 16 KB of A and NP / 2 rows of B per K chunk instead of all NP rows.  The even CTA's producer
// expects both CTAs' bytes on its full barrier, its MMA warp issues all MMAs, and the commits arrive on the
// stage and accumulator barriers of both CTAs; the epilogue warps of both CTAs release the accumulator on
// the even CTA's barriers (16 arrivals).
template <int CW, int NHALF, bool PAIR, bool LR, bool GATHER>
__global__ void __launch_bounds__(TC_THREADS, 1) m2l_tc_kernel(const __grid_constant__ TcParams P) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned stage buffers (the swizzle pattern repeats every 512 B)
  unsigned char *smem = (unsigned char *)(((unsigned long long)smem_raw + 1023) & ~1023ull);
  __shared__ __align__(8) unsigned long long full_bar[MAX_STAGES], empty_bar[MAX_STAGES];
  __shared__ __align__(8) unsigned long long gfull_bar[MAX_STAGES];  // odd CTA of a pair: its gathers landed
  __shared__ __align__(8) unsigned long long acc_full[2][2], acc_empty[2][2], done_bar;
  __shared__ unsigned tmem_base_sh;
  __shared__ volatile int abort_sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = P.stages;
  const unsigned rank = PAIR ? cluster_rank() : 0u;
  const bool leader = rank == 0;
  // the work ranges of this CTA, or of this CTA pair
  const int g_id = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
  const int g_count = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;
  if (threadIdx.x == 0) {
    // A stage is full once the producer's expected bytes have landed and, in a launch with compacted blocks,
    // once the 32 gathering lanes of this CTA have arrived (each after its own copies landed) and, in a pair,
    // the odd CTA's relay has arrived for that CTA's gathers.
    const unsigned full_count = GATHER ? (PAIR ? 34u : 33u) : 1u;
    for (int s = 0; s < S; ++s) {
      mbar_init(&full_bar[s], full_count);
      mbar_init(&gfull_bar[s], 32);
      mbar_init(&empty_bar[s], NHALF);  // one commit per MMA issuer
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b][0], 1);
      mbar_init(&acc_full[b][1], 1);
      mbar_init(&acc_empty[b][0], PAIR ? 16 : 8);  // one arrive per epilogue warp (of both CTAs)
      mbar_init(&acc_empty[b][1], PAIR ? 16 : 8);
    }
    mbar_init(&done_bar, NHALF);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // the transfer-vector records, behind the stage buffers
  TvRec *tvs = (TvRec *)(smem + (size_t)S * P.stage_bytes);
  for (int i = threadIdx.x; i < 8 * 189; i += blockDim.x) tvs[i] = P.tv[i];
  if (warp == 1) {
    if constexpr (PAIR) {
      // both CTAs' warp 1 allocate together; the same columns are allocated in each CTA's TMEM
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_sh)),
                   "r"(P.ncols));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    } else {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_sh)),
                   "r"(P.ncols));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
  }
  tc_fence_before();
  __syncthreads();
  if constexpr (PAIR) cluster_sync_all();  // the peer's barriers are initialised before any remote arrival
  tc_fence_after();
  const unsigned tmem = tmem_base_sh;
  constexpr bool SPLIT_REGS = CW >= 112;  // running sums of CW columns per epilogue thread
  // a role that gives up marks the status word and stops both CTAs of a pair
  auto give_up = [&]() {
    atomicExch(P.status + 1, 1);
    abort_sh = 1;
    if constexpr (PAIR)
      asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(mapa_shared(su32((const void *)&abort_sh), rank ^ 1u)),
                   "r"(1)
                   : "memory");
  };
  auto wait_bar = [&](unsigned long long *b, unsigned parity) -> bool { return mbar_wait(b, parity); };
  auto item_mask = [&](const TcItem &w) -> BusyMask {
    if constexpr (PAIR) return busy_mask_pair<GATHER>(P, w);
    return busy_mask<GATHER>(P, w);
  };

  constexpr int KCH = LR ? 16 : KCHUNK;  // fp16 per K chunk: 16 (32-byte rows) or 32 (64-byte rows)
  constexpr int ROWB = KCH * 2;
  const int a_bytes = TILE_X * TILE_Y * TILE_Z * ROWB;  // 4 or 8 KB
  const int nb_rows = PAIR ? P.NH / 2 : P.NH;           // B rows of one column half in this CTA
  const int b_bytes = NHALF * nb_rows * ROWB;

  if (warp < 4) {
  give_registers<SPLIT_REGS>();
  if (warp == 0) {
    // ------------------------------------------------ TMA producer (both CTAs of a pair)
    if (lane == 0) {
      int stage = 0;
      unsigned phase = 0;
      // the barrier that counts this stage's bytes: this CTA's, or the even CTA's in a pair
      const unsigned full0 = PAIR ? mapa_shared(su32(&full_bar[0]), 0u) : su32(&full_bar[0]);
      const int stage_tx = (PAIR ? 2 : 1) * (2 * a_bytes + 2 * b_bytes);
      const int stage_tx_b = (PAIR ? 2 : 1) * 2 * b_bytes;  // compacted blocks: the A rows are gathered
      unsigned loaded = 0, lpar = 0;  // stages that received a load, and the phase parity of the last one
      for_each_fragment<GATHER>(P, g_id, g_count, [&](const TcItem &w, int r0, int r1) -> bool {
        const BusyMask bm = item_mask(w);
        const int bz = w.bz + (int)rank;
        int rank_e = 0;
        for (int e = 0; e < 189 && rank_e < r1 && !abort_sh; ++e) {
          if (!bm.src(e)) continue;
          if (rank_e++ < r0) continue;
          // K chunks of this transfer vector and the coordinates of its A and B boxes: dense (K offset,
          // rhs and source parity, operator slot) or low rank (Y chunk and U chunk of the slot)
          const TvRec tr = tvs[w.parity * 189 + e];
          const int ox = w.bx * TILE_X + tr.ox, oy = w.by * TILE_Y + tr.oy, oz = bz * TILE_Z + tr.oz;
          const int nk = LR ? (int)tr.nk : P.NK;
          const int a4 = w.rhs * (LR ? P.ycht : 8) + tr.ya;
          const int b2 = tr.ub;
          for (int kc = 0; kc < nk; ++kc) {
            if (!wait_bar(&empty_bar[stage], phase ^ 1)) {
              give_up();
              break;
            }
            unsigned char *sbuf = smem + (size_t)stage * P.stage_bytes;
            if (leader) mbar_expect_tx(&full_bar[stage], (GATHER && w.blk >= 0) ? stage_tx_b : stage_tx);
            const int k0 = LR ? 0 : kc * KCHUNK;  // K coordinate of the boxes
            const int c4 = LR ? a4 + kc : a4;
            const int c2 = LR ? b2 + kc : b2;
            if constexpr (PAIR) {
              const unsigned fb = full0 + 8u * (unsigned)stage;
              if (!GATHER || w.blk < 0) {
                tma_load_5d_pair(sbuf, &P.mapA_hi[w.level], fb, k0, ox, oy, oz, c4);
                tma_load_5d_pair(sbuf + a_bytes, &P.mapA_lo[w.level], fb, k0, ox, oy, oz, c4);
              }
              for (int h = 0; h < NHALF; ++h) {
                const int row0 = h * P.NH + (int)rank * nb_rows;
                tma_load_3d_pair(sbuf + 2 * a_bytes + h * nb_rows * ROWB, &P.mapB_hi, fb, k0, row0, c2);
                tma_load_3d_pair(sbuf + 2 * a_bytes + b_bytes + h * nb_rows * ROWB, &P.mapB_lo, fb, k0, row0, c2);
              }
            } else {
              if (!GATHER || w.blk < 0) {
                tma_load_5d(sbuf, &P.mapA_hi[w.level], &full_bar[stage], k0, ox, oy, oz, c4);
                tma_load_5d(sbuf + a_bytes, &P.mapA_lo[w.level], &full_bar[stage], k0, ox, oy, oz, c4);
              }
              for (int h = 0; h < NHALF; ++h) {
                tma_load_3d(sbuf + 2 * a_bytes + h * nb_rows * ROWB, &P.mapB_hi, &full_bar[stage], k0, h * P.NH, c2);
                tma_load_3d(sbuf + 2 * a_bytes + b_bytes + h * nb_rows * ROWB, &P.mapB_lo, &full_bar[stage], k0,
                            h * P.NH, c2);
              }
            }
            loaded |= 1u << stage;
            lpar = (lpar & ~(1u << stage)) | (phase << stage);
            if (++stage == S) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
        return !abort_sh;
      });
      // No bulk copy may still be landing in shared memory when the CTA exits, which a run that gave up can
      // leave behind: wait (bounded) for the last load of every stage.  The even CTA's barriers count the bytes
      // of both CTAs of a pair, and the cluster barrier at the end holds the odd CTA until then.
      if (leader)
        for (int st = 0; st < S; ++st)
          if ((loaded >> st) & 1u) mbar_wait(&full_bar[st], (lpar >> st) & 1u);
    }
  } else if (warp == 1 || (NHALF == 2 && warp == 2)) {
    // ------------------------------------------------ MMA issuers (the even CTA of a pair)
    // With two column halves each half has its own issuing thread (warp 1: half 0, warp 2: half 1), so
    // that each thread issues 6 MMAs per K chunk and each half drains while the other half's MMAs run.
    const int hh = warp == 1 ? 0 : 1;
    if (lane == 0 && leader) {
      const unsigned idesc =
          (1u << 4) | ((unsigned)(P.NH >> 3) << 17) | ((unsigned)((PAIR ? 256 : 128) >> 4) << 24);
      // descriptors of stage 0's operands: another stage, K step or column half adds (byte offset >> 4) to
      // the 14-bit start-address field, which never carries (shared addresses stay below 2^18 bytes)
      const unsigned long long dA_hi = LR ? sdesc32(smem) : sdesc(smem), dA_lo = dA_hi + (unsigned)(a_bytes >> 4);
      const unsigned long long dB_hi = dA_hi + (unsigned)((2 * a_bytes) >> 4), dB_lo = dB_hi + (unsigned)(b_bytes >> 4);
      const unsigned stage_step = (unsigned)P.stage_bytes >> 4;
      const unsigned half_step = (unsigned)(nb_rows * ROWB) >> 4;
      int stage = 0;
      unsigned phase = 0;
      auto commit = [&](unsigned long long *bar) {
        if constexpr (PAIR)
          mma_commit_pair_both(bar);
        else
          mma_commit(bar);
      };
      // the 6 MMAs of one column half of the K chunk in stage st: D += A_hi B_lo + A_lo B_hi + A_hi B_hi
      // (the small cross terms first, the leading term last); `first` starts a new accumulation
      auto issue_half = [&](int st, int h, unsigned d, bool first) {
        const unsigned so = (unsigned)st * stage_step;
        const unsigned bo = so + (unsigned)h * half_step;
#pragma unroll
        for (int ks = 0; ks < KCH / 16; ++ks) {
          const unsigned k2 = 2u * ks;  // 16 fp16 = 32 bytes of K
          if constexpr (PAIR) {
            mma_f16_pair(d, dA_hi + so + k2, dB_lo + bo + k2, idesc, (first && ks == 0) ? 0u : 1u);
            mma_f16_pair(d, dA_lo + so + k2, dB_hi + bo + k2, idesc, 1u);
            mma_f16_pair(d, dA_hi + so + k2, dB_hi + bo + k2, idesc, 1u);
          } else {
            mma_f16(d, dA_hi + so + k2, dB_lo + bo + k2, idesc, (first && ks == 0) ? 0u : 1u);
            mma_f16(d, dA_lo + so + k2, dB_hi + bo + k2, idesc, 1u);
            mma_f16(d, dA_hi + so + k2, dB_hi + bo + k2, idesc, 1u);
          }
        }
      };
      // the next stage in order once its operands have landed, or -1
      auto next_full = [&]() -> int {
        // a pair's stages with gathered rows are completed by the odd CTA's release arrival
        if (!((PAIR && GATHER) ? mbar_wait_cluster(&full_bar[stage], phase) : wait_bar(&full_bar[stage], phase))) {
          give_up();
          return -1;
        }
        const int st = stage;
        if (++stage == S) {
          stage = 0;
          phase ^= 1;
        }
        return st;
      };
      unsigned empty_par = 0xFu;  // parity to wait for, per (buffer, half): starts at 1 (passes at once)
      int seg = 0;
      for_each_fragment<GATHER>(P, g_id, g_count, [&](const TcItem &w, int r0, int r1) -> bool {
        if constexpr (LR) {
          // low rank: the fragment's K chunks (1..3 per transfer vector) form one stream, cut into
          // segments of lr_seglen chunks; with two column halves both issuers cut it at the same places
          const BusyMask bm = item_mask(w);
          int cs = 0;  // chunks issued in the open segment
          int b = 0;   // its accumulator (one column half: two alternate when they fit)
          int rank_e = 0;
          for (int e = 0; e < 189 && rank_e < r1 && !abort_sh; ++e) {
            if (!bm.src(e)) continue;
            if (rank_e++ < r0) continue;
            const int nk = tvs[w.parity * 189 + e].nk;
            for (int kc = 0; kc < nk && !abort_sh; ++kc) {
              if (cs == 0) {
                const int hb = NHALF == 2 ? 0 : (P.nbuf == 2 ? (seg & 1) : 0);
                const int bit = NHALF == 2 ? hh : 2 * hb;
                if (!wait_bar(&acc_empty[hb][NHALF == 2 ? hh : 0], (empty_par >> bit) & 1u)) {
                  give_up();
                  break;
                }
                empty_par ^= 1u << bit;
                b = hb;
                tc_fence_after();
              }
              const int st = next_full();
              if (st < 0) break;
              if constexpr (NHALF == 2)
                issue_half(st, hh, tmem + (unsigned)(hh * P.NH), cs == 0);
              else
                issue_half(st, 0, tmem + (unsigned)(b * P.NP), cs == 0);
              commit(&empty_bar[st]);
              if (++cs == P.lr_seglen) {
                commit(&acc_full[b][NHALF == 2 ? hh : 0]);
                cs = 0;
                ++seg;
              }
            }
          }
          if (cs > 0 && !abort_sh) {
            commit(&acc_full[b][NHALF == 2 ? hh : 0]);
            ++seg;
          }
          return !abort_sh;
        }
        // every MMA of a fragment runs the same schedule: only the count of transfer vectors matters here
        (void)w;
        for (int ev = r0; ev < r1 && !abort_sh; ++ev) {
          for (int sg = 0; sg < P.nseg && !abort_sh; ++sg, ++seg) {
            const int k0 = sg * P.NK / P.nseg, k1 = (sg + 1) * P.NK / P.nseg;
            if constexpr (NHALF == 1) {
              // one accumulator per segment, alternating between two when they fit
              const int b = P.nbuf == 2 ? (seg & 1) : 0;
              if (!wait_bar(&acc_empty[b][0], (empty_par >> (2 * b)) & 1u)) {
                give_up();
                break;
              }
              empty_par ^= 1u << (2 * b);
              tc_fence_after();
              for (int kc = k0; kc < k1; ++kc) {
                const int st = next_full();
                if (st < 0) break;
                issue_half(st, 0, tmem + (unsigned)(b * P.NP), kc == k0);
                commit(&empty_bar[st]);  // frees the stage (in both CTAs) once these MMAs have read it
              }
              commit(&acc_full[b][0]);  // segment accumulated
            } else {
              // one accumulator of two column halves (order 7): this thread's half
              if (!wait_bar(&acc_empty[0][hh], (empty_par >> hh) & 1u)) {
                give_up();
                break;
              }
              empty_par ^= 1u << hh;
              tc_fence_after();
              for (int kc = k0; kc < k1; ++kc) {
                const int st = next_full();
                if (st < 0) break;
                issue_half(st, hh, tmem + (unsigned)(hh * P.NH), kc == k0);
                commit(&empty_bar[st]);
              }
              commit(&acc_full[0][hh]);
            }
          }
        }
        return !abort_sh;
      });
      // every MMA issued here has completed before the CTAs (and their TMEM) are released
      if constexpr (PAIR)
        mma_commit_pair_local(&done_bar);
      else
        mma_commit(&done_bar);
      if (!wait_bar(&done_bar, 0)) give_up();
    }
    if (GATHER && PAIR && !leader && warp == 1 && lane == 0) {
      // ------------------------------------------------ relay (odd CTA of a pair)
      // The gathering lanes can only arrive on this CTA's own barriers: once a stage's rows of this CTA have
      // landed (gfull), one release arrival on the even CTA's full barrier hands them over, stage by stage.
      const unsigned full0r = mapa_shared(su32(&full_bar[0]), 0u);
      int stage = 0;
      unsigned phase = 0;
      for_each_fragment<GATHER>(P, g_id, g_count, [&](const TcItem &w, int r0, int r1) -> bool {
        const BusyMask bm = item_mask(w);
        int rank_e = 0;
        for (int e = 0; e < 189 && rank_e < r1 && !abort_sh; ++e) {
          if (!bm.src(e)) continue;
          if (rank_e++ < r0) continue;
          const int nk = LR ? (int)tvs[w.parity * 189 + e].nk : P.NK;
          for (int kc = 0; kc < nk; ++kc) {
            if (!wait_bar(&gfull_bar[stage], phase)) {
              give_up();
              break;
            }
            mbar_arrive_cluster_release(full0r + 8u * (unsigned)stage);
            if (++stage == S) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
        return !abort_sh;
      });
    }
  } else if (GATHER && warp == 3) {
    // ------------------------------------------------ row gathers of compacted blocks (all 32 lanes)
    // A compacted block's A tile holds, for transfer vector e, the source row of each of its 128 cells: the
    // cell's half-grid position shifted by the box offset of e, in the source parity's grid.  Rows outside the
    // grid are zero-filled, as the TMA boxes of the tile form read them, and so are, where Y is stored by
    // compacted row, the positions without a cell.  Lane l copies rows l, l + 32, l + 64, l + 96 in 16-byte
    // pieces, placed where the TMA unit's 32- or 64-byte swizzle would put them, and arrives once its copies
    // have landed.  Stages of grid tiles (TMA-loaded A) get the 32 arrivals at once.  Half-grid coordinates
    // are packed in 10 bits each (levels up to 11).
    constexpr int PPR = ROWB / 16;                     // 16-byte pieces per row: 2 or 4
    constexpr int SWZ_SHIFT = ROWB == 32 ? 2 : 1;      // row bits that select the XOR of the piece index
    unsigned long long *gbar = (PAIR && !leader) ? gfull_bar : full_bar;
    int stage = 0;
    unsigned phase = 0;
    for_each_fragment<GATHER>(P, g_id, g_count, [&](const TcItem &w, int r0, int r1) -> bool {
      const BusyMask bm = item_mask(w);
      const bool cmp = w.blk >= 0;
      const TcLevel &Lv = P.lv[w.level];
      unsigned hc[4];  // this lane's rows: half-grid x | y << 10 | z << 20, or ~0u for no cell
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        hc[i] = ~0u;
        if (cmp) {
          const int code = Lv.crow[(long long)(w.blk + (int)rank) * 128 + lane + 32 * i];
          if (code >= 0) {
            const int pos = code & 0x0FFFFFFF;
            const int yz = pos / Lv.HX;
            hc[i] = (unsigned)(pos - yz * Lv.HX) | ((unsigned)(yz % Lv.HY) << 10) | ((unsigned)(yz / Lv.HY) << 20);
          }
        }
      }
      bool stop = false;
      int rank_e = 0;
      for (int e = 0; e < 189 && rank_e < r1 && !stop; ++e) {
        if (!bm.src(e)) continue;
        if (rank_e++ < r0) continue;
        const TvRec tr = tvs[w.parity * 189 + e];
        const int nk = LR ? (int)tr.nk : P.NK;
        // this lane's source rows under e: a grid position, or (Y stored by compacted row) the cell's row;
        // -1 where the source lies outside the grid or holds no cell
        int srow[4];
        {
          const int c = w.parity;
          const int sp = ((((c >> 2) & 1) + P.off[c][e][0]) & 1) << 2 | ((((c >> 1) & 1) + P.off[c][e][1]) & 1) << 1 |
                         (((c & 1) + P.off[c][e][2]) & 1);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int x = (int)(hc[i] & 1023u) + tr.ox, y = (int)((hc[i] >> 10) & 1023u) + tr.oy,
                      z = (int)(hc[i] >> 20) + tr.oz;
            const bool in = hc[i] != ~0u && x >= 0 && x < Lv.HX && y >= 0 && y < Lv.HY && z >= 0 && z < Lv.HZ;
            const int pos = (z * Lv.HY + y) * Lv.HX + x;
            srow[i] = in ? pos : -1;
            if (LR && Lv.ypr > 0 && in) srow[i] = Lv.rowmap[(long long)sp * Lv.plane + pos];
          }
        }
        for (int kc = 0; kc < nk; ++kc) {
          // lane 0 waits for the stage to be free; the warp follows its outcome
          int ok = 1;
          if (lane == 0) ok = wait_bar(&empty_bar[stage], phase ^ 1) ? 1 : 0;
          ok = __shfl_sync(0xffffffffu, ok, 0);
          if (!ok) {
            if (lane == 0) give_up();
            stop = true;
            break;
          }
          const unsigned bar = su32(&gbar[stage]);
          if (cmp) {
            const unsigned sa = su32(smem + (size_t)stage * P.stage_bytes);
            // the rows of this K chunk: Y chunk tr.ya + kc of the source parity (low rank; by grid position or
            // by compacted row), or the source parity's multipoles at K offset kc * 32 (dense); row numbers fit
            // 32 bits (checked on the host)
            const int rows_per = (LR && Lv.ypr > 0) ? Lv.ypr : (int)Lv.plane;
            const int grow0 = (w.rhs * (LR ? P.ycht : 8) + tr.ya + (LR ? kc : 0)) * rows_per;
            const int kel = LR ? 0 : kc * KCHUNK;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const int r = lane + 32 * i;
              const bool v = srow[i] >= 0;
              const long long o = v ? (long long)(grow0 + srow[i]) * P.growlen + kel : 0;
              const unsigned nb = v ? 16u : 0u;
#pragma unroll
              for (int j = 0; j < PPR; ++j) {
                const unsigned d = sa + (unsigned)(r * ROWB) + ((unsigned)(j ^ ((r >> SWZ_SHIFT) & (PPR - 1))) << 4);
                cp_async16(d, Lv.ghi + o + 8 * j, nb);
                cp_async16(d + (unsigned)a_bytes, Lv.glo + o + 8 * j, nb);
              }
            }
            cp_async_arrive_noinc(bar);
          } else {
            __syncwarp();
            if (lane == 0) mbar_arrive_n(bar, 32);
          }
          if (++stage == S) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
      stop = __any_sync(0xffffffffu, stop || abort_sh != 0);
      return !stop;
    });
    // no copy of this warp may still be landing when the CTA exits
    cp_async_wait_all();
  }
  } else {
    take_registers<SPLIT_REGS>();
    // ------------------------------------------------ epilogue (warps 4..11 of both CTAs)
    constexpr int SPLIT = 16 * ((CW + 31) / 32);
    constexpr int BATCH = SPLIT_REGS ? 2 : 1;  // TMEM loads in flight per wait
    const int q = warp & 3;              // TMEM lane quarter this warp may access
    const int ch = (warp - 4) >> 2;      // which part of each half
    const int row = q * 32 + lane;       // target within the tile
    const unsigned tlane = tmem + ((unsigned)(q * 32) << 16);
    // the accumulator is released on the even CTA's barriers
    const unsigned empty0 = PAIR ? mapa_shared(su32(&acc_empty[0][0]), 0u) : 0u;
    auto release = [&](int b, int h) {
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        if constexpr (PAIR)
          mbar_arrive_cluster(empty0 + 8u * (unsigned)(b * 2 + h));
        else
          mbar_arrive(&acc_empty[b][h]);
      }
    };
    unsigned full_par = 0;
    int seg = 0;
    float acc[CW];
#pragma unroll
    for (int i = 0; i < CW; ++i) acc[i] = 0.f;
    for_each_fragment<GATHER>(P, g_id, g_count, [&](const TcItem &w, int r0, int r1) -> bool {
      // accumulator segments of this fragment: nseg per transfer vector, or (low rank) one per lr_seglen
      // K chunks of the fragment's chunk stream
      int nseg_item = (r1 - r0) * P.nseg;
      if constexpr (LR) {
        const BusyMask bm = item_mask(w);
        int nch = 0, rank_e = 0;
        for (int e = 0; e < 189 && rank_e < r1; ++e) {
          if (!bm.src(e)) continue;
          if (rank_e++ >= r0) nch += tvs[w.parity * 189 + e].nk;
        }
        nseg_item = (nch + P.lr_seglen - 1) / P.lr_seglen;
      }
      for (int sgi = 0; sgi < nseg_item; ++sgi, ++seg) {
        if constexpr (NHALF == 1) {
          const int b = P.nbuf == 2 ? (seg & 1) : 0;
          if (!mbar_wait_warp(&acc_full[b][0], (full_par >> b) & 1u)) {
            give_up();
            break;
          }
          full_par ^= 1u << b;
          tc_fence_after();
          drain_cols<CW, BATCH>(tlane + (unsigned)(b * P.NP) + ch * CW, acc);
          release(b, 0);
        } else {
          // each half is committed on its own barrier.  Both parts drain G = CW - SPLIT columns of each
          // half into acc[0, G) and acc[SPLIT, CW); the remaining 16-column group, acc[G, SPLIT), comes from
          // half 0 for part 0 and half 1 for part 1
          constexpr int G = CW - SPLIT;
          static_assert(SPLIT - G == 16, "one extra group of 16 columns");
          if (!mbar_wait_warp(&acc_full[0][0], full_par & 1u)) {
            give_up();
            break;
          }
          full_par ^= 1u;
          tc_fence_after();
          // part 0: half 0 columns [0, SPLIT) -> acc[0, SPLIT); part 1: columns [SPLIT, CW) -> acc[0, G)
          if (ch == 0)
            drain_cols<SPLIT, BATCH>(tlane, acc);
          else
            drain_cols<G, BATCH>(tlane + SPLIT, acc);
          release(0, 0);
          if (!mbar_wait_warp(&acc_full[0][1], (full_par >> 1) & 1u)) {
            give_up();
            break;
          }
          full_par ^= 2u;
          tc_fence_after();
          // part 0: half 1 columns [0, G) -> acc[SPLIT, CW); part 1: columns [G, CW) -> acc[G, CW)
          if (ch == 0)
            drain_cols<G, BATCH>(tlane + CW, acc + SPLIT);
          else
            drain_cols<CW - G, BATCH>(tlane + CW + G, acc + G);
          release(0, 1);
        }
      }
      if (abort_sh) return false;
      // flush the fragment's sums into the FP64 locals
      const TcLevel &Lv = P.lv[w.level];
      int cell = -1;
      if (GATHER && w.blk >= 0) {
        cell = Lv.ccell[(long long)(w.blk + (int)rank) * 128 + row];
      } else {
        const int c = w.parity;
        const int bz = w.bz + (int)rank;
        const int hx = w.bx * TILE_X + (row & 7), hy = w.by * TILE_Y + ((row >> 3) & 3), hz = bz * TILE_Z + (row >> 5);
        const int gx = 2 * hx + ((c >> 2) & 1), gy = 2 * hy + ((c >> 1) & 1), gz = 2 * hz + (c & 1);
        if (gx < Lv.side && gy < Lv.side && gz < Lv.side) cell = Lv.grid[((long long)gz * Lv.side + gy) * Lv.side + gx];
      }
      if (cell >= 0) {
        const double sc = *Lv.scale_out;
        double *Lrow = Lv.L + ((long long)cell * P.R + w.rhs) * P.nn;
        // the runs of accumulator columns this thread holds, each with its first node index
        const int nn = P.nn;
        if constexpr (NHALF == 1) {
          flush_cols<0, CW>(acc, Lrow + ch * CW, nn - ch * CW, sc);
        } else {
          constexpr int G = CW - SPLIT;
          if (ch == 0) {
            flush_cols<0, SPLIT>(acc, Lrow, nn, sc);             // half 0, nodes [0, SPLIT)
            flush_cols<SPLIT, CW>(acc, Lrow + CW, nn - CW, sc);  // half 1, nodes CW + [0, G)
          } else {
            flush_cols<0, G>(acc, Lrow + SPLIT, nn - SPLIT, sc);      // half 0, nodes [SPLIT, CW)
            flush_cols<G, CW>(acc, Lrow + CW + G, nn - CW - G, sc);   // half 1, nodes CW + [G, CW)
          }
        }
      }
#pragma unroll
      for (int i = 0; i < CW; ++i) acc[i] = 0.f;
      return true;
    });
  }
  tc_fence_before();
  __syncthreads();
  // neither CTA of a pair releases its TMEM or exits while the other may still use it
  if constexpr (PAIR) cluster_sync_all();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    if constexpr (PAIR)
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P.ncols));
    else
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P.ncols));
  }
}

// ---- low-rank M2L, first product: Y = V^T M for every source cell --------------------------------------
// For symmetric Chebyshev operators K_t = U_t V_t^T (FChebSymKernel's compression, rank 16..44 at order 7),
// the transfer of a source cell s to a target along slot t is U_t (V_t^T M_s).  Y_t = V_t^T M_s depends on
// the source only, so it is computed once per source cell and slot, for the slots that the cell's parity
// grid feeds: one GEMM per level, parity and 8x4x4 tile of source cells (M = 128 cells, N = 256 rank rows =
// 16 chunks of 16, K = p^3 in chunks of 32), A = the packed multipoles (hi, lo), B = the stacked V_t (hi,
// lo).  The K chunks are cut into segments of segc chunks that alternate between two TMEM accumulators:
// the tensor core's FP32 accumulation truncates, and the columns of V oscillate in sign, so long chains
// would lose accuracy against the partial sums.  The epilogue adds the segments in registers (rounded FP32
// adds) and writes Y as FP16 hi and lo, 16 ranks per chunk, in the parity-split grid layout that the second
// product's TMA boxes read.
struct __align__(64) LrYParams {
  CUtensorMap mapA_hi[kMaxHeight], mapA_lo[kMaxHeight];  // multipoles: 5-D boxes of 32 K x 8x4x4 cells
  CUtensorMap mapV_hi, mapV_lo;                          // V rows: 2-D boxes of 32 K x 256 rows
  __half *Yhi[kMaxHeight], *Ylo[kMaxHeight];             // [R * ycht][HZ][HY][HX][16]
  int HX[kMaxHeight], HY[kMaxHeight], HZ[kMaxHeight];
  int item0[kMaxHeight], nitems[kMaxHeight];             // items of each level, finest level first
  int l0, l1;                                            // levels of this launch
  int R, NK, nblk;                                       // rhs, K chunks, 256-row blocks per parity
  int segc;                                              // K chunks per accumulator segment
  float yscale;                                          // power of two that brings |Y| below 2^15
  int ycht, ybase[9];                                    // Y chunks per rhs; first chunk of each parity
  int stages, stage_bytes;
  int *status;
  // sparse trees: an item whose tile (either tile of a pair) holds no cell is not computed.  Its Y rows must
  // still read as zero for the second product, so ydirty[2 * item + rank] records whether this CTA's tile rows
  // of the item hold values of an earlier computation; those are zeroed once, when the tile has become empty.
  const unsigned *busy;                                  // the second product's tile masks (bit 191: occupied)
  int tile0[kMaxHeight];                                 // first tile of each level in busy
  unsigned full_levels;                                  // bit l: every cell of level l is present
  int issuers;                                           // MMA-issuing threads: 1, or 2 (one per accumulator)
  unsigned char *ydirty;                                 // [2 * items of all levels]
  int dirty0[kMaxHeight];                                // each level's first item in the tile-mode numbering of ydirty
  // Compacted levels (sparse levels, one right-hand side, single CTAs): the items run over blocks of 128
  // occupied cells of one parity instead of the parity grid's tiles, so that a level whose few cells touch
  // most tiles costs its cells, not its grid.
  unsigned compact_levels;                               // bit l: level l is compacted
  CUtensorMap mapC_hi[kMaxHeight], mapC_lo[kMaxHeight];  // compacted multipoles [rows][KP]: 2-D boxes of 32 K x 128 rows
  const int *crow[kMaxHeight];                           // [rows]: (parity << 28) | (hz * HY + hy) * HX + hx, or -1
  int cblk0[kMaxHeight][9];                              // first 128-row block of each parity; [8] = blocks
  // ypr > 0: this compacted level's Y is stored by compacted row, [R * ycht][ypr][16] with the row counted
  // from its parity's first block, instead of by grid position (the second product gathers it by row)
  int ypr[kMaxHeight];
};

constexpr int YBLK = 256;  // rank rows per item (16 chunks of 16)

// PAIR: clusters of two CTAs on the z-adjacent tiles (bz, bz + 1) of an item, M = 256 MMAs (cta_group::2)
// issued by the even CTA, each CTA loading its own tile of multipoles and half of the V block (the same
// protocol as the second product's CTA pairs).
template <bool PAIR>
__global__ void __launch_bounds__(TC_THREADS, 1) lr_y_kernel(const __grid_constant__ LrYParams P) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem = (unsigned char *)(((unsigned long long)smem_raw + 1023) & ~1023ull);
  __shared__ __align__(8) unsigned long long full_bar[MAX_STAGES], empty_bar[MAX_STAGES];
  __shared__ __align__(8) unsigned long long acc_full[2], acc_empty[2], done_bar;
  __shared__ unsigned tmem_base_sh;
  __shared__ volatile int abort_sh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = P.stages;
  const unsigned rank = PAIR ? cluster_rank() : 0u;
  const bool leader = rank == 0;
  const int g_id = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
  const int g_count = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full_bar[s], 1);
      // a stage is released by every issuing thread: the owner of its chunk commits, the other arrives
      mbar_init(&empty_bar[s], PAIR ? 1 : P.issuers);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], PAIR ? 16 : 8);  // the epilogue warps of both CTAs
    }
    mbar_init(&done_bar, P.issuers);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    if constexpr (PAIR) {
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_sh)),
                   "r"(2 * YBLK));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    } else {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_sh)),
                   "r"(2 * YBLK));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
  }
  tc_fence_before();
  __syncthreads();
  if constexpr (PAIR) cluster_sync_all();
  tc_fence_after();
  const unsigned tmem = tmem_base_sh;
  auto give_up = [&]() {
    atomicExch(P.status + 1, 1);
    abort_sh = 1;
    if constexpr (PAIR)
      asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(mapa_shared(su32((const void *)&abort_sh), rank ^ 1u)),
                   "r"(1)
                   : "memory");
  };
  const int a_bytes = TILE_X * TILE_Y * TILE_Z * KCHUNK * 2;  // 8 KB
  const int vrows = PAIR ? YBLK / 2 : YBLK;                   // V rows of a block in this CTA
  const int b_bytes = vrows * KCHUNK * 2;                     // 8 or 16 KB
  const int segc = P.segc;
  const int nseg = (P.NK + segc - 1) / segc;                  // segments per item
  const int nitems = P.item0[P.l0] + P.nitems[P.l0] - P.item0[P.l1];
  auto tz_units = [&](int l) { return PAIR ? (P.HZ[l] / TILE_Z + 1) / 2 : P.HZ[l] / TILE_Z; };
  // item -> level, rhs, parity, tile, block; items of a tile are consecutive (blocks innermost) so that the
  // CTAs working at the same time share the tile's multipoles and the V blocks through L2
  struct YItem {
    int level, rhs, par, bx, by, bz, nb, blk;  // blk: the 128-row block of a compacted level, else -1
    int g;                                     // the item's index over all levels
  };
  auto decode = [&](int it) {
    YItem y;
    int g = it + P.item0[P.l1];
    int l = P.l1;
    while (l > P.l0 && g >= P.item0[l] + P.nitems[l]) --l;
    int r = g - P.item0[l];
    y.level = l;
    y.g = g;
    y.nb = r % P.nblk;
    r /= P.nblk;
    y.blk = -1;
    if ((P.compact_levels >> l) & 1u) {
      int p = 0;
      while (p < 7 && r >= P.cblk0[l][p + 1]) ++p;
      y.blk = r;
      y.par = p;
      y.rhs = 0;
      y.bx = y.by = y.bz = 0;
      return y;
    }
    const int TX = P.HX[l] / TILE_X, TY = P.HY[l] / TILE_Y, TZu = tz_units(l);
    y.bx = r % TX;
    r /= TX;
    y.by = r % TY;
    r /= TY;
    y.bz = (r % TZu) * (PAIR ? 2 : 1) + (int)rank;  // this CTA's tile
    r /= TZu;
    y.par = r & 7;
    y.rhs = r >> 3;
    return y;
  };
  // whether the item's tile (a pair: either tile) holds a cell; all roles skip the others alike
  auto occupied = [&](const YItem &y) -> bool {
    if (y.blk >= 0) return true;  // a block of a compacted level holds at least one cell
    const int l = y.level, TX = P.HX[l] / TILE_X, TY = P.HY[l] / TILE_Y, TZ = P.HZ[l] / TILE_Z;
    const int bz0 = PAIR ? y.bz - (int)rank : y.bz;
    if ((P.full_levels >> l) & 1u) {
      // a full level: a tile holds cells when it overlaps the parity grid [0, 2^(l-1))^3 (no memory read)
      const int sh = 1 << (l - 1);
      return y.bx * TILE_X < sh && y.by * TILE_Y < sh && (bz0 * TILE_Z < sh || (PAIR && (bz0 + 1) * TILE_Z < sh));
    }
    auto tile = [&](int bz) {
      const long long id = P.tile0[l] + (((long long)y.par * TZ + bz) * TY + y.by) * TX + y.bx;
      return (P.busy[6 * id + 5] >> 31) & 1u;
    };
    bool o = bz0 < TZ && tile(bz0);
    if (PAIR && bz0 + 1 < TZ) o = o || tile(bz0 + 1);
    return o;
  };

  if (warp < 4) {
  give_registers<true>();  // the epilogue holds 128 running sums per thread
  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      unsigned phase = 0;
      unsigned loaded = 0, lpar = 0;  // stages that received a load, and the phase parity of the last one
      const unsigned full0 = PAIR ? mapa_shared(su32(&full_bar[0]), 0u) : su32(&full_bar[0]);
      for (int it = g_id; it < nitems && !abort_sh; it += g_count) {
        const YItem y = decode(it);
        if (!occupied(y)) continue;
        const int vrow = (P.ybase[y.par] + y.nb * (YBLK / 16)) * 16 + (int)rank * vrows;
        for (int kc = 0; kc < P.NK; ++kc) {
          if (!mbar_wait(&empty_bar[stage], phase ^ 1)) {
            give_up();
            break;
          }
          unsigned char *sbuf = smem + (size_t)stage * P.stage_bytes;
          if (leader) mbar_expect_tx(&full_bar[stage], (PAIR ? 2 : 1) * (2 * a_bytes + 2 * b_bytes));
          const int c4 = y.rhs * 8 + y.par;
          if constexpr (PAIR) {
            const unsigned fb = full0 + 8u * (unsigned)stage;
            tma_load_5d_pair(sbuf, &P.mapA_hi[y.level], fb, kc * KCHUNK, y.bx * TILE_X, y.by * TILE_Y, y.bz * TILE_Z,
                             c4);
            tma_load_5d_pair(sbuf + a_bytes, &P.mapA_lo[y.level], fb, kc * KCHUNK, y.bx * TILE_X, y.by * TILE_Y,
                             y.bz * TILE_Z, c4);
            tma_load_2d_pair(sbuf + 2 * a_bytes, &P.mapV_hi, fb, kc * KCHUNK, vrow);
            tma_load_2d_pair(sbuf + 2 * a_bytes + b_bytes, &P.mapV_lo, fb, kc * KCHUNK, vrow);
          } else if (y.blk >= 0) {
            tma_load_2d(sbuf, &P.mapC_hi[y.level], &full_bar[stage], kc * KCHUNK, y.blk * 128);
            tma_load_2d(sbuf + a_bytes, &P.mapC_lo[y.level], &full_bar[stage], kc * KCHUNK, y.blk * 128);
            tma_load_2d(sbuf + 2 * a_bytes, &P.mapV_hi, &full_bar[stage], kc * KCHUNK, vrow);
            tma_load_2d(sbuf + 2 * a_bytes + b_bytes, &P.mapV_lo, &full_bar[stage], kc * KCHUNK, vrow);
          } else {
            tma_load_5d(sbuf, &P.mapA_hi[y.level], &full_bar[stage], kc * KCHUNK, y.bx * TILE_X, y.by * TILE_Y,
                        y.bz * TILE_Z, c4);
            tma_load_5d(sbuf + a_bytes, &P.mapA_lo[y.level], &full_bar[stage], kc * KCHUNK, y.bx * TILE_X,
                        y.by * TILE_Y, y.bz * TILE_Z, c4);
            tma_load_2d(sbuf + 2 * a_bytes, &P.mapV_hi, &full_bar[stage], kc * KCHUNK, vrow);
            tma_load_2d(sbuf + 2 * a_bytes + b_bytes, &P.mapV_lo, &full_bar[stage], kc * KCHUNK, vrow);
          }
          loaded |= 1u << stage;
          lpar = (lpar & ~(1u << stage)) | (phase << stage);
          if (++stage == S) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
      // as in the second product: no bulk copy may be landing when the CTA exits
      if (leader)
        for (int st = 0; st < S; ++st)
          if ((loaded >> st) & 1u) mbar_wait(&full_bar[st], (lpar >> st) & 1u);
    }
  } else if (warp == 1 || (warp == 2 && P.issuers == 2)) {
    // MMA issue: one thread for both accumulators, or one per accumulator (warp 1: segments into accumulator
    // 0, warp 2: into accumulator 1), so that one thread's waits and bookkeeping leave the other's MMAs queued
    if (lane == 0 && leader) {
      const unsigned mine = P.issuers == 2 ? (unsigned)(warp - 1) : 2u;
      const unsigned idesc = (1u << 4) | ((unsigned)(YBLK >> 3) << 17) | ((unsigned)((PAIR ? 256 : 128) >> 4) << 24);
      auto mma = [&](unsigned d, unsigned long long da, unsigned long long db, unsigned acc) {
        if constexpr (PAIR)
          mma_f16_pair(d, da, db, idesc, acc);
        else
          mma_f16(d, da, db, idesc, acc);
      };
      auto commit = [&](unsigned long long *bar) {
        if constexpr (PAIR)
          mma_commit_pair_both(bar);
        else
          mma_commit(bar);
      };
      const unsigned long long dA_hi = sdesc(smem), dA_lo = dA_hi + (unsigned)(a_bytes >> 4);
      const unsigned long long dB_hi = dA_hi + (unsigned)((2 * a_bytes) >> 4), dB_lo = dB_hi + (unsigned)(b_bytes >> 4);
      const unsigned stage_step = (unsigned)P.stage_bytes >> 4;
      int stage = 0;
      unsigned phase = 0, empty_par = 3u;
      // The tensor pipe keeps only a few MMAs queued, so every cycle this thread spends between MMA groups
      // (barrier tests, bookkeeping) idles it: the loop keeps per-chunk work to the two waits and counters.
      for (int it = g_id; it < nitems; it += g_count) {
        if (abort_sh) break;
        if (!occupied(decode(it))) continue;
        unsigned b = 0;  // accumulator of the current segment
        int sc = 0;      // chunks issued into it
        bool failed = false;
        for (int kc = 0; kc < P.NK; ++kc) {
          const bool own = mine == 2u || b == mine;
          if (own && sc == 0) {
            if (!mbar_wait(&acc_empty[b], (empty_par >> b) & 1u)) {
              failed = true;
              break;
            }
            empty_par ^= 1u << b;
            tc_fence_after();
          }
          // Every issuing thread waits for every stage, its own chunks or not, and a stage is refilled only
          // after both threads have passed it: a thread that skipped the other's chunks could otherwise wait
          // on a stage's full barrier two phases ahead, where the parity test passes before the data is in.
          if (!mbar_wait(&full_bar[stage], phase)) {
            failed = true;
            break;
          }
          if (own) {
            const unsigned so = (unsigned)stage * stage_step;
            const unsigned d = tmem + b * (unsigned)YBLK;
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              const unsigned k2 = 2u * ks;
              mma(d, dA_hi + so + k2, dB_lo + so + k2, (sc == 0 && ks == 0) ? 0u : 1u);
              mma(d, dA_lo + so + k2, dB_hi + so + k2, 1u);
              mma(d, dA_hi + so + k2, dB_hi + so + k2, 1u);
            }
            commit(&empty_bar[stage]);
          } else {
            mbar_arrive(&empty_bar[stage]);  // this thread's share of the stage's release
          }
          if (++stage == S) {
            stage = 0;
            phase ^= 1;
          }
          if (++sc == segc || kc == P.NK - 1) {
            if (own) commit(&acc_full[b]);
            sc = 0;
            b ^= 1u;
          }
        }
        if (failed) {
          give_up();
          break;
        }
      }
      if constexpr (PAIR)
        mma_commit_pair_local(&done_bar);
      else
        mma_commit(&done_bar);
      if (!mbar_wait(&done_bar, 0)) give_up();
    }
  }
  } else {
    take_registers<true>();
    const int q = warp & 3;
    const int ch = (warp - 4) >> 2;  // which 128 of the 256 columns
    const int row = q * 32 + lane;   // source cell within the tile
    const unsigned tlane = tmem + ((unsigned)(q * 32) << 16) + (unsigned)(ch * 128);
    const unsigned empty0 = PAIR ? mapa_shared(su32(&acc_empty[0]), 0u) : 0u;
    unsigned full_par = 0;
    float acc[128];
    for (int it = g_id; it < nitems && !abort_sh; it += g_count) {
      const YItem y = decode(it);
      // one flag per (item, CTA of the pair, epilogue warp): whether this warp's rows of the item hold values
      // (tile-mode levels only; the item's index in the tile-mode numbering)
      unsigned char *dirty =
          P.ydirty + ((2 * (size_t)(P.dirty0[y.level] + y.g - P.item0[y.level]) + rank) * 8 + (warp - 4));
      if (!occupied(y)) {
        // an empty tile: its rows of Y must read as zero; clear them if an earlier tree left values there
        const bool was = *dirty != 0;
        __syncwarp();
        if (was) {
          const int l = y.level;
          const int hx = y.bx * TILE_X + (row & 7), hy = y.by * TILE_Y + ((row >> 3) & 3),
                    hz = y.bz * TILE_Z + (row >> 5);
          const int nch = P.ybase[y.par + 1] - P.ybase[y.par];
          if (y.bz < P.HZ[l] / TILE_Z)
            for (int k = 0; k < 8; ++k) {
              const int chunk = y.nb * (YBLK / 16) + ch * 8 + k;
              if (chunk >= nch) break;
              const long long yi = (long long)y.rhs * P.ycht + P.ybase[y.par] + chunk;
              const long long off = (((yi * P.HZ[l] + hz) * P.HY[l] + hy) * P.HX[l] + hx) * 16;
              uint4 *dh = (uint4 *)(P.Yhi[l] + off), *dl = (uint4 *)(P.Ylo[l] + off);
              dh[0] = dh[1] = dl[0] = dl[1] = make_uint4(0u, 0u, 0u, 0u);
            }
          __syncwarp();
          if (lane == 0) *dirty = 0;
        }
        continue;
      }
#pragma unroll
      for (int i = 0; i < 128; ++i) acc[i] = 0.f;
      for (int sg = 0; sg < nseg; ++sg) {
        const int b = sg & 1;
        if (!mbar_wait_warp(&acc_full[b], (full_par >> b) & 1u)) {
          give_up();
          break;
        }
        full_par ^= 1u << b;
        tc_fence_after();
        drain_cols<128, 4>(tlane + (unsigned)(b * YBLK), acc);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          if constexpr (PAIR)
            mbar_arrive_cluster(empty0 + 8u * (unsigned)b);
          else
            mbar_arrive(&acc_empty[b]);
        }
      }
      if (abort_sh) break;
      // write the 8 chunks of 16 ranks this thread holds, as FP16 hi and lo
      const int l = y.level;
      long long plane = (long long)P.HZ[l] * P.HY[l] * P.HX[l];
      long long pos = 0;  // the row's cell in the parity grid: (hz * HY + hy) * HX + hx
      bool real = true;   // false for a padding row of a compacted parity's last block (lanes stay together)
      if (y.blk >= 0) {
        const int code = P.crow[l][y.blk * 128 + row];
        real = code >= 0;
        if (P.ypr[l] > 0) {
          // stored by compacted row: rows of this parity from its first block on
          plane = P.ypr[l];
          pos = (long long)(y.blk - P.cblk0[l][y.par]) * 128 + row;
        } else {
          pos = real ? (code & 0x0FFFFFFF) : 0;
        }
      } else {
        if (y.bz >= P.HZ[l] / TILE_Z) continue;  // the missing second tile of a pair at the z edge
        const int hx = y.bx * TILE_X + (row & 7), hy = y.by * TILE_Y + ((row >> 3) & 3), hz = y.bz * TILE_Z + (row >> 5);
        pos = ((long long)hz * P.HY[l] + hy) * P.HX[l] + hx;
      }
      const int nch = P.ybase[y.par + 1] - P.ybase[y.par];  // chunks of this parity
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int chunk = y.nb * (YBLK / 16) + ch * 8 + k;
        if (chunk >= nch) break;
        const long long yi = (long long)y.rhs * P.ycht + P.ybase[y.par] + chunk;
        const long long off = (yi * plane + pos) * 16;
        unsigned hv[8], lv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          // two values per packed conversion: hi = fp16(v), lo = fp16(v - hi)
          const float2 v = make_float2(acc[k * 16 + 2 * i] * P.yscale, acc[k * 16 + 2 * i + 1] * P.yscale);
          const __half2 h = __float22half2_rn(v);
          const float2 hf = __half22float2(h);
          const __half2 l = __float22half2_rn(make_float2(v.x - hf.x, v.y - hf.y));
          hv[i] = *reinterpret_cast<const unsigned *>(&h);
          lv[i] = *reinterpret_cast<const unsigned *>(&l);
        }
        if (real) {
          uint4 *dh = (uint4 *)(P.Yhi[l] + off), *dl = (uint4 *)(P.Ylo[l] + off);
          dh[0] = make_uint4(hv[0], hv[1], hv[2], hv[3]);
          dh[1] = make_uint4(hv[4], hv[5], hv[6], hv[7]);
          dl[0] = make_uint4(lv[0], lv[1], lv[2], lv[3]);
          dl[1] = make_uint4(lv[4], lv[5], lv[6], lv[7]);
        }
      }
      if (y.blk < 0 && lane == 0) *dirty = 1;
    }
  }
  tc_fence_before();
  __syncthreads();
  if constexpr (PAIR) cluster_sync_all();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    if constexpr (PAIR)
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * YBLK));
    else
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * YBLK));
  }
}

// ---- conversion kernels -----------------------------------------------------------------------------

// Occupied cells of every level's parity grids, then their summed-area tables, for all levels in one launch
// each.  The cell marks are stored one cell up/right so that three prefix passes give the exclusive table
// that box_count reads.
struct LevelCells {
  const long long *keys[kMaxHeight];
  long long start[kMaxHeight + 1];  // concatenated numbering of the cells of levels 2..LL
  long long lines[3][kMaxHeight + 1];  // the same for the lines of each prefix pass
  int l0, l1;
};

__device__ __forceinline__ int level_of(const long long *start, int l0, int l1, long long g) {
  int l = l0;
  while (l < l1 && g >= start[l + 1]) ++l;
  return l;
}

__global__ void occ_mark_kernel(const __grid_constant__ TcParams P, const __grid_constant__ LevelCells C) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= C.start[C.l1 + 1]) return;
  const int l = level_of(C.start, C.l0, C.l1, g);
  const TcLevel &L = P.lv[l];
  int ix, iy, iz;
  morton_decode3(C.keys[l][g - C.start[l]], ix, iy, iz);
  const int c = ((ix & 1) << 2) | ((iy & 1) << 1) | (iz & 1);
  const size_t SX = L.HX + 1, SY = L.HY + 1, SZ = L.HZ + 1;
  int *sat = const_cast<int *>(L.sat);
  sat[(((size_t)c * SZ + (iz >> 1) + 1) * SY + (iy >> 1) + 1) * SX + (ix >> 1) + 1] = 1;
}

__global__ void sat_pass_kernel(const __grid_constant__ TcParams P, const __grid_constant__ LevelCells C, int axis) {
  const long long *ls = C.lines[axis];
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= ls[C.l1 + 1]) return;
  const int l = level_of(ls, C.l0, C.l1, g);
  const long long t = g - ls[l];
  const TcLevel &L = P.lv[l];
  const long long SX = L.HX + 1, SY = L.HY + 1, SZ = L.HZ + 1;
  long long base, stride, len;
  if (axis == 0) {
    base = t * SX;
    stride = 1;
    len = SX;
  } else if (axis == 1) {
    base = (t / SX) * SY * SX + t % SX;
    stride = SX;
    len = SY;
  } else {
    base = (t / (SY * SX)) * SZ * SY * SX + t % (SY * SX);
    stride = SY * SX;
    len = SZ;
  }
  int *sat = const_cast<int *>(L.sat);
  int acc = 0;
  for (long long k = 0; k < len; ++k) {
    acc += sat[base + k * stride];
    sat[base + k * stride] = acc;
  }
}

// Whether a box of a parity grid holds a cell when its level is full (every cell of the level exists):
// the parity grids then hold exactly the positions [0, side / 2) on each axis.
__device__ __forceinline__ bool box_nonempty_full(const TcLevel &L, int x0, int y0, int z0, int nx, int ny, int nz) {
  const int h = L.side >> 1;
  return x0 < h && x0 + nx > 0 && y0 < h && y0 + ny > 0 && z0 < h && z0 + nz > 0;
}

// busy masks of every level: one thread per (tile, transfer vector); tiles are numbered across levels.  Bit l
// of full_levels marks a full level, whose boxes are tested by their bounds instead of the summed-area
// tables (which are then not built when every level is full).
__global__ void busy_mask_kernel(const __grid_constant__ TcParams P, int l0, int l1, long long ntiles,
                                 unsigned full_levels, unsigned *__restrict__ busy) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= ntiles * 189) return;
  const long long tg = g / 189;
  const int e = (int)(g % 189);
  int level = l0;
  while (level < l1 && tg >= P.lv[level + 1].tile0) ++level;
  const TcLevel &L = P.lv[level];
  const long long tl = tg - L.tile0;
  const int TX = L.HX / TILE_X, TY = L.HY / TILE_Y, TZ = L.HZ / TILE_Z;
  TcItem w;
  w.level = (short)level;
  w.blk = -1;
  w.bx = (short)(tl % TX);
  w.by = (short)((tl / TX) % TY);
  w.bz = (short)((tl / ((long long)TX * TY)) % TZ);
  w.parity = (short)(tl / ((long long)TX * TY * TZ));
  unsigned *m = busy + 6 * tg;
  const SrcBox b = src_box(P, w, w.bz, e);
  const bool full = (full_levels >> level) & 1u;
  const bool src = full ? box_nonempty_full(L, b.ox, b.oy, b.oz, TILE_X, TILE_Y, TILE_Z)
                        : box_count(L, b.sp, b.ox, b.oy, b.oz, TILE_X, TILE_Y, TILE_Z) > 0;
  if (src) atomicOr(m + (e >> 5), 1u << (e & 31));
  if (e == 0) {
    const int x0 = w.bx * TILE_X, y0 = w.by * TILE_Y, z0 = w.bz * TILE_Z;
    const bool tgt = full ? box_nonempty_full(L, x0, y0, z0, TILE_X, TILE_Y, TILE_Z)
                          : box_count(L, w.parity, x0, y0, z0, TILE_X, TILE_Y, TILE_Z) > 0;
    if (tgt) atomicOr(m + 5, 1u << 31);
  }
}

// Work of every unit of levels [P.l0, P.l1]: the number of transfer vectors with an occupied source box when
// the unit's target tile (either tile of a pair) is occupied, else 0.  Written to prefix[u], which the scan
// below turns into exclusive prefix sums.
// Whether a unit holds a target cell of the shard (cells [a, b) of its level in Morton order).
__device__ bool unit_in_shard(const TcParams &P, const TcItem &w) {
  const long long a = P.shard[2 + 2 * w.level], b = P.shard[3 + 2 * w.level];
  if (a >= b) return false;
  const TcLevel &L = P.lv[w.level];
  const int tiles = P.pair ? 2 : 1;
  for (int t = 0; t < tiles; ++t) {
    if (w.blk >= 0) {
      for (int r = 0; r < 128; ++r) {
        const int cell = L.ccell[(long long)(w.blk + t) * 128 + r];
        if (cell >= a && cell < b) return true;
      }
      continue;
    }
    const int bz = w.bz + t;
    if (bz >= L.HZ / TILE_Z) continue;
    const int c = w.parity;
    for (int r = 0; r < 128; ++r) {
      const int hx = w.bx * TILE_X + (r & 7), hy = w.by * TILE_Y + ((r >> 3) & 3), hz = bz * TILE_Z + (r >> 5);
      const int gx = 2 * hx + ((c >> 2) & 1), gy = 2 * hy + ((c >> 1) & 1), gz = 2 * hz + (c & 1);
      if (gx >= L.side || gy >= L.side || gz >= L.side) continue;
      const int cell = L.grid[((long long)gz * L.side + gy) * L.side + gx];
      if (cell >= a && cell < b) return true;
    }
  }
  return false;
}

__global__ void unit_work_kernel(const __grid_constant__ TcParams P, int nunits, int *__restrict__ prefix) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nunits) return;
  const TcItem w = decode_unit(P, u);
  const BusyMask b = P.pair ? busy_mask_pair(P, w) : busy_mask(P, w);
  int n = 0;
  if (b.tile() && (!P.shard || unit_in_shard(P, w))) {
#pragma unroll
    for (int k = 0; k < 5; ++k) n += __popc(b.w[k]);
    n += __popc(b.w[5] & ((1u << (189 - 160)) - 1u));
  }
  prefix[u] = n;
}

// In-place exclusive prefix sums of prefix[0, n) with the total in prefix[n] (one block of 1024 threads).
__global__ void __launch_bounds__(1024) unit_scan_kernel(int n, int *__restrict__ prefix) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const int chunk = (n + 1023) / 1024;
  const int a = min(n, t * chunk), b = min(n, a + chunk);
  int sum = 0;
  for (int i = a; i < b; ++i) sum += prefix[i];
  part[t] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - sum;  // exclusive start of this thread's chunk
  for (int i = a; i < b; ++i) {
    const int v = prefix[i];
    prefix[i] = run;
    run += v;
  }
  if (t == 1023) prefix[n] = part[1023];
}

// The multipoles of levels [l0, l1], for the three packing launches of one M2L pass.
struct PackLevels {
  int l0, l1;
  const double *M[kMaxHeight];
  long long nval[kMaxHeight];           // multipole values of the level (cells * R * p^3)
  long long pos0[kMaxHeight + 1];       // first grid position of each level (rhs, parity, z, y, x)
  int HX[kMaxHeight], HY[kMaxHeight], HZ[kMaxHeight], side[kMaxHeight];
  const int *grid[kMaxHeight];          // dense cell grid of the level: cell index or -1
  __half *hi[kMaxHeight], *lo[kMaxHeight];
  double scale_l[kMaxHeight];           // 2 / cell width
};

// max |M| of every level (blockIdx.y = level - l0)
__global__ void absmax_levels_kernel(const __grid_constant__ PackLevels L, unsigned long long *__restrict__ amax) {
  const int l = L.l0 + blockIdx.y;
  const double *v = L.M[l];
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < L.nval[l]; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(v[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(amax + l, (unsigned long long)__double_as_longlong(m));
}

// every grid position of levels [l0, l1]: the scaled multipole of its cell, split into FP16 hi + lo, or
// zeros where there is no cell (and in the K padding), so that the buffers need no clearing
__global__ void pack_levels_kernel(const __grid_constant__ PackLevels L, int R, int nn, int KP,
                                   const double *__restrict__ scal) {
  const long long p = blockIdx.x + L.pos0[L.l0];
  int l = L.l0;
  while (l < L.l1 && p >= L.pos0[l + 1]) ++l;
  long long r = p - L.pos0[l];
  const long long base = r * KP;
  const int hx = (int)(r % L.HX[l]);
  r /= L.HX[l];
  const int hy = (int)(r % L.HY[l]);
  r /= L.HY[l];
  const int hz = (int)(r % L.HZ[l]);
  const int r8 = (int)(r / L.HZ[l]);
  const int par = r8 & 7, rhs = r8 >> 3;
  const int gx = 2 * hx + ((par >> 2) & 1), gy = 2 * hy + ((par >> 1) & 1), gz = 2 * hz + (par & 1);
  const int side = L.side[l];
  int cell = -1;
  if (gx < side && gy < side && gz < side) cell = L.grid[l][((long long)gz * side + gy) * side + gx];
  const double s = scal[2 * l];
  const double *m = cell >= 0 ? L.M[l] + ((long long)cell * R + rhs) * nn : nullptr;
  for (int n = threadIdx.x; n < KP; n += blockDim.x) {
    const double a = (m && n < nn) ? m[n] * s : 0.0;
    const __half h = __double2half(a);
    L.hi[l][base + n] = h;
    L.lo[l][base + n] = __double2half(a - (double)__half2float(h));
  }
}

// ---- compacted levels ------------------------------------------------------------------------------
// Cells of a sparse level grouped by parity into blocks of 128 rows, in Morton order inside each parity (so
// that a block's cells, and the sources of each transfer vector, lie close together, and the placement is the
// same on every run): per group of 1024 cells the count of each parity, then per parity the exclusive
// offsets of the groups and the total, then each cell's row.
__device__ __forceinline__ int key_parity(long long key, int &ix, int &iy, int &iz) {
  morton_decode3(key, ix, iy, iz);
  return ((ix & 1) << 2) | ((iy & 1) << 1) | (iz & 1);
}
__global__ void __launch_bounds__(1024) cgroup_count_kernel(const long long *__restrict__ keys, long long n,
                                                            int *__restrict__ gcnt) {
  __shared__ int cnt[8];
  if (threadIdx.x < 8) cnt[threadIdx.x] = 0;
  __syncthreads();
  const long long i = blockIdx.x * 1024LL + threadIdx.x;
  if (i < n) {
    int ix, iy, iz;
    atomicAdd(&cnt[key_parity(keys[i], ix, iy, iz)], 1);
  }
  __syncthreads();
  if (threadIdx.x < 8) gcnt[blockIdx.x * 8 + threadIdx.x] = cnt[threadIdx.x];
}
// one warp per parity: the group counts become exclusive offsets in place, the total goes to tot[p]
__global__ void __launch_bounds__(256) cgroup_scan_kernel(int ngroups, int *__restrict__ gcnt, int *__restrict__ tot) {
  const int p = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int run = 0;
  for (int g0 = 0; g0 < ngroups; g0 += 32) {
    const int g = g0 + lane;
    const int v = g < ngroups ? gcnt[g * 8 + p] : 0;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (g < ngroups) gcnt[g * 8 + p] = run + x - v;
    run += __shfl_sync(0xffffffffu, x, 31);
  }
  if (lane == 0) tot[p] = run;
}
struct CPlace {
  int blk0[9];  // first 128-row block of each parity (placement), or first Y chunk of each parity (cclear)
  int HX, HY;
};
// rowmap (optional): [parity][position] -> the cell's row counted from its parity's first block
__global__ void __launch_bounds__(1024) cgroup_place_kernel(const long long *__restrict__ keys, long long n,
                                                            const __grid_constant__ CPlace C,
                                                            const int *__restrict__ goff, int *__restrict__ crow,
                                                            int *__restrict__ ccell, int *__restrict__ rowmap,
                                                            long long plane) {
  __shared__ int wcnt[32][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long i = blockIdx.x * 1024LL + threadIdx.x;
  int ix = 0, iy = 0, iz = 0, par = -1;
  if (i < n) par = key_parity(keys[i], ix, iy, iz);
  const unsigned same = __match_any_sync(0xffffffffu, par);
  const int rk = __popc(same & ((1u << lane) - 1u));  // earlier lanes of this warp with the same parity
  (&wcnt[0][0])[threadIdx.x & 255] = 0;
  __syncthreads();
  if (par >= 0 && rk == 0) wcnt[warp][par] = __popc(same);
  __syncthreads();
  if (par < 0) return;
  int before = 0;
  for (int w = 0; w < warp; ++w) before += wcnt[w][par];
  const int prow = goff[blockIdx.x * 8 + par] + before + rk;
  const int row = C.blk0[par] * 128 + prow;
  const int pos = ((iz >> 1) * C.HY + (iy >> 1)) * C.HX + (ix >> 1);
  crow[row] = (par << 28) | pos;
  ccell[row] = (int)i;
  if (rowmap) rowmap[par * plane + pos] = prow;
}
// Busy masks of the compacted blocks of every compacted level (one CTA of 128 threads per block, blocks
// numbered across levels from b0): bit e set when the source of some row under transfer vector e is a cell,
// bit 31 of word 5 when the block holds a cell.
struct CBlocks {
  int l0, l1;
  int b0[kMaxHeight + 1];  // first block of each level; levels that are not compacted have none
};
__global__ void __launch_bounds__(128) cbusy_kernel(const __grid_constant__ TcParams P, const __grid_constant__ CBlocks B,
                                                    unsigned *__restrict__ cbusy) {
  __shared__ unsigned m[6];
  const int gb = blockIdx.x;
  int l = B.l0;
  while (l < B.l1 && gb >= B.b0[l + 1]) ++l;
  const TcLevel &L = P.lv[l];
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 6) m[threadIdx.x] = 0;
  __syncthreads();
  const int code = L.crow[(long long)(gb - B.b0[l]) * 128 + threadIdx.x];
  int gx = 0, gy = 0, gz = 0, par = 0;
  if (code >= 0) {
    par = code >> 28;
    const int pos = code & 0x0FFFFFFF;
    const int hx = pos % L.HX, hy = (pos / L.HX) % L.HY, hz = pos / (L.HX * L.HY);
    gx = 2 * hx + ((par >> 2) & 1);
    gy = 2 * hy + ((par >> 1) & 1);
    gz = 2 * hz + (par & 1);
  }
  const unsigned any = __ballot_sync(0xffffffffu, code >= 0);
  // every row of a block has the same parity; rows without a cell take the first valid row's
  par = __shfl_sync(0xffffffffu, par, any ? __ffs(any) - 1 : 0);
  for (int e = 0; e < 189; ++e) {
    bool occ = false;
    if (code >= 0) {
      const int sx = gx + P.off[par][e][0], sy = gy + P.off[par][e][1], sz = gz + P.off[par][e][2];
      occ = sx >= 0 && sx < L.side && sy >= 0 && sy < L.side && sz >= 0 && sz < L.side &&
            L.grid[((long long)sz * L.side + sy) * L.side + sx] >= 0;
    }
    const unsigned v = __ballot_sync(0xffffffffu, occ);
    if (lane == 0 && v) atomicOr(&m[e >> 5], 1u << (e & 31));
  }
  if (lane == 0 && any) atomicOr(&m[5], 1u << 31);
  __syncthreads();
  if (threadIdx.x < 6) cbusy[6LL * gb + threadIdx.x] = m[threadIdx.x];
}
// zero the Y rows (every chunk of the row's parity) of the cells a compacted level wrote for an earlier tree
__global__ void cclear_kernel(const int *__restrict__ crow, long long plane, const __grid_constant__ CPlace B,
                              __half *__restrict__ yhi, __half *__restrict__ ylo) {
  const int code = crow[blockIdx.x];
  if (code < 0) return;
  const int par = code >> 28;
  const long long pos = code & 0x0FFFFFFF;
  for (int ch = B.blk0[par] + (int)threadIdx.x; ch < B.blk0[par + 1]; ch += blockDim.x) {
    uint4 *dh = (uint4 *)(yhi + ((long long)ch * plane + pos) * 16), *dl = (uint4 *)(ylo + ((long long)ch * plane + pos) * 16);
    dh[0] = dh[1] = dl[0] = dl[1] = make_uint4(0u, 0u, 0u, 0u);
  }
}
// the compacted multipoles of one evaluation: row -> its cell's multipole scaled and split as pack_levels does
__global__ void pack_compact_kernel(const int *__restrict__ ccell, const double *__restrict__ M, int nn, int KP,
                                    const double *__restrict__ scal_l, __half *__restrict__ hi,
                                    __half *__restrict__ lo) {
  const long long row = blockIdx.x;
  const int cell = ccell[row];
  const double s = *scal_l;
  const double *m = cell >= 0 ? M + (long long)cell * nn : nullptr;
  for (int n = threadIdx.x; n < KP; n += blockDim.x) {
    const double a = (m && n < nn) ? m[n] * s : 0.0;
    const __half h = __double2half(a);
    hi[row * KP + n] = h;
    lo[row * KP + n] = __double2half(a - (double)__half2float(h));
  }
}

// 2^sA with sA chosen so that max|M| * 2^sA ~ 2^14, and the epilogue factor scale_l * 2^-(sA + shift)
// with shift the operators' own pre-scale exponent (SB for the dense K, sV + sU - sY for the low-rank
// factors).  One thread per level of [l0, l1]; max|M| of level l is the largest of amax[l * nslots + s].
__global__ void level_scale_kernel(const __grid_constant__ PackLevels L, const unsigned long long *__restrict__ amax,
                                   int nslots, int shift, double *__restrict__ scal) {
  const int l = L.l0 + (int)threadIdx.x;
  if (l > L.l1) return;
  unsigned long long bits = 0;
  for (int q = 0; q < nslots; ++q) bits = max(bits, amax[(size_t)l * nslots + q]);
  const double m = __longlong_as_double((long long)bits);
  int e = 0;
  if (m > 0) frexp(m, &e);  // m = f * 2^e, f in [0.5, 1)
  const int sA = 14 - e;
  scal[2 * l] = ldexp(1.0, sA);
  scal[2 * l + 1] = L.scale_l[l] * ldexp(1.0, -(sA + shift));
}

// operators: K[t][n][m] (FP64, source node n, target node m) -> B[t][m][n] split fp16, scaled by 2^SB
__global__ void pack_operators(int nn, int KP, int NP, const double *__restrict__ K, __half *__restrict__ hi,
                               __half *__restrict__ lo) {
  const int t = blockIdx.y;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)NP * KP) return;
  const int m = (int)(e / KP), n = (int)(e % KP);
  double v = 0.0;
  if (m < nn && n < nn) v = ldexp(K[((long long)t * nn + n) * nn + m], SB);
  const __half h = __double2half(v);
  hi[(long long)t * NP * KP + e] = h;
  lo[(long long)t * NP * KP + e] = __double2half(v - (double)__half2float(h));
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

}  // namespace

struct DenseTC {
  int KP = 0, NP = 0, NH = 0, NHALF = 0, NK = 0, stages = 0, ncols = 0, stage_bytes = 0, nbuf = 1;
  bool pair = false;  // CTA pairs with cta_group::2 MMAs (B200FMM_TC_PAIR=1 / 0 forces them on / off)
  __half *Bhi = nullptr, *Blo = nullptr;
  // per level
  __half *Ahi[kMaxHeight] = {}, *Alo[kMaxHeight] = {};
  size_t Abytes[kMaxHeight] = {};
  int HX[kMaxHeight] = {}, HY[kMaxHeight] = {}, HZ[kMaxHeight] = {};
  double *scal = nullptr;                 // [kMaxHeight][2]: pre, post
  unsigned long long *amax = nullptr;     // [kMaxHeight]
 int *prefix = nullptr;                  // work units of all levels: work, then exclusive prefix sums
  int nunits_all = 0;
  int *sat = nullptr;                     // occupancy summed-area tables of all levels
  size_t satn = 0, sat_off[kMaxHeight] = {};
  long long sat_serial = -1;              // tree the tables describe
  unsigned *busy = nullptr;               // busy masks of every tile of every level
  long long ntiles_all = 0;
  long long built_for_N = -1;             // tree the per-level buffers were sized for
  int splits = 0;                         // work ranges per CTA (pair): 0 = default (1), else fixed
  int splits_used = 0;
  int built_for_gen = -1;                 // tree generation the tensor maps / pointers belong to
  TcParams *params = nullptr;             // host copy
  int grid = 0;
  // low-rank form (symmetric Chebyshev operators): Bhi / Blo hold U in 16-wide K chunks
  bool lr = false;
  __half *Vhi = nullptr, *Vlo = nullptr;  // stacked V rows [16 * ycht][KP]
  __half *Yhi[kMaxHeight] = {}, *Ylo[kMaxHeight] = {};
  unsigned char *ydirty = nullptr;  // first product: per item, CTA of the pair and epilogue warp, rows hold values
  size_t ydirty_n = 0;
  size_t Ybytes[kMaxHeight] = {};
  int ycht = 0, nblk = 0, ystages = 0, ystage_bytes = 0;
  // low-rank layout (host side): 16-wide rank chunks of each slot, its first U chunk, the first Y chunk of
  // each source parity and of each slot among that parity's chunks
  unsigned char tnk[343] = {};
  short uchunk0[343] = {};
  int ybase[8] = {};
  short ychunk0[8][343] = {};
  TvRec *tv = nullptr;  // transfer-vector records on the device
  bool ypair = false;                     // first product on CTA pairs (B200FMM_TC_YPAIR=1) or single CTAs
  int lr_shift = 0;                       // sV + sU: the power-of-two pre-scales of V and U
  LrYParams *yparams = nullptr;           // host copy
  double lr_rank_fed[8] = {};             // first product: sum of the ranks of the slots each parity feeds
  int lr_rank[343] = {};                  // rank of each far slot
  // first product on compacted levels (sparse levels of a tree): per level
  int titem0[kMaxHeight] = {}, tnitems[kMaxHeight] = {};  // tile-mode item numbering (the ydirty flags)
  // what Y holds besides zeros: 0 nothing, 1 tile-mode rows, 2 compacted first product by grid position,
  // 3 by compacted row
  int ymode[kMaxHeight] = {};
  int *crow[kMaxHeight] = {};             // [rows]: (parity << 28) | position in the parity grid, or -1
  int *ccell[kMaxHeight] = {};            // [rows]: cell index, or -1
  __half *Chi[kMaxHeight] = {}, *Clo[kMaxHeight] = {};  // compacted multipoles [rows][KP]
  long long ccap[kMaxHeight] = {};        // rows allocated
  long long chcap[kMaxHeight] = {};       // rows allocated in Chi / Clo
  int crows[kMaxHeight] = {};             // rows of the current tree (128-row blocks of each parity)
  int *ccnt = nullptr;                    // [kMaxHeight][8]: cells of each parity
  int *cgrp = nullptr;                    // per level and group of 1024 cells: counts, then offsets, per parity
  long long cgrp_cap = 0;
  // second product on compacted levels: the tile-mode unit count of each level, the blocks' busy masks
  int tunits[kMaxHeight] = {};
  int *rowmap[kMaxHeight] = {};           // [8][plane] cell rows of levels whose Y is stored by compacted row
  unsigned *cbusy = nullptr;
  long long cbusy_cap = 0;
  int prefix_cap = 0;                     // entries allocated in prefix
};

static b200fmm_status encode(CUtensorMap *map, void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                             const cuuint32_t *box, CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_64B) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(B200FMM_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available");
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, (cuuint32_t)rank, base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(B200FMM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return B200FMM_OK;
}

// Low-rank operators: per far slot t, K chunks of 16 ranks; U chunks [uch][NP][16] (B of the second
// product) and, per source parity, the stacked V rows of the slots that the parity's cells feed (B of the
// first product), both pre-scaled by powers of two and split into FP16 hi + lo.
// Packing of the low-rank operators on the device, from the per-slot FP64 factors F (row-major p^3 x rank per
// slot, at the slot's offset): each value is scaled by 2^sc and split into FP16 hi = fp16(v), lo = fp16(v - hi).
//   U chunks [uch][NP][16]: chunk (foff, rank, kc), node n, lane i -> U[n][kc * 16 + i];
//   V rows [nrows][KP]: row (foff, rank, a), node n -> V[n][a].
// Entries past the node count or the rank are zero.
__global__ void pack_lr_u(long long nel, int NP, int nn, const int3 *__restrict__ chunks, const double *__restrict__ F,
                          int sc, __half *__restrict__ hi, __half *__restrict__ lo) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= nel) return;
  const int3 ch = chunks[g / ((long long)NP * 16)];
  const int rem = (int)(g % ((long long)NP * 16)), n = rem / 16, a = ch.z * 16 + rem % 16;
  const double v = (n < nn && a < ch.y) ? ldexp(F[ch.x + (long long)n * ch.y + a], sc) : 0.0;
  const __half h = __double2half(v);
  hi[g] = h;
  lo[g] = __double2half(v - (double)__half2float(h));
}
__global__ void pack_lr_v(long long nrows, int KP, int nn, const int3 *__restrict__ rows, const double *__restrict__ F,
                          int sc, __half *__restrict__ hi, __half *__restrict__ lo) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= nrows * KP) return;
  const int3 r = rows[g / KP];
  const int n = (int)(g % KP);
  const double v = (n < nn && r.z < r.y) ? ldexp(F[r.x + (long long)n * r.y + r.z], sc) : 0.0;
  const __half h = __double2half(v);
  hi[g] = h;
  lo[g] = __double2half(v - (double)__half2float(h));
}

static b200fmm_status tc_init_lowrank(Context &c, DenseTC &t, TcParams &P, bool &use) {
  std::vector<double> Ut, Vt;
  std::vector<long long> toff;
  std::vector<int> trank;
  B200_CHECK(sym_slot_factors(c, Ut, Vt, toff, trank));
  const int nn = c.nn;
  int uch = 0;
  for (int s = 0; s < 343; ++s) t.lr_rank[s] = toff[s] < 0 ? 0 : trank[s];
  for (int s = 0; s < 343; ++s) {
    t.tnk[s] = 0;
    t.uchunk0[s] = 0;
    if (toff[s] < 0) continue;
    t.tnk[s] = (unsigned char)((trank[s] + 15) / 16);
    t.uchunk0[s] = (short)uch;
    uch += t.tnk[s];
  }
  // the slots whose sources lie in each parity grid: target parity c + offset of its entry, per axis
  std::vector<std::array<bool, 343>> need(8);
  for (auto &row : need) row.fill(false);
  for (int ct = 0; ct < 8; ++ct)
    for (int e = 0; e < 189; ++e) {
      const int dx = c.itab.off[ct][e][0], dy = c.itab.off[ct][e][1], dz = c.itab.off[ct][e][2];
      const int sp = ((((ct >> 2) & 1) + dx) & 1) << 2 | ((((ct >> 1) & 1) + dy) & 1) << 1 | (((ct & 1) + dz) & 1);
      need[sp][c.itab.slot[ct][e]] = true;
    }
  int ych = 0, maxch = 0;
  for (int sp = 0; sp < 8; ++sp) {
    t.ybase[sp] = ych;
    int k = 0;
    double rsum = 0;
    for (int s = 0; s < 343; ++s) {
      t.ychunk0[sp][s] = 0;
      if (!need[sp][s]) continue;
      if (t.tnk[s] == 0) return fail(B200FMM_ERR_INVALID, "low-rank M2L: an interaction slot has no operator");
      t.ychunk0[sp][s] = (short)k;
      k += t.tnk[s];
      rsum += trank[s];
    }
    t.lr_rank_fed[sp] = rsum;
    ych += k;
    maxch = std::max(maxch, k);
  }
  t.ycht = ych;
  P.ycht = ych;
  t.nblk = (maxch + (YBLK / 16) - 1) / (YBLK / 16);
  // Y of all levels must fit comfortably: else the dense form is used
  double ybytes = 0;
  for (int l = 2; l <= c.H - 1; ++l) {
    const double h = (double)(1LL << (l - 1));
    ybytes += (double)c.R * ych * std::max(h, (double)TILE_X) * std::max(h, (double)TILE_Y) *
              std::max(h, (double)TILE_Z) * 16 * 2 * 2;
  }
  // the cap: 30 % of the device's memory (54 GB on a B200; 16 right-hand sides at height 6 take 14 GB), at
  // least 12 GB
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) total_b = 0;
  cudaGetLastError();
  if (ybytes > std::max(12e9, 0.3 * (double)total_b)) {
    use = false;
    return B200FMM_OK;
  }
  // pre-scales by powers of two.  The largest entries of A (level_scale_kernel), V and U lie in [2^13, 2^14),
  // so that the lo parts of the FP16 splits stay normal numbers (smaller scales put them among the FP16
  // subnormals and cost about 20x in accuracy); Y = V^T A, produced in FP32, is scaled by 2^-sY before its
  // own split so that |Y| < 2^15 (column sums of V times 2^14 bound it).
  double vmax = 0, colsum = 0, umax = 0;
  for (int s = 0; s < 343; ++s) {
    if (toff[s] < 0) continue;
    const int r = trank[s];
    for (int a = 0; a < r; ++a) {
      double cs = 0;
      for (int n = 0; n < nn; ++n) {
        const double v = std::fabs(Vt[toff[s] + (size_t)n * r + a]);
        cs += v;
        vmax = std::max(vmax, v);
      }
      colsum = std::max(colsum, cs);
    }
    for (long long i = 0; i < (long long)nn * r; ++i) umax = std::max(umax, std::fabs(Ut[toff[s] + i]));
  }
  int ev = 0, eu = 0, eb = 0;
  std::frexp(vmax, &ev);
  std::frexp(umax, &eu);
  const int sV = 14 - ev, sU = 14 - eu;
  std::frexp(std::ldexp(colsum, sV + 14), &eb);
  const int sY = eb - 15;
  t.lr_shift = sV + sU - sY;
  // the packed operators are written on the device from the per-slot factors: U chunks [uch][NP][16] and,
  // per source parity, the stacked V rows [ych * 16][KP], each value scaled and split into FP16 hi + lo
  std::vector<int3> uchunks((size_t)uch), vrows((size_t)ych * 16);
  for (int s = 0; s < 343; ++s) {
    if (toff[s] < 0) continue;
    for (int kc = 0; kc < t.tnk[s]; ++kc) uchunks[t.uchunk0[s] + kc] = make_int3((int)toff[s], trank[s], kc);
  }
  // V rows: row (ybase[sp] + ychunk0[sp][s] + kc) * 16 + i holds column kc * 16 + i of V_s along K
  for (int sp = 0; sp < 8; ++sp)
    for (int s = 0; s < 343; ++s) {
      if (!need[sp][s]) continue;
      for (int kc = 0; kc < t.tnk[s]; ++kc)
        for (int i = 0; i < 16; ++i)
          vrows[(size_t)(t.ybase[sp] + t.ychunk0[sp][s] + kc) * 16 + i] = make_int3((int)toff[s], trank[s], kc * 16 + i);
    }
  double *dU = nullptr, *dV = nullptr;
  int3 *dUc = nullptr, *dVr = nullptr;
  const size_t uel = (size_t)uch * t.NP * 16, vel = (size_t)ych * 16 * t.KP;
  B200_CUDA(cudaMalloc(&dU, sizeof(double) * Ut.size()));
  B200_CUDA(cudaMalloc(&dV, sizeof(double) * Vt.size()));
  B200_CUDA(cudaMalloc(&dUc, sizeof(int3) * std::max<size_t>(uchunks.size(), 1)));
  B200_CUDA(cudaMalloc(&dVr, sizeof(int3) * std::max<size_t>(vrows.size(), 1)));
  B200_CUDA(cudaMemcpy(dU, Ut.data(), sizeof(double) * Ut.size(), cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(dV, Vt.data(), sizeof(double) * Vt.size(), cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(dUc, uchunks.data(), sizeof(int3) * uchunks.size(), cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(dVr, vrows.data(), sizeof(int3) * vrows.size(), cudaMemcpyHostToDevice));
  B200_CUDA(cudaMalloc(&t.Bhi, uel * sizeof(__half)));
  B200_CUDA(cudaMalloc(&t.Blo, uel * sizeof(__half)));
  B200_CUDA(cudaMalloc(&t.Vhi, vel * sizeof(__half)));
  B200_CUDA(cudaMalloc(&t.Vlo, vel * sizeof(__half)));
  pack_lr_u<<<grid_for((long long)uel, 256), 256>>>((long long)uel, t.NP, nn, dUc, dU, sU, t.Bhi, t.Blo);
  pack_lr_v<<<grid_for((long long)vel, 256), 256>>>((long long)ych * 16, t.KP, nn, dVr, dV, sV, t.Vhi, t.Vlo);
  B200_CUDA(cudaGetLastError());
  B200_CUDA(cudaDeviceSynchronize());
  cudaFree(dU);
  cudaFree(dV);
  cudaFree(dUc);
  cudaFree(dVr);
  {
    cuuint64_t dims[3] = {16, (cuuint64_t)t.NP, (cuuint64_t)uch};
    cuuint64_t strides[2] = {32, (cuuint64_t)32 * t.NP};
    cuuint32_t box[3] = {16, (cuuint32_t)(t.pair ? t.NH / 2 : t.NH), 1};
    B200_CHECK(encode(&P.mapB_hi, t.Bhi, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_32B));
    B200_CHECK(encode(&P.mapB_lo, t.Blo, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_32B));
  }
  t.yparams = new LrYParams();
  std::memset(t.yparams, 0, sizeof(LrYParams));
  LrYParams &Y = *t.yparams;
  if (const char *e = getenv("B200FMM_TC_YPAIR")) t.ypair = atoi(e) != 0;
  {
    cuuint64_t dims[2] = {(cuuint64_t)t.KP, (cuuint64_t)ych * 16};
    cuuint64_t strides[1] = {(cuuint64_t)t.KP * 2};
    cuuint32_t box[2] = {KCHUNK, (cuuint32_t)(t.ypair ? YBLK / 2 : YBLK)};
    B200_CHECK(encode(&Y.mapV_hi, t.Vhi, 2, dims, strides, box));
    B200_CHECK(encode(&Y.mapV_lo, t.Vlo, 2, dims, strides, box));
  }
  for (int sp = 0; sp <= 8; ++sp) Y.ybase[sp] = sp < 8 ? t.ybase[sp] : ych;
  Y.ycht = ych;
  Y.nblk = t.nblk;
  Y.NK = t.NK;
  Y.R = c.R;
  Y.yscale = (float)std::ldexp(1.0, -sY);
  // first product: segments of 3 K chunks (18 MMAs); second product: segments of 12 chunks (36 MMAs).  At
  // order 7 this keeps the M2L within 5.5e-7 of FP64 (longer segments: 6-9e-7 for a few % less time)
  Y.segc = 3;
  if (const char *e = getenv("B200FMM_TC_LR_YSEG")) Y.segc = std::max(1, atoi(e));
  Y.issuers = 2;
  if (const char *e = getenv("B200FMM_TC_YISSUERS")) Y.issuers = atoi(e) == 1 ? 1 : 2;
  if (t.ypair) Y.issuers = 1;  // on CTA pairs the stage release is the leader's multicast commit alone
  t.ystage_bytes = 2 * (TILE_X * TILE_Y * TILE_Z * KCHUNK * 2) + 2 * (t.ypair ? YBLK / 2 : YBLK) * KCHUNK * 2;
  t.ystages = std::min(MAX_STAGES, (220 * 1024) / t.ystage_bytes);
  Y.stages = t.ystages;
  Y.stage_bytes = t.ystage_bytes;
  Y.status = c.d_status;
  // segments of the second product's chunk stream: as many 16-wide K steps as a dense segment has
  P.lr_seglen = 12;
  if (const char *e = getenv("B200FMM_TC_LR_SEGLEN")) P.lr_seglen = std::max(1, atoi(e));
  use = true;
  return B200FMM_OK;
}

b200fmm_status tc_init(Context &c) {
  DenseTC *t = new DenseTC();
  c.tc = t;
  const int nn = c.nn;
  t->KP = (nn + KCHUNK - 1) / KCHUNK * KCHUNK;
  t->NP = t->KP;
  t->NHALF = t->NP > 256 ? 2 : 1;
  t->NH = t->NP / t->NHALF;
  if (t->NH % 16 != 0 || t->NH > 256) return fail(B200FMM_ERR_UNSUPPORTED, "unsupported node count for the MMA tile");
  if (t->NP > 352) return fail(B200FMM_ERR_UNSUPPORTED, "the tensor-core M2L supports orders up to 7");
  t->NK = t->KP / KCHUNK;
  // CTA pairs halve each SM's operator traffic; they pay off at order 7 (two column halves, 38.9 KB instead
  // of 61.4 KB per stage), while single CTAs are a few percent faster at orders <= 6
  t->pair = t->NHALF == 2;
  if (const char *e = getenv("B200FMM_TC_PAIR")) t->pair = atoi(e) != 0;
  t->params = new TcParams();
  std::memset(t->params, 0, sizeof(TcParams));
  std::memcpy(t->params->off, c.itab.off, sizeof(t->params->off));
  std::memcpy(t->params->slot, c.itab.slot, sizeof(t->params->slot));
  // symmetric Chebyshev operators run in their compressed (low-rank) form; B200FMM_TC_LOWRANK=0 keeps the
  // dense operators
  bool lr = c.cfg.kernel == B200FMM_CHEB_SYM && !c.sym_ranks.empty();
  if (const char *e = getenv("B200FMM_TC_LOWRANK")) lr = lr && atoi(e) != 0;
  if (lr) B200_CHECK(tc_init_lowrank(c, *t, *t->params, lr));
  t->lr = lr;
  {
    // the transfer-vector records of both forms
    std::vector<TvRec> tv(8 * 189);
    for (int ct = 0; ct < 8; ++ct)
      for (int e = 0; e < 189; ++e) {
        const int cax[3] = {(ct >> 2) & 1, (ct >> 1) & 1, ct & 1};
        int sp = 0, o[3];
        for (int a = 0; a < 3; ++a) {
          const int v = cax[a] + c.itab.off[ct][e][a];  // source position in child cells
          o[a] = v >= 0 ? v / 2 : -((1 - v) / 2);       // floor(v / 2): the source tile's offset
          sp = (sp << 1) | (v & 1);
        }
        const int slot = c.itab.slot[ct][e];
        TvRec &r = tv[ct * 189 + e];
        r.ox = (signed char)o[0];
        r.oy = (signed char)o[1];
        r.oz = (signed char)o[2];
        r.ya = (short)(lr ? t->ybase[sp] + t->ychunk0[sp][slot] : sp);
        r.ub = (short)(lr ? t->uchunk0[slot] : slot);
        r.nk = lr ? t->tnk[slot] : 0;
      }
    B200_CUDA(cudaMalloc(&t->tv, tv.size() * sizeof(TvRec)));
    B200_CUDA(cudaMemcpy(t->tv, tv.data(), tv.size() * sizeof(TvRec), cudaMemcpyHostToDevice));
    t->params->tv = t->tv;
  }
  const int rowb = lr ? 32 : 64;  // bytes per operand row of a stage: 16 or 32 fp16 of K
  // a CTA of a pair holds NP / 2 rows of each operator chunk: NH / 2 rows of each column half
  const int b_rows = t->pair ? t->NP / 2 : t->NP;
  t->stage_bytes = 2 * (TILE_X * TILE_Y * TILE_Z * rowb) + 2 * b_rows * rowb;
  t->stages = std::min((t->pair || lr) ? MAX_STAGES : MAX_STAGES_SINGLE, (220 * 1024 - TV_BYTES) / t->stage_bytes);
  if (t->stages < 2) return fail(B200FMM_ERR_UNSUPPORTED, "stage buffers do not fit in shared memory");
  t->nbuf = 2 * t->NP <= 512 ? 2 : 1;
  t->ncols = 32;
  while (t->ncols < t->nbuf * t->NP) t->ncols *= 2;
  if (!lr) {
    B200_CHECK(build_dense_operators(c));  // FP64 K on the device
    const size_t bsz = (size_t)343 * t->NP * t->KP;
    B200_CUDA(cudaMalloc(&t->Bhi, bsz * sizeof(__half)));
    B200_CUDA(cudaMalloc(&t->Blo, bsz * sizeof(__half)));
    pack_operators<<<dim3(grid_for((long long)t->NP * t->KP, 256), 343), 256>>>(nn, t->KP, t->NP, c.d_dense, t->Bhi,
                                                                              t->Blo);
    B200_CUDA(cudaGetLastError());
    B200_CUDA(cudaDeviceSynchronize());
    // the FP64 dense operators are not needed by the mixed path after packing
    cudaFree(c.d_dense);
    c.d_dense = nullptr;
    cuuint64_t dims[3] = {(cuuint64_t)t->KP, (cuuint64_t)t->NP, 343};
    cuuint64_t strides[2] = {(cuuint64_t)t->KP * 2, (cuuint64_t)t->KP * 2 * t->NP};
    cuuint32_t box[3] = {KCHUNK, (cuuint32_t)(t->pair ? t->NH / 2 : t->NH), 1};
    B200_CHECK(encode(&t->params->mapB_hi, t->Bhi, 3, dims, strides, box));
    B200_CHECK(encode(&t->params->mapB_lo, t->Blo, 3, dims, strides, box));
  }
  B200_CUDA(cudaMalloc(&t->scal, sizeof(double) * kMaxHeight * 2));
  B200_CUDA(cudaMalloc(&t->amax, sizeof(unsigned long long) * kMaxHeight));
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c.device);
  t->grid = dev_sms;
  if (t->pair) {
    // persistent grid of CTA pairs: as many as can be resident at once
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    const size_t smem = (size_t)t->stages * t->stage_bytes + TV_BYTES + 1024;
    cfg.gridDim = dim3(dev_sms & ~1);
    cfg.blockDim = dim3(TC_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    cudaError_t err = cudaSuccess;
    auto occ = [&](auto kern) {
      err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (err == cudaSuccess) err = cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg);
    };
    switch (t->NP) {
#define B200_TC_OCC(NPV, CWV, NHV)                 \
  case NPV:                                        \
    if (lr)                                        \
      occ(m2l_tc_kernel<CWV, NHV, true, true, true>);  \
    else                                           \
      occ(m2l_tc_kernel<CWV, NHV, true, false, true>); \
    break;
      B200_TC_OCC(32, 16, 1)
      B200_TC_OCC(64, 32, 1)
      B200_TC_OCC(128, 64, 1)
      B200_TC_OCC(224, 112, 1)
      B200_TC_OCC(352, 176, 2)
#undef B200_TC_OCC
      default:
        break;
    }
    if (err != cudaSuccess || nclusters < 1) {
      cudaGetLastError();
      return fail(B200FMM_ERR_CUDA, "tensor-core M2L: no CTA pair can be resident (" +
                                        std::string(cudaGetErrorString(err)) + ")");
    }
    t->grid = 2 * std::min(nclusters, dev_sms / 2);
  }
  {
    // the kernels that move registers between warpgroups must run with exactly the registers the split
    // assumes, or their setmaxnreg.inc would wait for registers that were never allocated
    cudaFuncAttributes fa;
    bool regs_ok = true;
    auto check_regs = [&](auto kern) {
      if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess || fa.numRegs != TC_REGS) regs_ok = false;
    };
    check_regs(lr_y_kernel<true>);
    check_regs(lr_y_kernel<false>);
    check_regs(m2l_tc_kernel<176, 2, true, true, false>);
    check_regs(m2l_tc_kernel<176, 2, true, false, false>);
    check_regs(m2l_tc_kernel<176, 2, false, true, false>);
    check_regs(m2l_tc_kernel<176, 2, false, false, false>);
    check_regs(m2l_tc_kernel<112, 1, true, true, false>);
    check_regs(m2l_tc_kernel<112, 1, true, false, false>);
    check_regs(m2l_tc_kernel<112, 1, false, true, false>);
    check_regs(m2l_tc_kernel<112, 1, false, false, false>);
    check_regs(m2l_tc_kernel<176, 2, true, true, true>);
    check_regs(m2l_tc_kernel<176, 2, true, false, true>);
    check_regs(m2l_tc_kernel<176, 2, false, true, true>);
    check_regs(m2l_tc_kernel<176, 2, false, false, true>);
    check_regs(m2l_tc_kernel<112, 1, true, true, true>);
    check_regs(m2l_tc_kernel<112, 1, true, false, true>);
    check_regs(m2l_tc_kernel<112, 1, false, true, true>);
    check_regs(m2l_tc_kernel<112, 1, false, false, true>);
    if (!regs_ok) {
      cudaGetLastError();
      return fail(B200FMM_ERR_UNSUPPORTED, "tensor-core M2L: kernels not compiled to the register count their "
                                           "warpgroup register split needs");
    }
  }
  if (lr) {
    const int ysmem = t->ystages * t->ystage_bytes + 1024;
    if (t->ypair)
      B200_CUDA(cudaFuncSetAttribute(lr_y_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysmem));
    else
      B200_CUDA(cudaFuncSetAttribute(lr_y_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysmem));
  }
  return B200FMM_OK;
}

void tc_free(Context &c) {
  DenseTC *t = c.tc;
  if (!t) return;
  for (void *p : {(void *)t->Bhi, (void *)t->Blo, (void *)t->scal, (void *)t->amax, (void *)t->prefix, (void *)t->busy,
                  (void *)t->Vhi, (void *)t->Vlo, (void *)t->tv})
    if (p) cudaFree(p);
  for (int l = 0; l < kMaxHeight; ++l) {
    if (t->Ahi[l]) cudaFree(t->Ahi[l]);
    if (t->Alo[l]) cudaFree(t->Alo[l]);
    if (t->Yhi[l]) cudaFree(t->Yhi[l]);
    if (t->Ylo[l]) cudaFree(t->Ylo[l]);
    for (void *q : {(void *)t->crow[l], (void *)t->ccell[l], (void *)t->Chi[l], (void *)t->Clo[l], (void *)t->rowmap[l]})
      if (q) cudaFree(q);
  }
  for (void *q : {(void *)t->ccnt, (void *)t->cgrp, (void *)t->cbusy})
    if (q) cudaFree(q);
  if (t->sat) cudaFree(t->sat);
  if (t->ydirty) cudaFree(t->ydirty);
  delete t->params;
  delete t->yparams;
  delete t;
  c.tc = nullptr;
}

// (Re)build the per-level A buffers, tensor maps and the work-item list for the current tree.
static b200fmm_status tc_prepare(Context &c) {
  DenseTC *t = c.tc;
  TcParams &P = *t->params;
  const int LL = c.H - 1;
  t->ntiles_all = 0;
  size_t sat_total = 0;
  bool y_moved = false;  // a level's Y was (re)allocated: every Y row and dirty flag starts from zero
  for (int l = 2; l <= LL; ++l) {
    const int h = 1 << (l - 1);
    t->HX[l] = std::max(h, TILE_X);
    t->HY[l] = std::max(h, TILE_Y);
    t->HZ[l] = std::max(h, TILE_Z);
    const size_t elems = (size_t)c.R * 8 * t->HZ[l] * t->HY[l] * t->HX[l] * t->KP;
    if (t->Abytes[l] != elems * sizeof(__half)) {
      if (t->Ahi[l]) cudaFree(t->Ahi[l]);
      if (t->Alo[l]) cudaFree(t->Alo[l]);
      B200_CUDA(cudaMalloc(&t->Ahi[l], elems * sizeof(__half)));
      B200_CUDA(cudaMalloc(&t->Alo[l], elems * sizeof(__half)));
      t->Abytes[l] = elems * sizeof(__half);
    }
    cuuint64_t dims[5] = {(cuuint64_t)t->KP, (cuuint64_t)t->HX[l], (cuuint64_t)t->HY[l], (cuuint64_t)t->HZ[l],
                          (cuuint64_t)(8 * c.R)};
    cuuint64_t st[4] = {(cuuint64_t)t->KP * 2, (cuuint64_t)t->KP * 2 * t->HX[l],
                        (cuuint64_t)t->KP * 2 * t->HX[l] * t->HY[l],
                        (cuuint64_t)t->KP * 2 * t->HX[l] * t->HY[l] * t->HZ[l]};
    cuuint32_t box[5] = {KCHUNK, TILE_X, TILE_Y, TILE_Z, 1};
    if (t->lr) {
      // the multipoles feed the first product; the second product's A is Y
      LrYParams &Y = *t->yparams;
      B200_CHECK(encode(&Y.mapA_hi[l], t->Ahi[l], 5, dims, st, box));
      B200_CHECK(encode(&Y.mapA_lo[l], t->Alo[l], 5, dims, st, box));
      const size_t yel = (size_t)c.R * t->ycht * t->HZ[l] * t->HY[l] * t->HX[l] * 16;
      if (t->Ybytes[l] != yel * sizeof(__half)) {
        if (t->Yhi[l]) cudaFree(t->Yhi[l]);
        if (t->Ylo[l]) cudaFree(t->Ylo[l]);
        t->Yhi[l] = t->Ylo[l] = nullptr;
        B200_CUDA(cudaMalloc(&t->Yhi[l], yel * sizeof(__half)));
        B200_CUDA(cudaMalloc(&t->Ylo[l], yel * sizeof(__half)));
        t->Ybytes[l] = yel * sizeof(__half);
        y_moved = true;
      }
      Y.Yhi[l] = t->Yhi[l];
      Y.Ylo[l] = t->Ylo[l];
      Y.HX[l] = t->HX[l];
      Y.HY[l] = t->HY[l];
      Y.HZ[l] = t->HZ[l];
      cuuint64_t ydims[5] = {16, (cuuint64_t)t->HX[l], (cuuint64_t)t->HY[l], (cuuint64_t)t->HZ[l],
                             (cuuint64_t)c.R * t->ycht};
      cuuint64_t yst[4] = {32, (cuuint64_t)32 * t->HX[l], (cuuint64_t)32 * t->HX[l] * t->HY[l],
                           (cuuint64_t)32 * t->HX[l] * t->HY[l] * t->HZ[l]};
      cuuint32_t ybox[5] = {16, TILE_X, TILE_Y, TILE_Z, 1};
      B200_CHECK(encode(&P.mapA_hi[l], t->Yhi[l], 5, ydims, yst, ybox, CU_TENSOR_MAP_SWIZZLE_32B));
      B200_CHECK(encode(&P.mapA_lo[l], t->Ylo[l], 5, ydims, yst, ybox, CU_TENSOR_MAP_SWIZZLE_32B));
    } else {
      B200_CHECK(encode(&P.mapA_hi[l], t->Ahi[l], 5, dims, st, box));
      B200_CHECK(encode(&P.mapA_lo[l], t->Alo[l], 5, dims, st, box));
    }
    P.lv[l].HX = t->HX[l];
    P.lv[l].HY = t->HY[l];
    P.lv[l].HZ = t->HZ[l];
    P.lv[l].side = 1 << l;
    P.lv[l].grid = c.lv[l].grid;
    P.lv[l].L = c.lv[l].L;
    P.lv[l].scale_out = t->scal + 2 * l + 1;
    t->sat_off[l] = sat_total;
    sat_total += (size_t)8 * (t->HX[l] + 1) * (t->HY[l] + 1) * (t->HZ[l] + 1);
    P.lv[l].tile0 = (int)t->ntiles_all;
    t->ntiles_all += 8LL * (t->HX[l] / TILE_X) * (t->HY[l] / TILE_Y) * (t->HZ[l] / TILE_Z);
    t->sat_serial = -1;
  }
  // work units, finest level first: every tile (or pair of z-adjacent tiles) of every right-hand side
  int nunits = 0;
  for (int l = LL; l >= 2; --l) {
    const int TZ = t->HZ[l] / TILE_Z;
    P.lv[l].TZu = t->pair ? (TZ + 1) / 2 : TZ;
    P.lv[l].unit0 = nunits;
    P.lv[l].nunits = c.R * 8 * P.lv[l].TZu * (t->HY[l] / TILE_Y) * (t->HX[l] / TILE_X);
    t->tunits[l] = P.lv[l].nunits;
    P.lv[l].cmode = 0;
    P.lv[l].plane = (long long)t->HX[l] * t->HY[l] * t->HZ[l];
    P.lv[l].ghi = t->lr ? t->Yhi[l] : t->Ahi[l];
    P.lv[l].glo = t->lr ? t->Ylo[l] : t->Alo[l];
    nunits += P.lv[l].nunits;
  }
  t->nunits_all = nunits;
  if (t->lr) {
    // first-product items, finest level first: rhs, parity, tile, 256-row block
    LrYParams &Y = *t->yparams;
    int n = 0;
    for (int l = LL; l >= 2; --l) {
      Y.item0[l] = n;
      const int TZ = t->HZ[l] / TILE_Z;
      Y.nitems[l] = c.R * 8 * (t->ypair ? (TZ + 1) / 2 : TZ) * (t->HY[l] / TILE_Y) * (t->HX[l] / TILE_X) * t->nblk;
      t->titem0[l] = Y.dirty0[l] = Y.item0[l];
      t->tnitems[l] = Y.nitems[l];
      n += Y.nitems[l];
    }
    Y.compact_levels = 0;
    // the first product skips items of empty tiles; their Y rows must read as zero (dirty flags: 2 CTAs x 8
    // epilogue warps per item)
    const size_t nd = (size_t)16 * std::max(n, 1);
    if (t->ydirty_n != nd) {
      if (t->ydirty) cudaFree(t->ydirty);
      t->ydirty = nullptr;
      B200_CUDA(cudaMalloc(&t->ydirty, nd));
      t->ydirty_n = nd;
      y_moved = true;
    }
    if (y_moved) {
      for (int l = 0; l < kMaxHeight; ++l) t->ymode[l] = 0;
      B200_CUDA(cudaMemsetAsync(t->ydirty, 0, nd, c.stream));
      for (int l = 2; l <= LL; ++l) {
        B200_CUDA(cudaMemsetAsync(t->Yhi[l], 0, t->Ybytes[l], c.stream));
        B200_CUDA(cudaMemsetAsync(t->Ylo[l], 0, t->Ybytes[l], c.stream));
      }
    }
    Y.ydirty = t->ydirty;
    for (int l = 2; l <= LL; ++l) Y.tile0[l] = P.lv[l].tile0;
  }
  int ns = t->splits > 0 ? t->splits : 1;  // work ranges per CTA (pair), chosen by b200fmm_autotune
  if (const char *e = getenv("B200FMM_TC_SPLITS")) ns = std::max(1, std::min(64, atoi(e)));
  t->splits_used = ns;
  if (t->satn != sat_total) {
    if (t->sat) cudaFree(t->sat);
    B200_CUDA(cudaMalloc(&t->sat, std::max<size_t>(sat_total, 1) * sizeof(int)));
    t->satn = sat_total;
  }
  for (int l = 2; l <= LL; ++l) P.lv[l].sat = t->sat + t->sat_off[l];
  if (t->busy) cudaFree(t->busy);
  B200_CUDA(cudaMalloc(&t->busy, sizeof(unsigned) * 6 * std::max<long long>(t->ntiles_all, 1)));
  P.busy = t->busy;
  if (t->lr) t->yparams->busy = t->busy;
  if (t->prefix) cudaFree(t->prefix);
  B200_CUDA(cudaMalloc(&t->prefix, sizeof(int) * (nunits + 1)));
  t->prefix_cap = nunits + 1;
  P.prefix = t->prefix;
  P.growlen = t->lr ? 16 : t->KP;
  P.ranges_per_cta = ns;
  P.pair = t->pair ? 1 : 0;
  P.R = c.R;
  P.nn = c.nn;
  P.KP = t->KP;
  P.NP = t->NP;
  P.NH = t->NH;
  P.NHALF = t->NHALF;
  P.NK = t->NK;
  P.stages = t->stages;
  P.ncols = t->ncols;
  P.stage_bytes = t->stage_bytes;
  // accumulator resets per transfer vector: 2 for p >= 6 keeps the M2L within ~1e-6 of FP64
  P.nseg = std::min(t->NK, c.p >= 6 ? 2 : 1);
  P.nbuf = t->nbuf;
  // a group of two chunks holds two stages while the producer fills the next ones: only with 5 or more
  if (const char *e = getenv("B200FMM_TC_SEGMENTS")) P.nseg = std::max(1, std::min(t->NK, atoi(e)));
  std::memcpy(P.off, c.itab.off, sizeof(P.off));
  std::memcpy(P.slot, c.itab.slot, sizeof(P.slot));
  P.status = c.d_status;
  t->built_for_N = c.N;
  t->built_for_gen = c.tree_gen;
  return B200FMM_OK;
}

// Per tree: which sparse levels run compacted, and their cells grouped by parity into 128-row blocks.
//   * A level is sparse when fewer than three quarters of its cells exist; compaction needs one right-hand side.
//   * The second product (U Y, or K M in the dense form) runs a compacted level's units over blocks (pairs of
//     blocks of one parity on CTA pairs) instead of grid tiles: the unit numbering of every level is redone
//     here, and the blocks get their busy masks.  B200FMM_TC_TCOMPACT=0 keeps the tiles.
//   * Low-rank form, single CTAs: the first product (Y = V^T M) of a compacted level runs over the same blocks,
//     with the compacted multipoles' tensor maps and its item numbering (B200FMM_TC_YCOMPACT=0 keeps the
//     tiles).  Y must read as zero wherever no cell is: rows that an earlier tree's compacted first product
//     wrote are cleared here, and a level whose first product turns compacted after tile-mode runs has its Y
//     and tile flags cleared (tile mode keeps clearing its own rows through the flags).
// One host synchronisation (the per-parity counts) when some level is compacted.
static b200fmm_status compact_setup(Context &c, DenseTC &t) {
  TcParams &P = *t.params;
  const int LL = c.H - 1;
  const char *ye = getenv("B200FMM_TC_YCOMPACT"), *te = getenv("B200FMM_TC_TCOMPACT");
  const bool yallow = t.lr && !t.ypair && c.R == 1 && !(ye && atoi(ye) == 0);
  const bool tallow = c.R == 1 && !(te && atoi(te) == 0);
  // a level runs compacted below this share of occupied cells (B200FMM_TC_COMPACT_BELOW in (0, 1]); on the
  // Plummer problems of height 7, 0.75 was 2-10 % faster per evaluation than 0.5 and 0.25 clearly slower
  double below = 0.75;
  if (const char *e = getenv("B200FMM_TC_COMPACT_BELOW")) {
    const double v = atof(e);
    if (v > 0.0 && v <= 1.0) below = v;
  }
  unsigned ymask = 0, tmask = 0;
  for (int l = 2; l <= LL; ++l) {
    const long long plane = (long long)t.HX[l] * t.HY[l] * t.HZ[l];
    const bool sparse = c.lv[l].n > 0 && (double)c.lv[l].n < below * (double)(1LL << (3 * l)) && plane < (1LL << 28);
    // the gathers number the rows of a level's source grid in 32 bits
    const long long grid_rows = (long long)c.R * (t.lr ? t.ycht : 8) * plane;
    if (yallow && sparse) ymask |= 1u << l;
    if (tallow && sparse && grid_rows < (1LL << 31)) tmask |= 1u << l;
  }
  const unsigned mask = ymask | tmask;
  // per-parity counts of every placed level, in groups of 1024 cells
  int cnt[kMaxHeight][8] = {};
  long long g0[kMaxHeight + 1] = {};
  if (mask) {
    for (int l = 2; l <= LL; ++l) g0[l + 1] = g0[l] + (((mask >> l) & 1u) ? (c.lv[l].n + 1023) / 1024 : 0);
    const long long ng = g0[LL + 1];
    if (t.cgrp_cap < 8 * ng) {
      if (t.cgrp) cudaFree(t.cgrp);
      t.cgrp = nullptr;
      t.cgrp_cap = 0;
      B200_CUDA(cudaMalloc(&t.cgrp, sizeof(int) * 8 * ng));
      t.cgrp_cap = 8 * ng;
    }
    if (!t.ccnt) B200_CUDA(cudaMalloc(&t.ccnt, sizeof(int) * kMaxHeight * 8));
    B200_CUDA(cudaMemsetAsync(t.ccnt, 0, sizeof(int) * kMaxHeight * 8, c.stream));
    for (int l = 2; l <= LL; ++l)
      if ((mask >> l) & 1u) {
        const int ngl = (int)(g0[l + 1] - g0[l]);
        cgroup_count_kernel<<<ngl, 1024, 0, c.stream>>>(c.lv[l].keys, c.lv[l].n, t.cgrp + 8 * g0[l]);
        cgroup_scan_kernel<<<1, 256, 0, c.stream>>>(ngl, t.cgrp + 8 * g0[l], t.ccnt + 8 * l);
        c.launches += 2;
      }
    B200_CUDA(cudaMemcpyAsync(cnt, t.ccnt, sizeof(cnt), cudaMemcpyDeviceToHost, c.stream));
    B200_CUDA(cudaStreamSynchronize(c.stream));
  }
  // blocks of every placed level (an even count per parity for CTA pairs).  A level compacted in both products
  // (low rank) stores its Y by compacted row when the largest parity's rows fit the grid layout's rows.
  CPlace Cl[kMaxHeight] = {};
  int ypr[kMaxHeight] = {};
  for (int l = 2; l <= LL; ++l) {
    if (!((mask >> l) & 1u)) continue;
    CPlace &C = Cl[l];
    C.blk0[0] = 0;
    int most = 0;
    for (int p = 0; p < 8; ++p) {
      int nb = (cnt[l][p] + 127) / 128;
      if (t.pair && ((tmask >> l) & 1u)) nb += nb & 1;
      C.blk0[p + 1] = C.blk0[p] + nb;
      most = std::max(most, nb);
    }
    C.HX = t.HX[l];
    C.HY = t.HY[l];
    const long long plane = (long long)t.HX[l] * t.HY[l] * t.HZ[l];
    if (t.lr && ((ymask & tmask) >> l & 1u) && 128LL * most <= plane) ypr[l] = 128 * most;
  }
  // Low rank: Y must read as zero wherever the second product may read a row that holds no cell of this tree.
  // Modes of a level's Y: 1 tile-mode rows (kept clear by the tile flags), 2 compacted first product by grid
  // position, 3 by compacted row (the gathers read only rows of cells, so leftovers elsewhere are never read).
  // Leaving mode 2 for 1 or 2 clears the earlier tree's rows; leaving mode 3 for 1 or 2, or turning from 1 to 2,
  // clears Y and the tile flags.
  if (t.lr) {
    CPlace chunks{};
    for (int p = 0; p <= 8; ++p) chunks.blk0[p] = p < 8 ? t.ybase[p] : t.ycht;
    for (int l = 2; l <= LL; ++l) {
      const long long plane = (long long)t.HX[l] * t.HY[l] * t.HZ[l];
      const int next = !((ymask >> l) & 1u) ? 1 : (ypr[l] > 0 ? 3 : 2);
      const int prev = t.ymode[l];
      if (prev == 2 && next != 3 && t.crows[l] > 0) {
        cclear_kernel<<<(unsigned)t.crows[l], 64, 0, c.stream>>>(t.crow[l], plane, chunks, t.Yhi[l], t.Ylo[l]);
        ++c.launches;
      }
      if ((prev == 3 && next != 3) || (prev == 1 && next == 2)) {
        B200_CUDA(cudaMemsetAsync(t.Yhi[l], 0, t.Ybytes[l], c.stream));
        B200_CUDA(cudaMemsetAsync(t.Ylo[l], 0, t.Ybytes[l], c.stream));
        B200_CUDA(cudaMemsetAsync(t.ydirty + 16 * (size_t)t.titem0[l], 0, 16 * (size_t)t.tnitems[l], c.stream));
      }
      t.ymode[l] = next;
    }
  }
  for (int l = 2; l <= LL; ++l) t.crows[l] = 0;
  // rows and cells of every placed level
  CBlocks B{};
  B.l0 = 2;
  B.l1 = LL;
  int nblocks[kMaxHeight] = {};
  for (int l = 2; l <= LL; ++l) {
    P.lv[l].cmode = 0;
    P.lv[l].ypr = 0;
    P.lv[l].rowmap = nullptr;
    if (t.lr) t.yparams->ypr[l] = 0;
    B.b0[l + 1] = B.b0[l];
    if (!((mask >> l) & 1u)) continue;
    const CPlace &C = Cl[l];
    const long long plane = (long long)t.HX[l] * t.HY[l] * t.HZ[l];
    nblocks[l] = C.blk0[8];
    const long long rows = 128LL * C.blk0[8];
    if (t.ccap[l] < rows) {
      for (void *q : {(void *)t.crow[l], (void *)t.ccell[l]})
        if (q) cudaFree(q);
      t.crow[l] = t.ccell[l] = nullptr;
      t.ccap[l] = 0;
      B200_CUDA(cudaMalloc(&t.crow[l], sizeof(int) * rows));
      B200_CUDA(cudaMalloc(&t.ccell[l], sizeof(int) * rows));
      t.ccap[l] = rows;
    }
    B200_CUDA(cudaMemsetAsync(t.crow[l], 0xFF, sizeof(int) * rows, c.stream));
    B200_CUDA(cudaMemsetAsync(t.ccell[l], 0xFF, sizeof(int) * rows, c.stream));
    int *rmap = nullptr;
    if (ypr[l] > 0) {
      if (!t.rowmap[l]) B200_CUDA(cudaMalloc(&t.rowmap[l], sizeof(int) * 8 * plane));
      rmap = t.rowmap[l];
      B200_CUDA(cudaMemsetAsync(rmap, 0xFF, sizeof(int) * 8 * plane, c.stream));
    }
    const int ngl = (int)(g0[l + 1] - g0[l]);
    cgroup_place_kernel<<<ngl, 1024, 0, c.stream>>>(c.lv[l].keys, c.lv[l].n, C, t.cgrp + 8 * g0[l], t.crow[l],
                                                    t.ccell[l], rmap, plane);
    ++c.launches;
    t.crows[l] = (int)rows;
    P.lv[l].crow = t.crow[l];
    P.lv[l].ccell = t.ccell[l];
    for (int p = 0; p <= 8; ++p) P.lv[l].cblk0[p] = C.blk0[p];
    if ((tmask >> l) & 1u) {
      P.lv[l].cmode = 1;
      P.lv[l].cb0 = B.b0[l];
      B.b0[l + 1] = B.b0[l] + C.blk0[8];
      P.lv[l].ypr = ypr[l];
      P.lv[l].rowmap = rmap;
    }
    if (t.lr && ((ymask >> l) & 1u)) {
      LrYParams &Y = *t.yparams;
      if (t.chcap[l] < rows) {
        for (void *q : {(void *)t.Chi[l], (void *)t.Clo[l]})
          if (q) cudaFree(q);
        t.Chi[l] = t.Clo[l] = nullptr;
        t.chcap[l] = 0;
        B200_CUDA(cudaMalloc(&t.Chi[l], sizeof(__half) * rows * t.KP));
        B200_CUDA(cudaMalloc(&t.Clo[l], sizeof(__half) * rows * t.KP));
        t.chcap[l] = rows;
      }
      cuuint64_t dims[2] = {(cuuint64_t)t.KP, (cuuint64_t)rows};
      cuuint64_t strides[1] = {(cuuint64_t)t.KP * 2};
      cuuint32_t box[2] = {KCHUNK, 128};
      B200_CHECK(encode(&Y.mapC_hi[l], t.Chi[l], 2, dims, strides, box));
      B200_CHECK(encode(&Y.mapC_lo[l], t.Clo[l], 2, dims, strides, box));
      Y.crow[l] = t.crow[l];
      for (int p = 0; p <= 8; ++p) Y.cblk0[l][p] = C.blk0[p];
      Y.ypr[l] = ypr[l];
    }
  }
  // first-product items (low rank), finest level first
  if (t.lr) {
    LrYParams &Y = *t.yparams;
    int n = 0;
    for (int l = LL; l >= 2; --l) {
      Y.item0[l] = n;
      Y.nitems[l] = ((ymask >> l) & 1u) ? nblocks[l] * t.nblk : t.tnitems[l];
      n += Y.nitems[l];
    }
    Y.compact_levels = ymask;
  }
  // second-product units, finest level first, and the busy masks of the compacted blocks
  int nunits = 0;
  for (int l = LL; l >= 2; --l) {
    P.lv[l].unit0 = nunits;
    P.lv[l].nunits = P.lv[l].cmode ? nblocks[l] / (t.pair ? 2 : 1) : t.tunits[l];
    nunits += P.lv[l].nunits;
  }
  t.nunits_all = nunits;
  if (t.prefix_cap < nunits + 1) {
    if (t.prefix) cudaFree(t.prefix);
    t.prefix = nullptr;
    t.prefix_cap = 0;
    B200_CUDA(cudaMalloc(&t.prefix, sizeof(int) * (nunits + 1)));
    t.prefix_cap = nunits + 1;
    P.prefix = t.prefix;
  }
  const int nb_all = B.b0[LL + 1];
  if (nb_all > 0) {
    if (t.cbusy_cap < nb_all) {
      if (t.cbusy) cudaFree(t.cbusy);
      t.cbusy = nullptr;
      t.cbusy_cap = 0;
      B200_CUDA(cudaMalloc(&t.cbusy, sizeof(unsigned) * 6 * nb_all));
      t.cbusy_cap = nb_all;
    }
    P.cbusy = t.cbusy;
    cbusy_kernel<<<nb_all, 128, 0, c.stream>>>(P, B, t.cbusy);
    ++c.launches;
  }
  return B200FMM_OK;
}

// The per-tree tables of the tensor-core M2L: occupancy, busy masks, compacted levels and the work units with
// their prefix sums.  They depend on the tree only; execute() builds them beside the near field, before P2M.
b200fmm_status tc_tree_setup(Context &c) {
  DenseTC *t = c.tc;
  if (!t) return fail(B200FMM_ERR_STATE, "tensor-core M2L not initialised");
  const int LL = c.H - 1;
  if (t->built_for_gen != c.tree_gen) B200_CHECK(tc_prepare(c));
  if (t->sat_serial != c.tree_serial) {
    // which cells of each level are occupied: lets the kernel skip empty target tiles and source boxes
    LevelCells C{};
    C.l0 = 2;
    C.l1 = LL;
    C.start[2] = 0;
    for (int a = 0; a < 3; ++a) C.lines[a][2] = 0;
    for (int l = 2; l <= LL; ++l) {
      const long long HX = t->HX[l], HY = t->HY[l], HZ = t->HZ[l];
      C.keys[l] = c.lv[l].keys;
      C.start[l + 1] = C.start[l] + c.lv[l].n;
      C.lines[0][l + 1] = C.lines[0][l] + 8 * (HZ + 1) * (HY + 1);
      C.lines[1][l + 1] = C.lines[1][l] + 8 * (HZ + 1) * (HX + 1);
      C.lines[2][l + 1] = C.lines[2][l] + 8 * (HY + 1) * (HX + 1);
    }
    const TcParams &P0 = *t->params;
    // full levels (every cell present, as in uniform trees) need no occupancy tables
    unsigned full_levels = 0;
    for (int l = 2; l <= LL; ++l)
      if (c.lv[l].n == (1LL << (3 * l))) full_levels |= 1u << l;
    const bool all_full = full_levels == (((1u << (LL + 1)) - 1u) & ~3u);
    if (t->lr) t->yparams->full_levels = full_levels;
    B200_CUDA(cudaMemsetAsync(t->busy, 0, sizeof(unsigned) * 6 * t->ntiles_all, c.stream));
    if (!all_full) {
      B200_CUDA(cudaMemsetAsync(t->sat, 0, t->satn * sizeof(int), c.stream));
      if (C.start[LL + 1] > 0) {
        occ_mark_kernel<<<grid_for(C.start[LL + 1], 256), 256, 0, c.stream>>>(P0, C);
        ++c.launches;
      }
      for (int a = 0; a < 3; ++a) {
        sat_pass_kernel<<<grid_for(C.lines[a][LL + 1], 128), 128, 0, c.stream>>>(P0, C, a);
        ++c.launches;
      }
    }
    busy_mask_kernel<<<grid_for(t->ntiles_all * 189, 256), 256, 0, c.stream>>>(P0, 2, LL, t->ntiles_all, full_levels,
                                                                                 t->busy);
    ++c.launches;
    // compacted levels: placement, unit numbering and block masks
    B200_CHECK(compact_setup(c, *t));
    // the work of every unit of every level and its prefix sums, from which each launch splits its units
    // into ranges of equal work
    t->params->shard = c.shard_count > 1 ? c.d_shard : nullptr;
    TcParams Pw = *t->params;
    Pw.l0 = 2;
    Pw.l1 = LL;
    unit_work_kernel<<<grid_for(t->nunits_all, 256), 256, 0, c.stream>>>(Pw, t->nunits_all, t->prefix);
    unit_scan_kernel<<<1, 1024, 0, c.stream>>>(t->nunits_all, t->prefix);
    c.launches += 2;
    t->sat_serial = c.tree_serial;
  }
  return B200FMM_OK;
}

void tc_invalidate_units(Context &c) {
  if (c.tc) c.tc->sat_serial = -1;
}

bool tc_tables_pending(const Context &c) {
  return c.tc && (c.tc->built_for_gen != c.tree_gen || c.tc->sat_serial != c.tree_serial);
}

b200fmm_status run_m2l_tc(Context &c, int level) {
  DenseTC *t = c.tc;
  if (!t) return fail(B200FMM_ERR_STATE, "tensor-core M2L not initialised");
  const int LL = c.H - 1;
  if (level != -1 && (level < 2 || level > LL)) return fail(B200FMM_ERR_INVALID, "m2l: level out of range");
  B200_CHECK(tc_tree_setup(c));
  const int l0 = level == -1 ? 2 : level, l1 = level == -1 ? LL : level;
  {
    // the multipoles of all levels of the launch: their maxima, the level scales, then the packed FP16 hi / lo
    // grids (every position written, empty ones with zeros)
    PackLevels L{};
    L.l0 = l0;
    L.l1 = l1;
    L.pos0[l0] = 0;
    long long maxval = 0;
    for (int l = l0; l <= l1; ++l) {
      L.M[l] = c.lv[l].M;
      L.nval[l] = c.lv[l].n * c.R * c.nn;
      maxval = std::max(maxval, L.nval[l]);
      L.HX[l] = t->HX[l];
      L.HY[l] = t->HY[l];
      L.HZ[l] = t->HZ[l];
      L.side[l] = 1 << l;
      L.grid[l] = c.lv[l].grid;
      L.hi[l] = t->Ahi[l];
      L.lo[l] = t->Alo[l];
      L.scale_l[l] = 2.0 / (c.cfg.box_width / (double)(1LL << l));
      const bool compact = t->lr && ((t->yparams->compact_levels >> l) & 1u);
      L.pos0[l + 1] = L.pos0[l] + (compact ? 0LL : 8LL * c.R * t->HZ[l] * t->HY[l] * t->HX[l]);
    }
    const int shift = t->lr ? t->lr_shift : SB;
    if (c.mmax_ready) {
      // the upward pass of this evaluation recorded the maxima as it wrote the multipoles
      level_scale_kernel<<<1, 32, 0, c.stream>>>(L, c.d_mmax, kMmaxSlots, shift, t->scal);
    } else {
      B200_CUDA(cudaMemsetAsync(t->amax + l0, 0, sizeof(unsigned long long) * (l1 - l0 + 1), c.stream));
      const unsigned gx = (unsigned)std::max<long long>(1, std::min<long long>(256, grid_for(maxval, 256)));
      absmax_levels_kernel<<<dim3(gx, l1 - l0 + 1), 256, 0, c.stream>>>(L, t->amax);
      level_scale_kernel<<<1, 32, 0, c.stream>>>(L, t->amax, 1, shift, t->scal);
      ++c.launches;
    }
    if (L.pos0[l1 + 1] > 0) {
      pack_levels_kernel<<<(unsigned)L.pos0[l1 + 1], 128, 0, c.stream>>>(L, c.R, c.nn, t->KP, t->scal);
      ++c.launches;
    }
    ++c.launches;
    if (t->lr)
      for (int l = l0; l <= l1; ++l)
        if (((t->yparams->compact_levels >> l) & 1u) && t->crows[l] > 0) {
          pack_compact_kernel<<<(unsigned)t->crows[l], 128, 0, c.stream>>>(t->ccell[l], c.lv[l].M, c.nn, t->KP,
                                                                           t->scal + 2 * l, t->Chi[l], t->Clo[l]);
          ++c.launches;
        }
  }
  // units are ordered by level, finest first: levels [l0, l1] are one contiguous range
  TcParams &P = *t->params;
  P.l0 = l0;
  P.l1 = l1;
  P.u_begin = P.lv[l1].unit0;
  P.u_end = P.lv[l0].unit0 + P.lv[l0].nunits;
  P.gather = 0;
  for (int l = l0; l <= l1; ++l)
    if (P.lv[l].cmode) P.gather = 1;
  if (P.u_end <= P.u_begin) return B200FMM_OK;
  const size_t smem = (size_t)t->stages * t->stage_bytes + TV_BYTES + 1024;
  const int grid = t->grid;  // persistent: one CTA (pair) per SM (pair of SMs)
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = t->pair ? 2 : 1;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(TC_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c.stream;
  cfg.attrs = at;
  cfg.numAttrs = t->pair ? 1 : 0;
  B200_CUDA(record_event(c, 8));
  if (t->lr) {
    // first product: Y = V^T M for every source cell of levels [l0, l1]
    LrYParams &Y = *t->yparams;
    Y.l0 = l0;
    Y.l1 = l1;
    const int ny = Y.item0[l0] + Y.nitems[l0] - Y.item0[l1];
    if (ny > 0) {
      int dev_sms = 148;
      cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c.device);
      cudaLaunchConfig_t ycfg = {};
      cudaLaunchAttribute yat[1];
      yat[0].id = cudaLaunchAttributeClusterDimension;
      yat[0].val.clusterDim.x = t->ypair ? 2 : 1;
      yat[0].val.clusterDim.y = 1;
      yat[0].val.clusterDim.z = 1;
      ycfg.gridDim = dim3(t->ypair ? 2 * std::min(dev_sms / 2, ny) : std::min(dev_sms, ny));
      ycfg.blockDim = dim3(TC_THREADS);
      ycfg.dynamicSmemBytes = (size_t)t->ystages * t->ystage_bytes + 1024;
      ycfg.stream = c.stream;
      ycfg.attrs = yat;
      ycfg.numAttrs = t->ypair ? 1 : 0;
      if (t->ypair)
        B200_CUDA(cudaLaunchKernelEx(&ycfg, lr_y_kernel<true>, Y));
      else
        B200_CUDA(cudaLaunchKernelEx(&ycfg, lr_y_kernel<false>, Y));
      ++c.launches;
    }
  }
  auto launch = [&](auto kern) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernelEx(&cfg, kern, P);
  };
  switch (t->NP) {
  // one instance per (pair, form, gathers): launches without compacted levels run the tile form alone
#define B200_TC_PICK(CWV, NHV, PR, LRV)                                                             \
  (P.gather ? launch(m2l_tc_kernel<CWV, NHV, PR, LRV, true>) : launch(m2l_tc_kernel<CWV, NHV, PR, LRV, false>))
#define B200_TC_CASE(NPV, CWV, NHV)                                                                \
  case NPV:                                                                                          \
    if (t->pair)                                                                                     \
      B200_CUDA(t->lr ? B200_TC_PICK(CWV, NHV, true, true) : B200_TC_PICK(CWV, NHV, true, false));   \
    else                                                                                             \
      B200_CUDA(t->lr ? B200_TC_PICK(CWV, NHV, false, true) : B200_TC_PICK(CWV, NHV, false, false)); \
    break;
    B200_TC_CASE(32, 16, 1)
    B200_TC_CASE(64, 32, 1)
    B200_TC_CASE(128, 64, 1)
    B200_TC_CASE(224, 112, 1)
    B200_TC_CASE(352, 176, 2)
#undef B200_TC_CASE
#undef B200_TC_PICK
    default:
      return fail(B200FMM_ERR_UNSUPPORTED, "no tensor-core M2L instance for this order");
  }
  B200_CUDA(record_event(c, 9));
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

}  // namespace b200

namespace b200 {

// Splits of the 189 transfer vectors of each tile into work items: set (0 = automatic) and read back.
void tc_set_splits(Context &c, int splits) {
  if (!c.tc) return;
  c.tc->splits = splits;
  c.tc->built_for_gen = -1;  // the item list is rebuilt by the next run
}
int tc_splits_used(const Context &c) { return c.tc ? c.tc->splits_used : 0; }

// Low-rank form in use: the rank of every slot and, per source parity, the sum of the ranks of the slots
// that the parity's cells feed.
bool tc_lowrank_info(const Context &c, int *rank_of_slot, double *rank_fed) {
  if (!c.tc || !c.tc->lr) return false;
  std::memcpy(rank_of_slot, c.tc->lr_rank, sizeof(int) * 343);
  std::memcpy(rank_fed, c.tc->lr_rank_fed, sizeof(double) * 8);
  return true;
}

}  // namespace b200
