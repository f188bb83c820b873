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
// Roles: warp 0 = TMA producer (one elected thread), warp 1 = MMA issuer (one thread) and TMEM owner,
// warps 2..9 = epilogue (TMEM lane quarter = warp % 4, column half = (warp - 2) / 4).  Shared memory: STAGES x {A_hi, A_lo, B_hi, B_lo}
// K-chunks with the 64-byte swizzle the UMMA descriptors describe.  Every mbarrier wait is bounded; a wait
// that runs out sets a device status word, the CTA abandons its work, frees its TMEM and returns.
#include "common.cuh"

#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace b200 {

namespace {

constexpr int TC_THREADS = 320;
constexpr int TILE_X = 8, TILE_Y = 4, TILE_Z = 4;  // 128 targets
constexpr int KCHUNK = 32;                          // fp16 elements per 64-byte swizzle row
constexpr int SB = 15;                              // operator pre-scale 2^15
constexpr int MAX_STAGES = 4;
constexpr long long WAIT_LIMIT = 1LL << 22;

struct TcItem {
  short level, rhs, parity, split;
  short bx, by, bz;
  short t0, t1;
};

struct TcLevel {
  int HX, HY, HZ;      // padded half-grid extents
  int side;            // real grid side 2^level
  int *grid;           // [side^3] cell index or -1
  double *L;           // locals of the level
  double *scale_out;   // device scalar: scale_l * 2^-(sA + SB)
  const int *sat;      // [8][HZ+1][HY+1][HX+1] occupied cells of each parity grid below (x, y, z), exclusive
  int tile0;           // first tile of this level in the busy masks
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
  const TcItem *items;
  int item0, nitems;  // items [item0, item0 + nitems) of the list run in this launch
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
};

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
// UMMA shared-memory descriptor: K-major, 64-byte swizzle, rows of 64 B in 8-row groups 512 B apart.
__device__ __forceinline__ unsigned long long sdesc(const void *p) {
  const unsigned long long a = su32(p);
  return ((a >> 4) & 0x3FFFull) | (1ull << 16) | (32ull << 32) | (1ull << 46) | (4ull << 61);
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

// add N accumulator columns starting at TMEM address taddr (a multiple of 16 columns) into acc[0..N)
template <int N>
__device__ __forceinline__ void drain_cols(unsigned taddr, float *acc) {
  static_assert(N % 16 == 0, "drained in groups of 16 columns");
#pragma unroll
  for (int c0 = 0; c0 < N; c0 += 16) {
    unsigned r[16];
    tmem_ld16(taddr + c0, r);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[c0 + i] += __uint_as_float(r[i]);
  }
}

// The source box of transfer vector e for an item: parity grid sp, half-grid origin (ox, oy, oz), operator
// slot.  Every warp role derives the same box, and skips the transfer vectors whose source box is empty
// (those A tiles are all zero) and the items whose target tile is empty, so that sparse trees (surface or
// clustered distributions) cost only their occupied tiles.
struct SrcBox {
  int sp, ox, oy, oz, slot;
};
__device__ __forceinline__ SrcBox src_box(const TcParams &P, const TcItem &w, int e) {
  const int c = w.parity;
  const int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;
  const int dx = P.off[c][e][0], dy = P.off[c][e][1], dz = P.off[c][e][2];
  SrcBox b;
  b.sp = (((cx + dx) & 1) << 2) | (((cy + dy) & 1) << 1) | ((cz + dz) & 1);
  b.ox = w.bx * TILE_X + ((cx + dx) >> 1);
  b.oy = w.by * TILE_Y + ((cy + dy) >> 1);
  b.oz = w.bz * TILE_Z + ((cz + dz) >> 1);
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
__device__ __forceinline__ BusyMask busy_mask(const TcParams &P, const TcItem &w) {
  const unsigned *m = P.busy + 6 * tile_id(P, w.level, w.parity, w.bx, w.by, w.bz);
  BusyMask b;
#pragma unroll
  for (int k = 0; k < 6; ++k) b.w[k] = m[k];
  return b;
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
template <int CW, int NHALF>
__global__ void __launch_bounds__(TC_THREADS, 1) m2l_tc_kernel(const __grid_constant__ TcParams P) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned stage buffers (the swizzle pattern repeats every 512 B)
  unsigned char *smem = (unsigned char *)(((unsigned long long)smem_raw + 1023) & ~1023ull);
  __shared__ __align__(8) unsigned long long full_bar[MAX_STAGES], empty_bar[MAX_STAGES];
  __shared__ __align__(8) unsigned long long acc_full[2], acc_empty[2][2];
  __shared__ unsigned tmem_base_sh;
  __shared__ volatile int abort_sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = P.stages;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b][0], 8);  // one arrive per epilogue warp
      mbar_init(&acc_empty[b][1], 8);
    }
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_sh)),
                 "r"(P.ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = tmem_base_sh;

  const int a_bytes = TILE_X * TILE_Y * TILE_Z * KCHUNK * 2;  // 8 KB
  const int b_bytes = P.NP * KCHUNK * 2;

  if (warp == 0) {
    // ------------------------------------------------ TMA producer
    if (lane == 0) {
      int stage = 0;
      unsigned phase = 0;
      for (int it = blockIdx.x; it < P.nitems && !abort_sh; it += gridDim.x) {
        const TcItem w = P.items[P.item0 + it];
        const BusyMask bm = busy_mask(P, w);
        if (!bm.tile()) continue;
        for (int e = w.t0; e < w.t1 && !abort_sh; ++e) {
          if (!bm.src(e)) continue;
          const SrcBox sb = src_box(P, w, e);
          const int sp = sb.sp, ox = sb.ox, oy = sb.oy, oz = sb.oz, slot = sb.slot;
          for (int kc = 0; kc < P.NK; ++kc) {
            if (!mbar_wait(&empty_bar[stage], phase ^ 1)) {
              atomicExch(P.status + 1, 1);
              abort_sh = 1;
              break;
            }
            unsigned char *sbuf = smem + (size_t)stage * P.stage_bytes;
            mbar_expect_tx(&full_bar[stage], 2 * a_bytes + 2 * b_bytes);
            tma_load_5d(sbuf, &P.mapA_hi[w.level], &full_bar[stage], kc * KCHUNK, ox, oy, oz, w.rhs * 8 + sp);
            tma_load_5d(sbuf + a_bytes, &P.mapA_lo[w.level], &full_bar[stage], kc * KCHUNK, ox, oy, oz,
                        w.rhs * 8 + sp);
            for (int h = 0; h < P.NHALF; ++h) {
              tma_load_3d(sbuf + 2 * a_bytes + h * P.NH * 64, &P.mapB_hi, &full_bar[stage], kc * KCHUNK, h * P.NH, slot);
              tma_load_3d(sbuf + 2 * a_bytes + b_bytes + h * P.NH * 64, &P.mapB_lo, &full_bar[stage], kc * KCHUNK,
                          h * P.NH, slot);
            }
            if (++stage == S) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      const unsigned idesc = (1u << 4) | ((unsigned)(P.NH >> 3) << 17) | ((unsigned)(128 >> 4) << 24);
      int stage = 0;
      unsigned phase = 0;
      unsigned empty_par = 0xFu;  // parity to wait for, per (buffer, half): starts at 1 (passes at once)
      int seg = 0;
      const bool defer = (P.nbuf == 1 && NHALF == 2);
      for (int it = blockIdx.x; it < P.nitems && !abort_sh; it += gridDim.x) {
        const TcItem w = P.items[P.item0 + it];
        const BusyMask bm = busy_mask(P, w);
        if (!bm.tile()) continue;
        for (int e = w.t0; e < w.t1 && !abort_sh; ++e) {
          if (!bm.src(e)) continue;
          for (int sg = 0; sg < P.nseg && !abort_sh; ++sg, ++seg) {
            const int k0 = sg * P.NK / P.nseg, k1 = (sg + 1) * P.NK / P.nseg;
            const int b = P.nbuf == 2 ? (seg & 1) : 0;
            const unsigned dbase = tmem + (unsigned)(b * P.NP);
            // the epilogue has drained this accumulator (both halves, or half 0 only when deferring half 1)
            for (int h = 0; h < (defer ? 1 : NHALF); ++h) {
              const int bit = b * 2 + h;
              if (!mbar_wait(&acc_empty[b][h], (empty_par >> bit) & 1u)) {
                atomicExch(P.status + 1, 1);
                abort_sh = 1;
                break;
              }
              empty_par ^= 1u << bit;
            }
            if (abort_sh) break;
            tc_fence_after();
            for (int kc = k0; kc < k1; ++kc) {
              if (!mbar_wait(&full_bar[stage], phase)) {
                atomicExch(P.status + 1, 1);
                abort_sh = 1;
                break;
              }
              tc_fence_after();
              const unsigned char *sbuf = smem + (size_t)stage * P.stage_bytes;
              const unsigned char *ahi = sbuf, *alo = sbuf + a_bytes;
              const unsigned char *bhi = sbuf + 2 * a_bytes, *blo = sbuf + 2 * a_bytes + b_bytes;
              const bool firstc = (kc == k0);
#pragma unroll
              for (int h = 0; h < NHALF; ++h) {
                if (firstc && defer && h == 1) {
                  if (!mbar_wait(&acc_empty[0][1], (empty_par >> 1) & 1u)) {
                    atomicExch(P.status + 1, 1);
                    abort_sh = 1;
                    break;
                  }
                  empty_par ^= 2u;
                  tc_fence_after();
                }
                const unsigned d = dbase + h * P.NH;
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                  const int bo = h * P.NH * 64 + ks * 32;
                  // the small cross terms first, the leading term last
                  mma_f16(d, sdesc(ahi + ks * 32), sdesc(blo + bo), idesc, (firstc && ks == 0) ? 0u : 1u);
                  mma_f16(d, sdesc(alo + ks * 32), sdesc(bhi + bo), idesc, 1u);
                  mma_f16(d, sdesc(ahi + ks * 32), sdesc(bhi + bo), idesc, 1u);
                }
              }
              if (abort_sh) break;
              mma_commit(&empty_bar[stage]);  // frees the stage once these MMAs have read it
              if (++stage == S) {
                stage = 0;
                phase ^= 1;
              }
            }
            mma_commit(&acc_full[b]);  // segment accumulated
          }
        }
      }
    }
  } else {
    // ------------------------------------------------ epilogue (warps 2..9)
    constexpr int SPLIT = 16 * ((CW + 31) / 32);
    const int q = warp & 3;              // TMEM lane quarter this warp may access
    const int ch = (warp - 2) >> 2;      // which part of each half
    const int row = q * 32 + lane;       // target within the tile
    const unsigned tlane = tmem + ((unsigned)(q * 32) << 16);
    unsigned full_par = 0;
    int seg = 0;
    float acc[CW];
#pragma unroll
    for (int i = 0; i < CW; ++i) acc[i] = 0.f;
    for (int it = blockIdx.x; it < P.nitems && !abort_sh; it += gridDim.x) {
      const TcItem w = P.items[P.item0 + it];
      int nbusy = 0;  // transfer vectors of this item that the MMA warp runs
      const BusyMask bm = busy_mask(P, w);
      if (bm.tile())
        for (int e = w.t0; e < w.t1; ++e) nbusy += bm.src(e) ? 1 : 0;
      if (nbusy == 0) continue;  // nothing accumulated: no flush
      const int nseg_item = nbusy * P.nseg;
      for (int sgi = 0; sgi < nseg_item; ++sgi, ++seg) {
        const int b = P.nbuf == 2 ? (seg & 1) : 0;
        if (!mbar_wait(&acc_full[b], (full_par >> b) & 1u)) {
          atomicExch(P.status + 1, 1);
          abort_sh = 1;
          break;
        }
        full_par ^= 1u << b;
        tc_fence_after();
        const unsigned tb = tlane + (unsigned)(b * P.NP);
        if constexpr (NHALF == 1) {
          drain_cols<CW>(tb + ch * CW, acc);
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[b][0]);
        } else {
          // both parts drain G = CW - SPLIT columns of each half into acc[0, G) and acc[SPLIT, CW); the
          // remaining 16-column group, acc[G, SPLIT), comes from half 0 for part 0 and half 1 for part 1
          constexpr int G = CW - SPLIT;
          static_assert(SPLIT - G == 16, "one extra group of 16 columns");
          drain_cols<G>(tb + (ch == 0 ? 0 : SPLIT), acc);
          if (ch == 0) drain_cols<16>(tb + G, acc + G);
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[b][0]);
          if (ch != 0) drain_cols<16>(tb + CW + G, acc + G);
          drain_cols<G>(tb + CW + (ch == 0 ? 0 : SPLIT), acc + SPLIT);
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[b][1]);
        }
      }
      if (abort_sh) break;
      // flush the item's sums into the FP64 locals
      const TcLevel &Lv = P.lv[w.level];
      const int c = w.parity;
      const int hx = w.bx * TILE_X + (row & 7), hy = w.by * TILE_Y + ((row >> 3) & 3), hz = w.bz * TILE_Z + (row >> 5);
      const int gx = 2 * hx + ((c >> 2) & 1), gy = 2 * hy + ((c >> 1) & 1), gz = 2 * hz + (c & 1);
      int cell = -1;
      if (gx < Lv.side && gy < Lv.side && gz < Lv.side) cell = Lv.grid[((long long)gz * Lv.side + gy) * Lv.side + gx];
      if (cell >= 0) {
        const double sc = *Lv.scale_out;
        double *Lrow = Lv.L + ((long long)cell * P.R + w.rhs) * P.nn;
        // first accumulator column of this thread's part in each half, and the part's width in half 0
        const int n0 = NHALF == 1 ? ch * CW : (ch == 0 ? 0 : SPLIT);
        const int w0 = NHALF == 1 ? CW : (ch == 0 ? SPLIT : CW - SPLIT);
        const int n1 = NHALF == 1 ? 0 : (ch == 0 ? CW : 2 * CW - SPLIT);
#pragma unroll
        for (int i = 0; i < CW; ++i) {
          const int n = i < w0 ? n0 + i : n1 + (i - w0);
          if (n < P.nn) atomicAdd(Lrow + n, (double)acc[i] * sc);
        }
      }
#pragma unroll
      for (int i = 0; i < CW; ++i) acc[i] = 0.f;
    }
  }
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P.ncols));
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

// busy masks of every level: one thread per (tile, transfer vector); tiles are numbered across levels
__global__ void busy_mask_kernel(const __grid_constant__ TcParams P, int l0, int l1, long long ntiles,
                                 unsigned *__restrict__ busy) {
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
  w.bx = (short)(tl % TX);
  w.by = (short)((tl / TX) % TY);
  w.bz = (short)((tl / ((long long)TX * TY)) % TZ);
  w.parity = (short)(tl / ((long long)TX * TY * TZ));
  unsigned *m = busy + 6 * tg;
  const SrcBox b = src_box(P, w, e);
  if (box_count(L, b.sp, b.ox, b.oy, b.oz, TILE_X, TILE_Y, TILE_Z) > 0) atomicOr(m + (e >> 5), 1u << (e & 31));
  if (e == 0 && box_count(L, w.parity, w.bx * TILE_X, w.by * TILE_Y, w.bz * TILE_Z, TILE_X, TILE_Y, TILE_Z) > 0)
    atomicOr(m + 5, 1u << 31);
}

// max |M| of a level -> bit pattern (non-negative doubles order like their bit patterns)
__global__ void absmax_kernel(long long n, const double *__restrict__ v, unsigned long long *__restrict__ out) {
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(v[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// 2^sA with sA chosen so that max|M| * 2^sA ~ 2^14, and the epilogue factor scale_l * 2^-(sA + SB)
__global__ void level_scale_kernel(const unsigned long long *__restrict__ amax, double scale_l,
                                   double *__restrict__ pre, double *__restrict__ post) {
  const double m = __longlong_as_double((long long)*amax);
  int e = 0;
  if (m > 0) frexp(m, &e);  // m = f * 2^e, f in [0.5, 1)
  const int sA = 14 - e;
  *pre = ldexp(1.0, sA);
  *post = scale_l * ldexp(1.0, -(sA + SB));
}

__global__ void pack_multipoles(long long ncells, int R, int nn, int KP, int HX, int HY, int HZ,
                                const long long *__restrict__ keys, const double *__restrict__ M,
                                const double *__restrict__ pre, __half *__restrict__ hi, __half *__restrict__ lo) {
  const long long cell = blockIdx.x;
  int ix, iy, iz;
  morton_decode3(keys[cell], ix, iy, iz);
  const int c = ((ix & 1) << 2) | ((iy & 1) << 1) | (iz & 1);
  const double s = *pre;
  for (int r = 0; r < R; ++r) {
    const long long base = ((((long long)(r * 8 + c) * HZ + (iz >> 1)) * HY + (iy >> 1)) * HX + (ix >> 1)) * KP;
    for (int n = threadIdx.x; n < nn; n += blockDim.x) {
      const double a = M[(cell * R + r) * nn + n] * s;
      const __half h = __double2half(a);
      hi[base + n] = h;
      lo[base + n] = __double2half(a - (double)__half2float(h));
    }
  }
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
  __half *Bhi = nullptr, *Blo = nullptr;
  // per level
  __half *Ahi[kMaxHeight] = {}, *Alo[kMaxHeight] = {};
  size_t Abytes[kMaxHeight] = {};
  int HX[kMaxHeight] = {}, HY[kMaxHeight] = {}, HZ[kMaxHeight] = {};
  double *scal = nullptr;                 // [kMaxHeight][2]: pre, post
  unsigned long long *amax = nullptr;     // [kMaxHeight]
  TcItem *items = nullptr;
  int nitems = 0;
  int *sat = nullptr;                     // occupancy summed-area tables of all levels
  size_t satn = 0, sat_off[kMaxHeight] = {};
  long long sat_serial = -1;              // tree the tables describe
  unsigned *busy = nullptr;               // busy masks of every tile of every level
  long long ntiles_all = 0;
  int lvl_begin[kMaxHeight] = {}, lvl_end[kMaxHeight] = {};
  long long built_for_N = -1;             // tree the per-level buffers were sized for
  int splits = 0;                         // transfer-vector splits per tile: 0 = by SM fill, else fixed
  int splits_used = 0;
  int built_for_gen = -1;                 // tree generation the tensor maps / pointers belong to
  TcParams *params = nullptr;             // host copy
  int grid = 0;
};

static b200fmm_status encode(CUtensorMap *map, void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                             const cuuint32_t *box) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(B200FMM_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available");
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, (cuuint32_t)rank, base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(B200FMM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return B200FMM_OK;
}

b200fmm_status tc_init(Context &c) {
  B200_CHECK(build_dense_operators(c));  // FP64 K on the device
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
  t->stage_bytes = 2 * (TILE_X * TILE_Y * TILE_Z * KCHUNK * 2) + 2 * t->NP * KCHUNK * 2;
  t->stages = std::min(MAX_STAGES, (220 * 1024) / t->stage_bytes);
  if (t->stages < 2) return fail(B200FMM_ERR_UNSUPPORTED, "stage buffers do not fit in shared memory");
  t->nbuf = 2 * t->NP <= 512 ? 2 : 1;
  t->ncols = 32;
  while (t->ncols < t->nbuf * t->NP) t->ncols *= 2;
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
  B200_CUDA(cudaMalloc(&t->scal, sizeof(double) * kMaxHeight * 2));
  B200_CUDA(cudaMalloc(&t->amax, sizeof(unsigned long long) * kMaxHeight));
  t->params = new TcParams();
  std::memset(t->params, 0, sizeof(TcParams));
  cuuint64_t dims[3] = {(cuuint64_t)t->KP, (cuuint64_t)t->NP, 343};
  cuuint64_t strides[2] = {(cuuint64_t)t->KP * 2, (cuuint64_t)t->KP * 2 * t->NP};
  cuuint32_t box[3] = {KCHUNK, (cuuint32_t)t->NH, 1};
  B200_CHECK(encode(&t->params->mapB_hi, t->Bhi, 3, dims, strides, box));
  B200_CHECK(encode(&t->params->mapB_lo, t->Blo, 3, dims, strides, box));
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c.device);
  t->grid = dev_sms;
  return B200FMM_OK;
}

void tc_free(Context &c) {
  DenseTC *t = c.tc;
  if (!t) return;
  for (void *p : {(void *)t->Bhi, (void *)t->Blo, (void *)t->scal, (void *)t->amax, (void *)t->items, (void *)t->busy})
    if (p) cudaFree(p);
  for (int l = 0; l < kMaxHeight; ++l) {
    if (t->Ahi[l]) cudaFree(t->Ahi[l]);
    if (t->Alo[l]) cudaFree(t->Alo[l]);
  }
  if (t->sat) cudaFree(t->sat);
  delete t->params;
  delete t;
  c.tc = nullptr;
}

// (Re)build the per-level A buffers, tensor maps and the work-item list for the current tree.
static b200fmm_status tc_prepare(Context &c) {
  DenseTC *t = c.tc;
  TcParams &P = *t->params;
  const int LL = c.H - 1;
  std::vector<TcItem> items;
  long long ntiles = 0;
  t->ntiles_all = 0;
  size_t sat_total = 0;
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
    B200_CHECK(encode(&P.mapA_hi[l], t->Ahi[l], 5, dims, st, box));
    B200_CHECK(encode(&P.mapA_lo[l], t->Alo[l], 5, dims, st, box));
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
    ntiles += (long long)c.R * 8 * (t->HX[l] / TILE_X) * (t->HY[l] / TILE_Y) * (t->HZ[l] / TILE_Z);
  }
  // split the 189 transfer vectors of each tile so that the items fill the SMs evenly
  int ns = 1;
  for (int k = 1; k <= 8; ++k) {
    const long long n = ntiles * k;
    const long long rounds = (n + t->grid - 1) / t->grid;
    ns = k;
    if ((double)n / (double)(rounds * t->grid) >= 0.9) break;
  }
  if (t->splits > 0) ns = t->splits;  // chosen by b200fmm_autotune
  if (const char *e = getenv("B200FMM_TC_SPLITS")) ns = std::max(1, std::min(189, atoi(e)));
  t->splits_used = ns;
  for (int l = LL; l >= 2; --l) {
    t->lvl_begin[l] = (int)items.size();
    for (int r = 0; r < c.R; ++r)
      for (int par = 0; par < 8; ++par)
        for (int bz = 0; bz < t->HZ[l] / TILE_Z; ++bz)
          for (int by = 0; by < t->HY[l] / TILE_Y; ++by)
            for (int bx = 0; bx < t->HX[l] / TILE_X; ++bx)
              for (int s = 0; s < ns; ++s) {
                TcItem w;
                w.level = (short)l;
                w.rhs = (short)r;
                w.parity = (short)par;
                w.split = (short)s;
                w.bx = (short)bx;
                w.by = (short)by;
                w.bz = (short)bz;
                w.t0 = (short)(189 * s / ns);
                w.t1 = (short)(189 * (s + 1) / ns);
                items.push_back(w);
              }
    t->lvl_end[l] = (int)items.size();
  }
  if (t->satn != sat_total) {
    if (t->sat) cudaFree(t->sat);
    B200_CUDA(cudaMalloc(&t->sat, std::max<size_t>(sat_total, 1) * sizeof(int)));
    t->satn = sat_total;
  }
  for (int l = 2; l <= LL; ++l) P.lv[l].sat = t->sat + t->sat_off[l];
  if (t->busy) cudaFree(t->busy);
  B200_CUDA(cudaMalloc(&t->busy, sizeof(unsigned) * 6 * std::max<long long>(t->ntiles_all, 1)));
  P.busy = t->busy;
  if (t->items) cudaFree(t->items);
  B200_CUDA(cudaMalloc(&t->items, sizeof(TcItem) * items.size()));
  B200_CUDA(cudaMemcpy(t->items, items.data(), sizeof(TcItem) * items.size(), cudaMemcpyHostToDevice));
  t->nitems = (int)items.size();
  P.items = t->items;
  P.item0 = 0;
  P.nitems = t->nitems;
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
  if (const char *e = getenv("B200FMM_TC_SEGMENTS")) P.nseg = std::max(1, std::min(t->NK, atoi(e)));
  std::memcpy(P.off, c.itab.off, sizeof(P.off));
  std::memcpy(P.slot, c.itab.slot, sizeof(P.slot));
  P.status = c.d_status;
  t->built_for_N = c.N;
  t->built_for_gen = c.tree_gen;
  return B200FMM_OK;
}

b200fmm_status run_m2l_tc(Context &c, int level) {
  DenseTC *t = c.tc;
  if (!t) return fail(B200FMM_ERR_STATE, "tensor-core M2L not initialised");
  const int LL = c.H - 1;
  if (level != -1 && (level < 2 || level > LL)) return fail(B200FMM_ERR_INVALID, "m2l: level out of range");
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
    B200_CUDA(cudaMemsetAsync(t->sat, 0, t->satn * sizeof(int), c.stream));
    B200_CUDA(cudaMemsetAsync(t->busy, 0, sizeof(unsigned) * 6 * t->ntiles_all, c.stream));
    if (C.start[LL + 1] > 0) {
      occ_mark_kernel<<<grid_for(C.start[LL + 1], 256), 256, 0, c.stream>>>(P0, C);
      ++c.launches;
    }
    for (int a = 0; a < 3; ++a) {
      sat_pass_kernel<<<grid_for(C.lines[a][LL + 1], 128), 128, 0, c.stream>>>(P0, C, a);
      ++c.launches;
    }
    busy_mask_kernel<<<grid_for(t->ntiles_all * 189, 256), 256, 0, c.stream>>>(P0, 2, LL, t->ntiles_all, t->busy);
    ++c.launches;
    t->sat_serial = c.tree_serial;
  }
  const int l0 = level == -1 ? 2 : level, l1 = level == -1 ? LL : level;
  for (int l = l0; l <= l1; ++l) {
    const Level &Lv = c.lv[l];
    B200_CUDA(cudaMemsetAsync(t->amax + l, 0, sizeof(unsigned long long), c.stream));
    B200_CUDA(cudaMemsetAsync(t->Ahi[l], 0, t->Abytes[l], c.stream));
    B200_CUDA(cudaMemsetAsync(t->Alo[l], 0, t->Abytes[l], c.stream));
    if (Lv.n == 0) continue;
    const long long cnt = Lv.n * c.R * c.nn;
    absmax_kernel<<<std::min<long long>(1024, grid_for(cnt, 256)), 256, 0, c.stream>>>(cnt, Lv.M, t->amax + l);
    level_scale_kernel<<<1, 1, 0, c.stream>>>(t->amax + l, 2.0 / (c.cfg.box_width / (double)(1LL << l)),
                                              t->scal + 2 * l, t->scal + 2 * l + 1);
    pack_multipoles<<<(unsigned)Lv.n, 128, 0, c.stream>>>(Lv.n, c.R, c.nn, t->KP, t->HX[l], t->HY[l], t->HZ[l],
                                                          Lv.keys, Lv.M, t->scal + 2 * l, t->Ahi[l], t->Alo[l]);
    c.launches += 3;
  }
  // items are ordered by level, finest first: levels [l0, l1] are one contiguous range
  TcParams &P = *t->params;
  P.item0 = t->lvl_begin[l1];
  P.nitems = t->lvl_end[l0] - t->lvl_begin[l1];
  if (P.nitems <= 0) return B200FMM_OK;
  const size_t smem = (size_t)t->stages * t->stage_bytes + 1024;
  const int grid = std::min(t->grid, P.nitems);
  B200_CUDA(record_event(c, 8));
  switch (t->NP) {
#define B200_TC_CASE(NPV, CWV, NHV)                                                                              \
  case NPV:                                                                                                        \
    B200_CUDA(cudaFuncSetAttribute(m2l_tc_kernel<CWV, NHV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    m2l_tc_kernel<CWV, NHV><<<grid, TC_THREADS, smem, c.stream>>>(P);                                              \
    break;
    B200_TC_CASE(32, 16, 1)
    B200_TC_CASE(64, 32, 1)
    B200_TC_CASE(128, 64, 1)
    B200_TC_CASE(224, 112, 1)
    B200_TC_CASE(352, 176, 2)
#undef B200_TC_CASE
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

}  // namespace b200
