// Near field P2P for the Laplace 1/r kernel over each leaf and its <=26 neighbour leaves.
//
// Pair math (FP2PR::MutualParticles / NonMutualParticles, Src/Kernels/P2P/FP2PR.hpp:14-69):
//   phi_t += q_s / r,   F_t += -q_t q_s (x_t - x_s) / r^3.
// The reference evaluates each unordered pair once (mutual half shell, FChebSymKernel.hpp:468-478);
// the ordered pairs summed here per target are the same set.
//
//  * FP64 (parity form): one CTA per target leaf, source leaves staged through shared memory, the
//    reference's arithmetic sequence (1/r^2, sqrt, products).
//  * FP32 (mixed form), two source particles per step with Blackwell's packed FP32x2 instructions
//    (add/mul/fma.f32x2): positions relative to the box corner as a float pair (hi, lo), so that per pair
//    dx = (t_hi - s_hi) + (t_lo - s_lo) with the first difference exact for nearby particles (Sterbenz),
//    which keeps the close pairs -- the ones that dominate the forces -- accurate to a few ulp.  One warp per
//    target leaf; the neighbour leaves are walked as contiguous runs of records (one per neighbour column)
//    copied into shared memory by the bulk-copy engine (cp.async.bulk + mbarrier, 3-deep ring); rsqrt on the
//    SFU; per-target compensated (two-sum) accumulation of the per-stage partial sums; the result is added
//    in FP64 to the far field.
#include "common.cuh"

#include <mutex>

namespace b200 {

namespace {

constexpr int P2P64_THREADS = 64;

// shard (optional): [first leaf, end leaf) of the targets to evaluate
__global__ void p2p_fp64_kernel(int R, long long N, const long long *__restrict__ leaf_start,
                                const int *__restrict__ nbr, int variant, const double *__restrict__ x,
                                const double *__restrict__ y, const double *__restrict__ z,
                                const double *__restrict__ q, double *__restrict__ phi, double *__restrict__ fx,
                                double *__restrict__ fy, double *__restrict__ fz, const long long *__restrict__ shard) {
  __shared__ double sx[P2P64_THREADS], sy[P2P64_THREADS], sz[P2P64_THREADS], sq[P2P64_THREADS];
  __shared__ long long sidx[P2P64_THREADS];
  const long long leaf = blockIdx.x;
  if (shard && (leaf < shard[0] || leaf >= shard[1])) return;
  const long long t0 = leaf_start[leaf], t1 = leaf_start[leaf + 1];
  for (int r = 0; r < R; ++r) {
    const double *qr = q + (long long)r * N;
    for (long long tb = t0; tb < t1; tb += blockDim.x) {
      const long long i = tb + threadIdx.x;
      const bool active = i < t1;
      const double tx = active ? x[i] : 0, ty = active ? y[i] : 0, tz = active ? z[i] : 0;
      const double tq = active ? qr[i] : 0;
      double pv = 0, gx = 0, gy = 0, gz = 0;
      for (int e = 0; e < 27; ++e) {
        if (variant == 1 && e == 13) continue;
        const int sl = nbr[leaf * 27 + e];
        if (sl < 0) continue;
        const long long s0 = leaf_start[sl], s1 = leaf_start[sl + 1];
        for (long long sb = s0; sb < s1; sb += blockDim.x) {
          __syncthreads();
          const long long j = sb + threadIdx.x;
          if (j < s1) {
            sx[threadIdx.x] = x[j];
            sy[threadIdx.x] = y[j];
            sz[threadIdx.x] = z[j];
            sq[threadIdx.x] = qr[j];
            sidx[threadIdx.x] = j;
          }
          __syncthreads();
          const int cnt = (int)min((long long)blockDim.x, s1 - sb);
          if (active) {
            for (int k = 0; k < cnt; ++k) {
              if (sidx[k] == i) continue;
              double dx = tx - sx[k], dy = ty - sy[k], dz = tz - sz[k];
              double inv2 = 1.0 / (dx * dx + dy * dy + dz * dz);
              const double inv = sqrt(inv2);
              inv2 *= inv;
              inv2 *= tq * sq[k];
              gx += -dx * inv2;
              gy += -dy * inv2;
              gz += -dz * inv2;
              pv += inv * sq[k];
            }
          }
        }
      }
      if (active) {
        const long long j = (long long)r * N + i;
        phi[j] += pv;
        fx[j] += gx;
        fy[j] += gy;
        fz[j] += gz;
      }
    }
  }
}

// ---- FP32 compensated ------------------------------------------------------------------------------
//
// Layout of the FP32 copies (one buffer, d_pq32):
//   tgt_hi[R][N] float4 (x_hi, y_hi, z_hi, q) and tgt_lo[N] float4 (x_lo, y_lo, z_lo, 0): the position of every
//     particle relative to the box corner as a float pair (hi = fl(x - x0), lo = fl(x - x0 - hi)), read by the
//     lane that owns the particle as a target;
//   src[R][N+2][4] float4: the same particles as sources, two per 64-byte record and pre-negated so that
//     packed FP32x2 instructions consume them directly: (-x0,-x1,-y0,-y1) (-z0,-z1,q0,q1) (-lx0,-lx1,-ly0,-ly1)
//     (-lz0,-lz1,0,0).  A leaf with an odd count is padded with a zero-charge particle far away.
// Record order: the leaves in column order (x, y, then z; rank_of[leaf], first record rec_base[rank]), so that
// the up to three z-neighbours of each of the 9 neighbour columns of a target leaf are one contiguous run of
// records.  Without rank_of/rec_base (the allocation-free entry point) the leaves stay in Morton order with
// leaf L's records starting at (leaf_start[L] + L) / 2 (gap records padded); only Morton-adjacent z-neighbours
// then share a run.
//
// Because the coordinates are relative to the box corner (>= 0) and hi carries 24 bits, for close pairs
// t_hi - s_hi is exact (Sterbenz), and dx = (t_hi - s_hi) + (t_lo - s_lo) is accurate to about one ulp of dx:
// the close pairs, which dominate the forces, keep full FP32 relative accuracy.
constexpr double P2P32_PAD = 1.0e15;

__host__ __device__ inline long long p2p_pairs_capacity(long long N) { return N + 2; }

// first source record of the leaf at position rank of the record order
__device__ __forceinline__ long long rec_begin(const long long *__restrict__ rec_base,
                                               const long long *__restrict__ leaf_start, long long rank) {
  return rec_base ? rec_base[rank] : (leaf_start[rank] + rank) >> 1;
}

__global__ void pack_records32(long long N, int R, const long long *__restrict__ leaf_start,
                               const int *__restrict__ rank_of, const long long *__restrict__ rec_base,
                               const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const double *__restrict__ q, double x0, double y0,
                               double z0, float4 *__restrict__ hi, float4 *__restrict__ lo,
                               float4 *__restrict__ src) {
  const long long leaf = blockIdx.x;
  const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1];
  const long long rank = rank_of ? rank_of[leaf] : leaf;
  const long long b0 = rec_begin(rec_base, leaf_start, rank), b1 = rec_begin(rec_base, leaf_start, rank + 1);
  for (long long i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
    const double lx = x[i] - x0, ly = y[i] - y0, lz = z[i] - z0;
    const float hx = (float)lx, hy = (float)ly, hz = (float)lz;
    lo[i] = make_float4((float)(lx - (double)hx), (float)(ly - (double)hy), (float)(lz - (double)hz), 0.f);
    for (int r = 0; r < R; ++r) hi[(long long)r * N + i] = make_float4(hx, hy, hz, (float)q[(long long)r * N + i]);
  }
  const long long P = p2p_pairs_capacity(N);
  for (long long pp = threadIdx.x; pp < b1 - b0; pp += blockDim.x) {
    float h[2][3], l[2][3];
    bool real[2];
    for (int u = 0; u < 2; ++u) {
      const long long j = s0 + 2 * pp + u;
      real[u] = j < s1;
      const double d[3] = {real[u] ? x[j] - x0 : P2P32_PAD, real[u] ? y[j] - y0 : P2P32_PAD,
                           real[u] ? z[j] - z0 : P2P32_PAD};
      for (int a = 0; a < 3; ++a) {
        h[u][a] = (float)d[a];
        l[u][a] = (float)(d[a] - (double)h[u][a]);
      }
    }
    for (int r = 0; r < R; ++r) {
      const long long j0 = s0 + 2 * pp;
      const float q0 = real[0] ? (float)q[(long long)r * N + j0] : 0.f;
      const float q1 = real[1] ? (float)q[(long long)r * N + j0 + 1] : 0.f;
      float4 *rec = src + ((long long)r * P + b0 + pp) * 4;
      rec[0] = make_float4(-h[0][0], -h[1][0], -h[0][1], -h[1][1]);
      rec[1] = make_float4(-h[0][2], -h[1][2], q0, q1);
      rec[2] = make_float4(-l[0][0], -l[1][0], -l[0][1], -l[1][1]);
      rec[3] = make_float4(-l[0][2], -l[1][2], 0.f, 0.f);
    }
  }
}

__device__ __forceinline__ void two_sum(float &hi, float &lo, float v) {
  const float s = hi + v;
  const float bp = s - hi;
  const float err = (hi - (s - bp)) + (v - bp);
  hi = s;
  lo += err;
}

constexpr int P2P32_WARPS = 4;   // target leaves per CTA (one warp each)
constexpr int P2P32_STAGE = 32;  // source records (64 particles) per bulk-copy stage: 24 KB per CTA, 7 CTAs per SM
constexpr int P2P32_NBUF = 3;    // stages in flight per warp

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// Bounded wait on an mbarrier phase; returns false when the iteration budget runs out.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned phase) {
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// The same wait taken by a whole warp: every lane polls, and the warp agrees on the outcome, so that either all
// lanes go on or all give up (a lane that left alone would break the full-mask shuffles that follow).
__device__ __forceinline__ bool mbar_wait_warp(unsigned long long *bar, unsigned phase) {
  return __all_sync(0xffffffffu, mbar_wait(bar, phase));
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// 1/sqrt(x) on the SFU with subnormal inputs flushed to zero (PTX rsqrt.approx.ftz.f32).  rsqrtf, which also
// serves subnormal inputs, made the near field about 8 % slower with bit-identical results on the bench tree;
// r^2 here is subnormal only for particles closer than ~1e-19 box widths, which the flush treats like
// coincident particles.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// One record (two sources) against the lane's target: packed FP32x2 difference, r^2, rsqrt on the SFU.
template <bool SELF>
__device__ __forceinline__ void p2p_record(const float4 *__restrict__ s, int k, int self_rel, float2 th_x,
                                           float2 th_y, float2 th_z, float2 tl_x, float2 tl_y, float2 tl_z,
                                           float2 &pv, float2 &ax, float2 &ay, float2 &az) {
  const float4 A = s[4 * k], B = s[4 * k + 1], C = s[4 * k + 2], D = s[4 * k + 3];
  const float2 dx = __fadd2_rn(__fadd2_rn(th_x, make_float2(A.x, A.y)), __fadd2_rn(tl_x, make_float2(C.x, C.y)));
  const float2 dy = __fadd2_rn(__fadd2_rn(th_y, make_float2(A.z, A.w)), __fadd2_rn(tl_y, make_float2(C.z, C.w)));
  const float2 dz = __fadd2_rn(__fadd2_rn(th_z, make_float2(B.x, B.y)), __fadd2_rn(tl_z, make_float2(D.x, D.y)));
  float2 r2 = __fmul2_rn(dx, dx);
  r2 = __ffma2_rn(dy, dy, r2);
  r2 = __ffma2_rn(dz, dz, r2);
  float2 inv;
  if (SELF) {
    inv = make_float2(2 * k == self_rel ? 0.f : rsqrt_ftz(r2.x), 2 * k + 1 == self_rel ? 0.f : rsqrt_ftz(r2.y));
  } else {
    inv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
  }
  const float2 qi = __fmul2_rn(make_float2(B.z, B.w), inv);
  const float2 qi3 = __fmul2_rn(qi, __fmul2_rn(inv, inv));
  pv = __fadd2_rn(pv, qi);
  ax = __ffma2_rn(dx, qi3, ax);
  ay = __ffma2_rn(dy, qi3, ay);
  az = __ffma2_rn(dz, qi3, az);
}

// One warp per target leaf.  The target particles are taken 32 at a time; a chunk of m <= 16 (or <= 8)
// targets is replicated over 2 (or 4) lane groups, each group walking every 2nd (4th) source record, and the
// groups' sums are combined by shuffles at the end, so that small and ragged leaves keep the lanes busy.
// The sources are walked as runs of contiguous records (one per neighbour column and z-adjacent group),
// each split into stages of <= P2P32_STAGE records copied by one bulk copy into a ring of P2P32_NBUF buffers,
// issued P2P32_NBUF - 1 stages ahead of the math.  Per stage the partial sums enter the target's (hi, lo)
// accumulators by a two-sum.
// With chunk_base, warp (CTA x, warp w) takes the work item blockIdx.x * P2P32_WARPS + w: a leaf of at most
// `whole` targets, or `isize` targets of a larger one (a dense leaf spreads over many warps; items past the count
// leave at once).  Without it (the allocation-free entry point) a warp takes a whole leaf.
__device__ __forceinline__ bool p2p_item(long long item, long long nleaves, const long long *__restrict__ leaf_start,
                                         const long long *__restrict__ chunk_base, int whole, int isize,
                                         long long &leaf, long long &c0, long long &c1) {
  if (!chunk_base) {
    if (item >= nleaves) return false;
    leaf = item;
    c0 = leaf_start[leaf];
    c1 = leaf_start[leaf + 1];
    return true;
  }
  if (item >= chunk_base[nleaves]) return false;
  long long lo = 0, hi = nleaves - 1;  // the last leaf whose first item is <= item
  while (lo < hi) {
    const long long mid = (lo + hi + 1) >> 1;
    if (chunk_base[mid] <= item)
      lo = mid;
    else
      hi = mid - 1;
  }
  leaf = lo;
  const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1];
  if (s1 - s0 <= whole) {
    c0 = s0;
    c1 = s1;
  } else {
    c0 = s0 + (long long)isize * (item - chunk_base[leaf]);
    c1 = min(c0 + isize, s1);
  }
  return true;
}

__global__ void __launch_bounds__(P2P32_WARPS * 32, 7) p2p_fp32_kernel(
    int R, long long N, long long nleaves, const long long *__restrict__ leaf_start, const int *__restrict__ nbr,
    int variant, const int *__restrict__ rank_of, const long long *__restrict__ rec_base,
    const long long *__restrict__ chunk_base, int whole, int isize, const long long *__restrict__ shard,
    const float4 *__restrict__ pq,
    const float4 *__restrict__ plo, const float4 *__restrict__ src, double *__restrict__ phi, double *__restrict__ fx, double *__restrict__ fy,
    double *__restrict__ fz, int *__restrict__ status) {
  __shared__ __align__(128) float4 buf[P2P32_WARPS][P2P32_NBUF][4 * P2P32_STAGE];
  __shared__ __align__(8) unsigned long long bar[P2P32_WARPS][P2P32_NBUF];
  __shared__ long long rbase[P2P32_WARPS][27];
  __shared__ int rcount[P2P32_WARPS][27];
  __shared__ unsigned char rself[P2P32_WARPS][27];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    for (int b = 0; b < P2P32_NBUF; ++b) mbar_init(&bar[w][b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  // the work items of the targets' leaves: all, or the shard's [shard[0], shard[1])
  const long long leaf_lo = shard ? shard[0] : 0, leaf_hi = shard ? shard[1] : nleaves;
  const long long item0 = chunk_base ? chunk_base[leaf_lo] : leaf_lo;
  const long long item1 = chunk_base ? chunk_base[leaf_hi] : leaf_hi;
  const long long item = item0 + (long long)blockIdx.x * P2P32_WARPS + w;
  long long leaf, c0, c1;
  if (item >= item1 || !p2p_item(item, nleaves, leaf_start, chunk_base, whole, isize, leaf, c0, c1)) return;
  const long long P = p2p_pairs_capacity(N);
  const long long t0 = leaf_start[leaf];
  const int my_rank = rank_of ? rank_of[leaf] : (int)leaf;
  const long long self_rec = rec_begin(rec_base, leaf_start, my_rank);
  // the runs of this leaf: lane e < 27 looks at neighbour position e = ((dx+1)*3 + dy+1)*3 + dz+1
  int nr = 0;
  {
    const int e = lane < 27 ? lane : 26;
    int nb = lane < 27 ? nbr[leaf * 27 + e] : -1;
    if (variant == 1 && e == 13) nb = -1;
    const int rk = nb >= 0 ? (rank_of ? rank_of[nb] : nb) : -1;
    const int dz = e % 3;
    const int rk_prev = __shfl_up_sync(0xffffffffu, rk, 1);
    const int rk_next = __shfl_down_sync(0xffffffffu, rk, 1);
    const int rk_next2 = __shfl_down_sync(0xffffffffu, rk, 2);
    const bool start = lane < 27 && rk >= 0 && !(dz > 0 && rk_prev >= 0 && rk_prev + 1 == rk);
    int last = rk;
    if (dz < 2 && rk_next >= 0 && rk_next == last + 1) {
      last = rk_next;
      if (dz == 0 && rk_next2 >= 0 && rk_next2 == last + 1) last = rk_next2;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, start);
    if (start) {
      const int k = __popc(mask & ((1u << lane) - 1u));
      const long long b0 = rec_begin(rec_base, leaf_start, rk), b1 = rec_begin(rec_base, leaf_start, last + 1);
      rbase[w][k] = b0;
      rcount[w][k] = (int)(b1 - b0);
      rself[w][k] = (variant == 0 && e / 3 == 4 && rk <= my_rank && my_rank <= last) ? 1 : 0;
    }
    nr = __popc(mask);
    __syncwarp();
  }
  unsigned phase_bits = 0;  // one parity bit per buffer
  for (int r = 0; r < R; ++r) {
    const float4 *pr = pq + (long long)r * N;
    const float4 *sr = src + (long long)r * P * 4;
    for (long long tb = c0; tb < c1; tb += 32) {
      const int m = (int)min(32LL, c1 - tb);
      const int T = m <= 8 ? 8 : (m <= 16 ? 16 : 32);  // targets per lane group
      const int G = 32 / T;                             // lane groups, each on every G-th record
      const int tl = lane & (T - 1), g = lane / T;
      const long long i = tb + tl;
      const bool active = tl < m;
      const float4 me = active ? pr[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 mel = active ? plo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      const long long self_slot = 2 * self_rec + (i - t0);  // the target's own slot in the record numbering
      const float2 th_x = make_float2(me.x, me.x), th_y = make_float2(me.y, me.y), th_z = make_float2(me.z, me.z);
      const float2 tl_x = make_float2(mel.x, mel.x), tl_y = make_float2(mel.y, mel.y), tl_z = make_float2(mel.z, mel.z);
      float ph_hi = 0.f, ph_lo = 0.f, gx_hi = 0.f, gx_lo = 0.f, gy_hi = 0.f, gy_lo = 0.f, gz_hi = 0.f, gz_lo = 0.f;
      // stage sequence: (run e, first record p, record count n); issue up to NBUF-1 stages ahead
      int ie = 0, ip = 0;  // next stage to issue
      int ce = 0, cp = 0;  // stage being computed
      int issued = 0, done = 0;
      auto next_stage = [&](int &e, int &p0, int &n) -> bool {
        while (e < nr && p0 >= rcount[w][e]) {
          ++e;
          p0 = 0;
        }
        if (e >= nr) return false;
        n = min(P2P32_STAGE, rcount[w][e] - p0);
        return true;
      };
      auto issue = [&]() {
        int n;
        if (!next_stage(ie, ip, n)) return false;
        const int b = issued % P2P32_NBUF;
        if (lane == 0) {
          mbar_expect_tx(&bar[w][b], n * 64);
          bulk_g2s(&buf[w][b][0], sr + (rbase[w][ie] + ip) * 4, n * 64, &bar[w][b]);
        }
        ip += n;
        ++issued;
        return true;
      };
      for (int k = 0; k < P2P32_NBUF - 1; ++k)
        if (!issue()) break;
      while (done < issued) {
        int cn;
        next_stage(ce, cp, cn);
        const int b = done % P2P32_NBUF;
        if (!mbar_wait_warp(&bar[w][b], (phase_bits >> b) & 1u)) {
          // give up: flag it, and let the copies still in flight land (bounded) before the CTA leaves
          if (lane == 0) {
            atomicExch(status, 1);
            for (int k = done; k < issued; ++k) {
              const int bk = k % P2P32_NBUF;
              mbar_wait(&bar[w][bk], (phase_bits >> bk) & 1u);
            }
          }
          __syncwarp();
          return;
        }
        phase_bits ^= 1u << b;
        float2 pv = make_float2(0.f, 0.f), ax = pv, ay = pv, az = pv;
        const float4 *s = buf[w][b];
        if (rself[w][ce]) {
          const int self_rel = (int)(self_slot - 2 * (rbase[w][ce] + cp));  // the target's slot in this stage
#pragma unroll 2
          for (int k = g; k < cn; k += G)
            p2p_record<true>(s, k, self_rel, th_x, th_y, th_z, tl_x, tl_y, tl_z, pv, ax, ay, az);
        } else {
          // two independent accumulator sets, so that consecutive records do not wait on each other's sums
          float2 pv2 = make_float2(0.f, 0.f), ax2 = pv2, ay2 = pv2, az2 = pv2;
          int k = g;
#pragma unroll 2
          for (; k + G < cn; k += 2 * G) {
            p2p_record<false>(s, k, 0, th_x, th_y, th_z, tl_x, tl_y, tl_z, pv, ax, ay, az);
            p2p_record<false>(s, k + G, 0, th_x, th_y, th_z, tl_x, tl_y, tl_z, pv2, ax2, ay2, az2);
          }
          if (k < cn) p2p_record<false>(s, k, 0, th_x, th_y, th_z, tl_x, tl_y, tl_z, pv, ax, ay, az);
          pv = __fadd2_rn(pv, pv2);
          ax = __fadd2_rn(ax, ax2);
          ay = __fadd2_rn(ay, ay2);
          az = __fadd2_rn(az, az2);
        }
        two_sum(ph_hi, ph_lo, pv.x + pv.y);
        two_sum(gx_hi, gx_lo, ax.x + ax.y);
        two_sum(gy_hi, gy_lo, ay.x + ay.y);
        two_sum(gz_hi, gz_lo, az.x + az.y);
        cp += cn;
        ++done;
        __syncwarp();  // every lane is done with buffer b before it is refilled
        issue();
      }
      // combine the lane groups that shared this chunk's targets
      for (int off = T; off < 32; off <<= 1) {
        float oh = __shfl_xor_sync(0xffffffffu, ph_hi, off), ol = __shfl_xor_sync(0xffffffffu, ph_lo, off);
        two_sum(ph_hi, ph_lo, oh);
        ph_lo += ol;
        oh = __shfl_xor_sync(0xffffffffu, gx_hi, off);
        ol = __shfl_xor_sync(0xffffffffu, gx_lo, off);
        two_sum(gx_hi, gx_lo, oh);
        gx_lo += ol;
        oh = __shfl_xor_sync(0xffffffffu, gy_hi, off);
        ol = __shfl_xor_sync(0xffffffffu, gy_lo, off);
        two_sum(gy_hi, gy_lo, oh);
        gy_lo += ol;
        oh = __shfl_xor_sync(0xffffffffu, gz_hi, off);
        ol = __shfl_xor_sync(0xffffffffu, gz_lo, off);
        two_sum(gz_hi, gz_lo, oh);
        gz_lo += ol;
      }
      if (active && g == 0) {
        const long long j = (long long)r * N + i;
        const double tq = -(double)me.w;
        phi[j] += (double)ph_hi + (double)ph_lo;
        fx[j] += tq * ((double)gx_hi + (double)gx_lo);
        fy[j] += tq * ((double)gy_hi + (double)gy_lo);
        fz[j] += tq * ((double)gz_hi + (double)gz_lo);
      }
    }
  }
}

// ---- several right-hand sides ------------------------------------------------------------------------
//
// With nrhs > 1 the charge vectors share the positions, so the geometry of a pair (differences, r^2, rsqrt,
// 1/r^3) is formed once for MR_G right-hand sides at a time, as the reference's multi-RHS near field forms it
// once for all NVALS vectors (FP2P::FullMutualMultiRhs, Src/Kernels/P2P/FP2PMultiRhs.hpp:10-189).  Layout:
//   tgt_hi[N] float4 (x_hi, y_hi, z_hi, 0), tgt_lo[N] float4 (x_lo, y_lo, z_lo, 0), tgt_q[R][N] float;
//   src[G][N+2][5] float4 for each group of MR_G right-hand sides, two sources per 80-byte record:
//     (-x0,-x1,-y0,-y1) (-z0,-z1,-lz0,-lz1) (-lx0,-lx1,-ly0,-ly1) (q0,q1 of rhs 0; q0,q1 of rhs 1) (rhs 2; rhs 3),
//   charges of right-hand sides past R are zero.  Record order and runs are those of the single-RHS kernel.
constexpr int MR_G = 4;
constexpr int MR_REC = 5;  // float4 per record

__global__ void pack_records32_mrhs(long long N, int R, const long long *__restrict__ leaf_start,
                                    const int *__restrict__ rank_of, const long long *__restrict__ rec_base,
                                    const double *__restrict__ x, const double *__restrict__ y,
                                    const double *__restrict__ z, const double *__restrict__ q, double x0, double y0,
                                    double z0, float4 *__restrict__ hi, float4 *__restrict__ lo, float *__restrict__ qt,
                                    float4 *__restrict__ src) {
  const long long leaf = blockIdx.x;
  const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1];
  const long long rank = rank_of ? rank_of[leaf] : leaf;
  const long long b0 = rec_begin(rec_base, leaf_start, rank), b1 = rec_begin(rec_base, leaf_start, rank + 1);
  for (long long i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
    const double lx = x[i] - x0, ly = y[i] - y0, lz = z[i] - z0;
    const float hx = (float)lx, hy = (float)ly, hz = (float)lz;
    hi[i] = make_float4(hx, hy, hz, 0.f);
    lo[i] = make_float4((float)(lx - (double)hx), (float)(ly - (double)hy), (float)(lz - (double)hz), 0.f);
    for (int r = 0; r < R; ++r) qt[(long long)r * N + i] = (float)q[(long long)r * N + i];
  }
  const long long P = p2p_pairs_capacity(N);
  const int G = (R + MR_G - 1) / MR_G;
  for (long long pp = threadIdx.x; pp < b1 - b0; pp += blockDim.x) {
    float h[2][3], l[2][3];
    bool real[2];
    for (int u = 0; u < 2; ++u) {
      const long long j = s0 + 2 * pp + u;
      real[u] = j < s1;
      const double d[3] = {real[u] ? x[j] - x0 : P2P32_PAD, real[u] ? y[j] - y0 : P2P32_PAD,
                           real[u] ? z[j] - z0 : P2P32_PAD};
      for (int a = 0; a < 3; ++a) {
        h[u][a] = (float)d[a];
        l[u][a] = (float)(d[a] - (double)h[u][a]);
      }
    }
    const long long j0 = s0 + 2 * pp;
    auto charge = [&](int r, int u) -> float {
      return (r < R && real[u]) ? (float)q[(long long)r * N + j0 + u] : 0.f;
    };
    for (int g = 0; g < G; ++g) {
      float4 *rec = src + ((long long)g * P + b0 + pp) * MR_REC;
      rec[0] = make_float4(-h[0][0], -h[1][0], -h[0][1], -h[1][1]);
      rec[1] = make_float4(-h[0][2], -h[1][2], -l[0][2], -l[1][2]);
      rec[2] = make_float4(-l[0][0], -l[1][0], -l[0][1], -l[1][1]);
      const int r0 = MR_G * g;
      rec[3] = make_float4(charge(r0, 0), charge(r0, 1), charge(r0 + 1, 0), charge(r0 + 1, 1));
      rec[4] = make_float4(charge(r0 + 2, 0), charge(r0 + 2, 1), charge(r0 + 3, 0), charge(r0 + 3, 1));
    }
  }
}

// One record (two sources) against the lane's target for MR_G right-hand sides: the geometry once, then per
// right-hand side phi += q / r and the force sums q d / r^3.
template <bool SELF>
__device__ __forceinline__ void p2p_record_mrhs(const float4 *__restrict__ s, int k, int self_rel, float2 th_x,
                                                float2 th_y, float2 th_z, float2 tl_x, float2 tl_y, float2 tl_z,
                                                float2 (&pv)[MR_G], float2 (&ax)[MR_G], float2 (&ay)[MR_G],
                                                float2 (&az)[MR_G]) {
  const float4 A = s[MR_REC * k], B = s[MR_REC * k + 1], C = s[MR_REC * k + 2], Q0 = s[MR_REC * k + 3],
               Q1 = s[MR_REC * k + 4];
  const float2 dx = __fadd2_rn(__fadd2_rn(th_x, make_float2(A.x, A.y)), __fadd2_rn(tl_x, make_float2(C.x, C.y)));
  const float2 dy = __fadd2_rn(__fadd2_rn(th_y, make_float2(A.z, A.w)), __fadd2_rn(tl_y, make_float2(C.z, C.w)));
  const float2 dz = __fadd2_rn(__fadd2_rn(th_z, make_float2(B.x, B.y)), __fadd2_rn(tl_z, make_float2(B.z, B.w)));
  float2 r2 = __fmul2_rn(dx, dx);
  r2 = __ffma2_rn(dy, dy, r2);
  r2 = __ffma2_rn(dz, dz, r2);
  float2 inv;
  if (SELF) {
    inv = make_float2(2 * k == self_rel ? 0.f : rsqrt_ftz(r2.x), 2 * k + 1 == self_rel ? 0.f : rsqrt_ftz(r2.y));
  } else {
    inv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
  }
  const float2 inv2 = __fmul2_rn(inv, inv);
  const float2 q[MR_G] = {make_float2(Q0.x, Q0.y), make_float2(Q0.z, Q0.w), make_float2(Q1.x, Q1.y),
                          make_float2(Q1.z, Q1.w)};
#pragma unroll
  for (int g = 0; g < MR_G; ++g) {
    const float2 qi = __fmul2_rn(q[g], inv);
    const float2 qi3 = __fmul2_rn(qi, inv2);
    pv[g] = __fadd2_rn(pv[g], qi);
    ax[g] = __ffma2_rn(dx, qi3, ax[g]);
    ay[g] = __ffma2_rn(dy, qi3, ay[g]);
    az[g] = __ffma2_rn(dz, qi3, az[g]);
  }
}

// The single-RHS kernel's walk (one warp per target leaf, runs of records in bulk-copy stages, lane groups for
// small leaves, per-stage two-sums), with MR_G right-hand sides per pass over the sources.
__global__ void __launch_bounds__(P2P32_WARPS * 32, 4) p2p_fp32_mrhs_kernel(
    int R, long long N, long long nleaves, const long long *__restrict__ leaf_start, const int *__restrict__ nbr,
    int variant, const int *__restrict__ rank_of, const long long *__restrict__ rec_base,
    const long long *__restrict__ chunk_base, int whole, int isize, const long long *__restrict__ shard,
    const float4 *__restrict__ pq, const float4 *__restrict__ plo, const float *__restrict__ qt,
    const float4 *__restrict__ src,
    double *__restrict__ phi, double *__restrict__ fx, double *__restrict__ fy, double *__restrict__ fz,
    int *__restrict__ status) {
  __shared__ __align__(128) float4 buf[P2P32_WARPS][P2P32_NBUF][MR_REC * P2P32_STAGE];
  __shared__ __align__(8) unsigned long long bar[P2P32_WARPS][P2P32_NBUF];
  __shared__ long long rbase[P2P32_WARPS][27];
  __shared__ int rcount[P2P32_WARPS][27];
  __shared__ unsigned char rself[P2P32_WARPS][27];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    for (int b = 0; b < P2P32_NBUF; ++b) mbar_init(&bar[w][b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  // the work items of the targets' leaves: all, or the shard's [shard[0], shard[1])
  const long long leaf_lo = shard ? shard[0] : 0, leaf_hi = shard ? shard[1] : nleaves;
  const long long item0 = chunk_base ? chunk_base[leaf_lo] : leaf_lo;
  const long long item1 = chunk_base ? chunk_base[leaf_hi] : leaf_hi;
  const long long item = item0 + (long long)blockIdx.x * P2P32_WARPS + w;
  long long leaf, c0, c1;
  if (item >= item1 || !p2p_item(item, nleaves, leaf_start, chunk_base, whole, isize, leaf, c0, c1)) return;
  const long long P = p2p_pairs_capacity(N);
  const long long t0 = leaf_start[leaf];
  const int my_rank = rank_of ? rank_of[leaf] : (int)leaf;
  const long long self_rec = rec_begin(rec_base, leaf_start, my_rank);
  int nr = 0;
  {
    const int e = lane < 27 ? lane : 26;
    int nb = lane < 27 ? nbr[leaf * 27 + e] : -1;
    if (variant == 1 && e == 13) nb = -1;
    const int rk = nb >= 0 ? (rank_of ? rank_of[nb] : nb) : -1;
    const int dz = e % 3;
    const int rk_prev = __shfl_up_sync(0xffffffffu, rk, 1);
    const int rk_next = __shfl_down_sync(0xffffffffu, rk, 1);
    const int rk_next2 = __shfl_down_sync(0xffffffffu, rk, 2);
    const bool start = lane < 27 && rk >= 0 && !(dz > 0 && rk_prev >= 0 && rk_prev + 1 == rk);
    int last = rk;
    if (dz < 2 && rk_next >= 0 && rk_next == last + 1) {
      last = rk_next;
      if (dz == 0 && rk_next2 >= 0 && rk_next2 == last + 1) last = rk_next2;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, start);
    if (start) {
      const int k = __popc(mask & ((1u << lane) - 1u));
      const long long b0 = rec_begin(rec_base, leaf_start, rk), b1 = rec_begin(rec_base, leaf_start, last + 1);
      rbase[w][k] = b0;
      rcount[w][k] = (int)(b1 - b0);
      rself[w][k] = (variant == 0 && e / 3 == 4 && rk <= my_rank && my_rank <= last) ? 1 : 0;
    }
    nr = __popc(mask);
    __syncwarp();
  }
  unsigned phase_bits = 0;
  const int G = (R + MR_G - 1) / MR_G;
  for (int grp = 0; grp < G; ++grp) {
    const float4 *sr = src + (long long)grp * P * MR_REC;
    for (long long tb = c0; tb < c1; tb += 32) {
      const int m = (int)min(32LL, c1 - tb);
      const int T = m <= 8 ? 8 : (m <= 16 ? 16 : 32);
      const int Gl = 32 / T;  // lane groups, each on every Gl-th record
      const int tl = lane & (T - 1), g = lane / T;
      const long long i = tb + tl;
      const bool active = tl < m;
      const float4 me = active ? pq[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 mel = active ? plo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      const long long self_slot = 2 * self_rec + (i - t0);
      const float2 th_x = make_float2(me.x, me.x), th_y = make_float2(me.y, me.y), th_z = make_float2(me.z, me.z);
      const float2 tl_x = make_float2(mel.x, mel.x), tl_y = make_float2(mel.y, mel.y), tl_z = make_float2(mel.z, mel.z);
      float ph_hi[MR_G], ph_lo[MR_G], gx_hi[MR_G], gx_lo[MR_G], gy_hi[MR_G], gy_lo[MR_G], gz_hi[MR_G], gz_lo[MR_G];
#pragma unroll
      for (int k = 0; k < MR_G; ++k)
        ph_hi[k] = ph_lo[k] = gx_hi[k] = gx_lo[k] = gy_hi[k] = gy_lo[k] = gz_hi[k] = gz_lo[k] = 0.f;
      int ie = 0, ip = 0, ce = 0, cp = 0, issued = 0, done = 0;
      auto next_stage = [&](int &e, int &p0, int &n) -> bool {
        while (e < nr && p0 >= rcount[w][e]) {
          ++e;
          p0 = 0;
        }
        if (e >= nr) return false;
        n = min(P2P32_STAGE, rcount[w][e] - p0);
        return true;
      };
      auto issue = [&]() {
        int n;
        if (!next_stage(ie, ip, n)) return false;
        const int b = issued % P2P32_NBUF;
        if (lane == 0) {
          mbar_expect_tx(&bar[w][b], n * MR_REC * 16);
          bulk_g2s(&buf[w][b][0], sr + (rbase[w][ie] + ip) * MR_REC, n * MR_REC * 16, &bar[w][b]);
        }
        ip += n;
        ++issued;
        return true;
      };
      for (int k = 0; k < P2P32_NBUF - 1; ++k)
        if (!issue()) break;
      while (done < issued) {
        int cn;
        next_stage(ce, cp, cn);
        const int b = done % P2P32_NBUF;
        if (!mbar_wait_warp(&bar[w][b], (phase_bits >> b) & 1u)) {
          if (lane == 0) {
            atomicExch(status, 1);
            for (int k = done; k < issued; ++k) {
              const int bk = k % P2P32_NBUF;
              mbar_wait(&bar[w][bk], (phase_bits >> bk) & 1u);
            }
          }
          __syncwarp();
          return;
        }
        phase_bits ^= 1u << b;
        float2 pv[MR_G], ax[MR_G], ay[MR_G], az[MR_G];
#pragma unroll
        for (int k = 0; k < MR_G; ++k) pv[k] = ax[k] = ay[k] = az[k] = make_float2(0.f, 0.f);
        const float4 *s = buf[w][b];
        if (rself[w][ce]) {
          const int self_rel = (int)(self_slot - 2 * (rbase[w][ce] + cp));
          for (int k = g; k < cn; k += Gl)
            p2p_record_mrhs<true>(s, k, self_rel, th_x, th_y, th_z, tl_x, tl_y, tl_z, pv, ax, ay, az);
        } else {
#pragma unroll 2
          for (int k = g; k < cn; k += Gl)
            p2p_record_mrhs<false>(s, k, 0, th_x, th_y, th_z, tl_x, tl_y, tl_z, pv, ax, ay, az);
        }
#pragma unroll
        for (int k = 0; k < MR_G; ++k) {
          two_sum(ph_hi[k], ph_lo[k], pv[k].x + pv[k].y);
          two_sum(gx_hi[k], gx_lo[k], ax[k].x + ax[k].y);
          two_sum(gy_hi[k], gy_lo[k], ay[k].x + ay[k].y);
          two_sum(gz_hi[k], gz_lo[k], az[k].x + az[k].y);
        }
        cp += cn;
        ++done;
        __syncwarp();
        issue();
      }
#pragma unroll
      for (int k = 0; k < MR_G; ++k) {
        for (int off = T; off < 32; off <<= 1) {
          float oh = __shfl_xor_sync(0xffffffffu, ph_hi[k], off), ol = __shfl_xor_sync(0xffffffffu, ph_lo[k], off);
          two_sum(ph_hi[k], ph_lo[k], oh);
          ph_lo[k] += ol;
          oh = __shfl_xor_sync(0xffffffffu, gx_hi[k], off);
          ol = __shfl_xor_sync(0xffffffffu, gx_lo[k], off);
          two_sum(gx_hi[k], gx_lo[k], oh);
          gx_lo[k] += ol;
          oh = __shfl_xor_sync(0xffffffffu, gy_hi[k], off);
          ol = __shfl_xor_sync(0xffffffffu, gy_lo[k], off);
          two_sum(gy_hi[k], gy_lo[k], oh);
          gy_lo[k] += ol;
          oh = __shfl_xor_sync(0xffffffffu, gz_hi[k], off);
          ol = __shfl_xor_sync(0xffffffffu, gz_lo[k], off);
          two_sum(gz_hi[k], gz_lo[k], oh);
          gz_lo[k] += ol;
        }
        const int r = MR_G * grp + k;
        if (active && g == 0 && r < R) {
          const long long j = (long long)r * N + i;
          const double tq = -(double)qt[j];
          phi[j] += (double)ph_hi[k] + (double)ph_lo[k];
          fx[j] += tq * ((double)gx_hi[k] + (double)gx_lo[k]);
          fy[j] += tq * ((double)gy_hi[k] + (double)gy_lo[k]);
          fz[j] += tq * ((double)gz_hi[k] + (double)gz_lo[k]);
        }
      }
    }
  }
}

}  // namespace

b200fmm_status run_p2p(Context &c, int variant, const long long *shard) {
  const int LL = c.H - 1;
  const Level &L = c.lv[LL];
  if (L.n == 0) return B200FMM_OK;
  if (c.cfg.precision == B200FMM_MIXED && c.R > 1) {
    // several right-hand sides: targets hi [N], lo [N], charges [R][N] (floats), then the record groups; the
    // buffer sized for the single-RHS layout of R vectors holds this one
    float4 *hi = c.d_pq32, *lo = c.d_pq32 + c.N;
    float *qt = (float *)(c.d_pq32 + 2 * c.N);
    float4 *src = c.d_pq32 + 2 * c.N + (c.N * c.R + 3) / 4;
    if (!c.packed32) {
      c.packed32 = true;
      if (c.column_serial != c.tree_serial) {
        B200_CHECK(leaf_column_order(c));
        c.column_serial = c.tree_serial;
      }
      const double W = c.cfg.box_width;
      pack_records32_mrhs<<<(unsigned)L.n, 64, 0, c.stream>>>(
          c.N, c.R, c.d_leaf_start, c.d_leaf_rank, c.d_rec_base, c.d_x, c.d_y, c.d_z, c.d_q, c.cfg.center[0] - W / 2,
          c.cfg.center[1] - W / 2, c.cfg.center[2] - W / 2, hi, lo, qt, src);
      ++c.launches;
    }
    // work items (p2p_leaf_items per leaf): nleaves + N / item bounds their count
    const unsigned blocks = grid_for(L.n + c.N / c.p2p_item, P2P32_WARPS);
    B200_CUDA(record_event(c, 10));
    p2p_fp32_mrhs_kernel<<<blocks, P2P32_WARPS * 32, 0, c.stream>>>(
        c.R, c.N, L.n, c.d_leaf_start, c.d_leaf_nbr, variant, c.d_leaf_rank, c.d_rec_base, c.d_chunk_base, c.p2p_whole,
        c.p2p_item, shard, hi, lo, qt, src, c.d_phi, c.d_fx, c.d_fy, c.d_fz, c.d_status);
    B200_CUDA(record_event(c, 11));
    ++c.launches;
  } else if (c.cfg.precision == B200FMM_MIXED) {
    float4 *hi = c.d_pq32, *lo = c.d_pq32 + c.N * c.R, *src = c.d_pq32 + c.N * (c.R + 1);
    if (!c.packed32) {
      c.packed32 = true;
      if (c.column_serial != c.tree_serial) {
        B200_CHECK(leaf_column_order(c));
        c.column_serial = c.tree_serial;
      }
      const double W = c.cfg.box_width;
      pack_records32<<<(unsigned)L.n, 64, 0, c.stream>>>(c.N, c.R, c.d_leaf_start, c.d_leaf_rank, c.d_rec_base, c.d_x,
                                                         c.d_y, c.d_z, c.d_q, c.cfg.center[0] - W / 2,
                                                         c.cfg.center[1] - W / 2, c.cfg.center[2] - W / 2, hi, lo, src);
      ++c.launches;
    }
    int *status = c.d_status;
    // work items (p2p_leaf_items per leaf): nleaves + N / item bounds their count
    const unsigned blocks = grid_for(L.n + c.N / c.p2p_item, P2P32_WARPS);
    B200_CUDA(record_event(c, 10));
    p2p_fp32_kernel<<<blocks, P2P32_WARPS * 32, 0, c.stream>>>(
        c.R, c.N, L.n, c.d_leaf_start, c.d_leaf_nbr, variant, c.d_leaf_rank, c.d_rec_base, c.d_chunk_base, c.p2p_whole,
        c.p2p_item, shard, hi, lo, src, c.d_phi, c.d_fx, c.d_fy, c.d_fz, status);
    B200_CUDA(record_event(c, 11));
    ++c.launches;
  } else {
    B200_CUDA(record_event(c, 10));
    p2p_fp64_kernel<<<(unsigned)L.n, P2P64_THREADS, 0, c.stream>>>(c.R, c.N, c.d_leaf_start, c.d_leaf_nbr, variant,
                                                                   c.d_x, c.d_y, c.d_z, c.d_q, c.d_phi, c.d_fx,
                                                                   c.d_fy, c.d_fz, shard);
    B200_CUDA(record_event(c, 11));
    ++c.launches;
  }
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

}  // namespace b200

// ---- allocation-free entry point -------------------------------------------------------------------
// Scratch of b200fmm_p2p_noalloc: the FP32 copies of the particles -- targets (hi, lo) and
// pair-packed sources, 6 float4 per particle plus 8 (24 MiB at 2^18 particles) -- and the status words:
// [0] a bounded wait of the near-field kernel ran out, [1] the caller's leaf tables failed the checks.  In host
// code these names are host-side stand-ins, not device addresses: the host passes the addresses looked up with
// cudaGetSymbolAddress.
static __device__ __align__(256) float4 g_noalloc_stage[6 * B200FMM_NOALLOC_MAX_PARTICLES + 8];
static __device__ __align__(256) int g_noalloc_status[4];

namespace b200 {
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float4 *g_noalloc_stage_ptr[kMaxDevices] = {};
int *g_noalloc_status_ptr[kMaxDevices] = {};

// Once per device, with that device current: the device addresses of the file-scope arrays.
b200fmm_status noalloc_addresses(float4 **stage, int **status) {
  int dev = -1;
  B200_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(B200FMM_ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_stage_ptr[dev]) {
    void *a = nullptr, *b = nullptr;
    B200_CUDA(cudaGetSymbolAddress(&a, g_noalloc_stage));
    B200_CUDA(cudaGetSymbolAddress(&b, g_noalloc_status));
    g_noalloc_stage_ptr[dev] = (float4 *)a;
    g_noalloc_status_ptr[dev] = (int *)b;
  }
  *stage = g_noalloc_stage_ptr[dev];
  *status = g_noalloc_status_ptr[dev];
  return B200FMM_OK;
}

// The caller's leaf tables are checked before any kernel indexes memory through them: leaf_start rises from 0
// to n, the leaf keys rise strictly inside the leaf level, every neighbour entry is -1 or a leaf index, and
// position 13 names the leaf itself.  With these, every particle index the packing and near-field kernels form
// lies in [0, n) and every source record in [0, n + 2), inside the scratch array.  A failure sets status[1].
__global__ void noalloc_check_tables(long long n, long long nleaves, const long long *__restrict__ leaf_keys,
                                     const long long *__restrict__ leaf_start, const int *__restrict__ nbr,
                                     long long key_end, int *__restrict__ status) {
  bool bad = false;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nleaves * 27; i += stride) {
    const int v = nbr[i];
    const long long leaf = i / 27;
    bad |= v < -1 || v >= nleaves || (i % 27 == 13 && v != leaf);
    if (i % 27 == 0) {
      const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1], k = leaf_keys[leaf];
      bad |= s0 < 0 || s1 < s0 || s1 > n || k < 0 || k >= key_end;
      bad |= leaf == 0 && s0 != 0;
      bad |= leaf == nleaves - 1 && s1 != n;
      bad |= leaf > 0 && leaf_keys[leaf - 1] >= k;
    }
  }
  if (bad) atomicExch(status + 1, 1);
}
}  // namespace
}  // namespace b200

extern "C" b200fmm_status b200fmm_p2p_noalloc(long long n, const double *x, const double *y, const double *z,
                                              const double *q, long long nleaves, const long long *leaf_keys,
                                              const long long *leaf_start, const int *leaf_nbr, int height,
                                              double box_width, const double *center, int variant, double *phi,
                                              double *fx, double *fy, double *fz, void *stream) {
  using namespace b200;
  if (n < 1 || nleaves < 1 || nleaves > n) return fail(B200FMM_ERR_INVALID, "p2p_noalloc: bad particle/leaf count");
  if (n > B200FMM_NOALLOC_MAX_PARTICLES)
    return fail(B200FMM_ERR_INVALID, "p2p_noalloc: more than B200FMM_NOALLOC_MAX_PARTICLES (262144) particles");
  if (!x || !y || !z || !q || !leaf_keys || !leaf_start || !leaf_nbr || !center || !phi || !fx || !fy || !fz)
    return fail(B200FMM_ERR_INVALID, "p2p_noalloc: null pointer");
  if (height < 2 || height > kMaxHeight) return fail(B200FMM_ERR_INVALID, "p2p_noalloc: height out of range");
  if (variant != 0 && variant != 1) return fail(B200FMM_ERR_INVALID, "p2p_noalloc: variant must be 0 or 1");
  if (!(box_width > 0)) return fail(B200FMM_ERR_INVALID, "p2p_noalloc: bad box width");
  float4 *stage = nullptr;
  int *status = nullptr;
  B200_CHECK(noalloc_addresses(&stage, &status));
  cudaStream_t s = (cudaStream_t)stream;
  int st[2] = {0, 0};
  // 1) the tables, read back before anything indexes through them
  B200_CUDA(cudaMemsetAsync(status, 0, sizeof(int) * 4, s));
  const long long key_end = 1LL << (3 * (height - 1));
  noalloc_check_tables<<<grid_for(nleaves * 27, 256) < 1184 ? grid_for(nleaves * 27, 256) : 1184, 256, 0, s>>>(
      n, nleaves, leaf_keys, leaf_start, leaf_nbr, key_end, status);
  B200_CUDA(cudaGetLastError());
  B200_CUDA(cudaMemcpyAsync(st, status, sizeof(st), cudaMemcpyDeviceToHost, s));
  B200_CUDA(cudaStreamSynchronize(s));
  if (st[1])
    return fail(B200FMM_ERR_INVALID,
                "p2p_noalloc: inconsistent leaf tables (leaf_start must rise from 0 to n, leaf keys rise strictly "
                "inside the leaf level, neighbour entries be -1 or a leaf index with position 13 the leaf itself)");
  // 2) the FP32 copies and the near field
  pack_records32<<<(unsigned)nleaves, 64, 0, s>>>(n, 1, leaf_start, nullptr, nullptr, x, y, z, q,
                                                 center[0] - box_width / 2, center[1] - box_width / 2,
                                                 center[2] - box_width / 2, stage, stage + n, stage + 2 * n);
  p2p_fp32_kernel<<<grid_for(nleaves, P2P32_WARPS), P2P32_WARPS * 32, 0, s>>>(
      1, n, nleaves, leaf_start, leaf_nbr, variant, nullptr, nullptr, nullptr, 0, 0, nullptr, stage, stage + n,
      stage + 2 * n, phi, fx, fy, fz, status);
  B200_CUDA(cudaGetLastError());
  B200_CUDA(cudaMemcpyAsync(st, status, sizeof(st), cudaMemcpyDeviceToHost, s));
  B200_CUDA(cudaStreamSynchronize(s));
  if (st[0]) return fail(B200FMM_ERR_CUDA, "p2p_noalloc: a device wait ran out of its iteration budget");
  return B200FMM_OK;
}
