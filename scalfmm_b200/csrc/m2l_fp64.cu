// FP64 M2L (parity form).
//
//  * CHEB_SYM: FChebSymKernel::M2L (Src/Kernels/Chebyshev/FChebSymKernel.hpp:210-328).  For each target the
//    reference permutes every source multipole into its symmetry class frame (pvectors, pindices), applies the
//    16 compressed operators as Y = V^T M' then scale * U Y per class, and adds the result back through the
//    same permutation.  Here one CTA handles the (up to) 8 children of one parent, so each class operator is
//    read once for 8 targets; pairs are processed class by class in chunks.
//  * CHEB_DENSE / LAGRANGE: L[m] += scale * sum_n K_t(X_m, Y_n) M[n] (FChebDenseKernel::M2L,
//    FChebDenseKernel.hpp:116-127; FUnifKernel applies the same Toeplitz operator through FFTs).
//  scale = 2 / cell width (FInterpMatrixKernelR::getScaleFactor, FInterpMatrixKernel.hpp:124-133).
#include "common.cuh"

namespace b200 {

namespace {

constexpr int SYM_CHUNK = 16;
constexpr int SYM_THREADS = 256;

struct SymArgs {
  int p, nn, R;
  double scale;
  const int *child;        // parents' [8] children at the target level
  const long long *keys;   // target keys (child type = key & 7)
  const int *ilist;        // [ntargets][189]
  const int *class_order;  // [8][189]
  const int *cls_bounds;   // [8][17]
  const int *cls_slot;     // [16] class slot ids
  const int *pvec;         // [343][nn]
  const int *pind;         // [343]
  const double *U, *V;     // per class [r][nn]
  const long long *off;    // [343]
  const int *rank;         // [343]
  const IListTable *itab;
  const double *M;         // source multipoles at this level
  double *L;               // target locals at this level
  int max_rank;
};

__global__ void __launch_bounds__(SYM_THREADS) m2l_sym_kernel(SymArgs a) {
  extern __shared__ double sh[];
  const int nn = a.nn;
  double *Lacc = sh;                          // [8][nn]
  double *Mb = Lacc + 8 * nn;                 // [SYM_CHUNK][nn]
  double *Y = Mb + SYM_CHUNK * nn;            // [SYM_CHUNK][max_rank]
  int *pchild = (int *)(Y + SYM_CHUNK * a.max_rank);  // [SYM_CHUNK]
  int *psrc = pchild + SYM_CHUNK;
  int *pslot = psrc + SYM_CHUNK;
  __shared__ int tgt[8];
  const long long parent = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if (threadIdx.x < 8) tgt[threadIdx.x] = a.child[parent * 8 + threadIdx.x];
  for (int r = 0; r < a.R; ++r) {
    __syncthreads();
    for (int e = threadIdx.x; e < 8 * nn; e += blockDim.x) Lacc[e] = 0.0;
    for (int ci = 0; ci < 16; ++ci) {
      const int cls = a.cls_slot[ci];
      const int rk = a.rank[cls];
      const double *U = a.U + a.off[cls];
      const double *V = a.V + a.off[cls];
      // walk the class-ci entries of the 8 children as one sequence, chunk by chunk
      int k = 0, pos = 0;  // child, position within its class run
      while (true) {
        __syncthreads();
        // the next SYM_CHUNK existing pairs (thread 0 builds the chunk list)
        if (threadIdx.x == 0) {
          int cnt = 0;
          while (k < 8 && cnt < SYM_CHUNK) {
            const int tc = tgt[k];
            if (tc < 0) {
              ++k;
              pos = 0;
              continue;
            }
            const int b0 = a.cls_bounds[k * 17 + ci], b1 = a.cls_bounds[k * 17 + ci + 1];
            if (b0 + pos >= b1) {
              ++k;
              pos = 0;
              continue;
            }
            const int e = a.class_order[k * 189 + b0 + pos];
            ++pos;
            const int src = a.ilist[(long long)tc * 189 + e];
            if (src < 0) continue;
            pchild[cnt] = k;
            psrc[cnt] = src;
            pslot[cnt] = a.itab->slot[k][e];
            ++cnt;
          }
          for (int j = cnt; j < SYM_CHUNK; ++j) pchild[j] = -1;
        }
        __syncthreads();
        if (pchild[0] < 0) break;
        // gather the permuted source multipoles: Mb[j][pvec[t][m]] = M[src][m]
        for (int e = threadIdx.x; e < SYM_CHUNK * nn; e += blockDim.x) {
          const int j = e / nn, m = e % nn;
          if (pchild[j] < 0) continue;
          Mb[j * nn + a.pvec[pslot[j] * nn + m]] = a.M[((long long)psrc[j] * a.R + r) * nn + m];
        }
        __syncthreads();
        // Y[j][q] = sum_m V[q][m] Mb[j][m]   (one warp per dot product)
        for (int d = warp; d < SYM_CHUNK * rk; d += nwarps) {
          const int j = d / rk, q = d % rk;
          double s = 0.0;
          if (pchild[j] >= 0)
            for (int m = lane; m < nn; m += 32) s += V[(long long)q * nn + m] * Mb[j * nn + m];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
          if (lane == 0) Y[j * a.max_rank + q] = s;
        }
        __syncthreads();
        // Lacc[child][n] += scale * sum_q U[q][pvec[t][n]] Y[j][q]  (each thread owns outputs; deterministic)
        for (int e = threadIdx.x; e < 8 * nn; e += blockDim.x) {
          const int kk = e / nn, n = e % nn;
          double acc = 0.0;
          for (int j = 0; j < SYM_CHUNK; ++j) {
            if (pchild[j] != kk) continue;
            const int idx = a.pvec[pslot[j] * nn + n];
            double s = 0.0;
            for (int q = 0; q < rk; ++q) s += U[(long long)q * nn + idx] * Y[j * a.max_rank + q];
            acc += s;
          }
          Lacc[e] += a.scale * acc;
        }
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 8 * nn; e += blockDim.x) {
      const int kk = e / nn, n = e % nn;
      if (tgt[kk] >= 0) a.L[((long long)tgt[kk] * a.R + r) * nn + n] += Lacc[e];
    }
  }
}

__global__ void m2l_dense_kernel(int p, int R, double scale, const long long *__restrict__ keys,
                                 const int *__restrict__ ilist, const IListTable *__restrict__ itab,
                                 const double *__restrict__ K, const double *__restrict__ M, double *__restrict__ L) {
  extern __shared__ double sM[];
  const int nn = p * p * p;
  const long long c = blockIdx.x;
  const int ct = (int)(keys[c] & 7);
  for (int r = 0; r < R; ++r) {
    double acc[4] = {0, 0, 0, 0};
    for (int e = 0; e < 189; ++e) {
      const int src = ilist[c * 189 + e];
      if (src < 0) continue;
      const int t = itab->slot[ct][e];
      __syncthreads();
      for (int i = threadIdx.x; i < nn; i += blockDim.x) sM[i] = M[((long long)src * R + r) * nn + i];
      __syncthreads();
      const double *Kt = K + (long long)t * nn * nn;
      for (int k = 0; k < 4; ++k) {
        const int m = threadIdx.x + k * blockDim.x;
        if (m >= nn) break;
        double s = 0.0;
        for (int n = 0; n < nn; ++n) s += Kt[(long long)n * nn + m] * sM[n];
        acc[k] += s;
      }
    }
    for (int k = 0; k < 4; ++k) {
      const int m = threadIdx.x + k * blockDim.x;
      if (m < nn) L[(c * R + r) * nn + m] += scale * acc[k];
    }
  }
}

}  // namespace

b200fmm_status run_m2l_fp64(Context &c, int level) {
  if (level < 2 || level > c.H - 1) return fail(B200FMM_ERR_INVALID, "m2l: level must be in [2, height-1]");
  const Level &T = c.lv[level];
  if (T.n == 0) return B200FMM_OK;
  const double scale = 2.0 / (c.cfg.box_width / (double)(1LL << level));
  if (c.cfg.kernel == B200FMM_CHEB_SYM && c.cfg.precision == B200FMM_FP64) {
    SymArgs a;
    a.p = c.p;
    a.nn = c.nn;
    a.R = c.R;
    a.scale = scale;
    a.child = c.lv[level - 1].child;
    a.keys = T.keys;
    a.ilist = T.ilist;
    a.class_order = c.d_class_order;
    a.cls_bounds = c.d_cls_bounds;
    a.cls_slot = c.d_cls_slots;
    a.pvec = c.d_pvec;
    a.pind = c.d_pindices;
    a.U = c.d_symU;
    a.V = c.d_symV;
    a.off = c.d_symoff;
    a.rank = c.d_symrank;
    a.itab = c.d_itab;
    a.M = T.M;
    a.L = T.L;
    a.max_rank = c.max_rank;
    const size_t sh = sizeof(double) * (8 * c.nn + SYM_CHUNK * c.nn + SYM_CHUNK * c.max_rank) + sizeof(int) * 3 * SYM_CHUNK;
    B200_CUDA(cudaFuncSetAttribute(m2l_sym_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
    m2l_sym_kernel<<<(unsigned)c.lv[level - 1].n, SYM_THREADS, sh, c.stream>>>(a);
    ++c.launches;
  } else {
    m2l_dense_kernel<<<(unsigned)T.n, 128, sizeof(double) * c.nn, c.stream>>>(
        c.p, c.R, scale, T.keys, T.ilist, c.d_itab, c.d_dense, T.M, T.L);
    ++c.launches;
  }
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

}  // namespace b200
