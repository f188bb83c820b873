// FP64 M2L (parity form).
//
//  * CHEB_SYM: FChebSymKernel::M2L (Src/Kernels/Chebyshev/FChebSymKernel.hpp:210-328).  For each target the
//    reference permutes every source multipole into its symmetry class frame (pvectors, pindices), applies the
//    16 compressed operators as Y = V^T M' then scale * U Y per class, and adds the result back through the
//    same permutation.  Here the permutation is folded into per-slot factors U_t, V_t once (precompute.cu),
//    and one CTA applies them for 32 targets of one child type -- which share their 189 slots -- keeping the
//    local sums in registers.
//  * CHEB_DENSE / LAGRANGE: L[m] += scale * sum_n K_t(X_m, Y_n) M[n] (FChebDenseKernel::M2L,
//    FChebDenseKernel.hpp:116-127; FUnifKernel applies the same Toeplitz operator through FFTs).
//  scale = 2 / cell width (FInterpMatrixKernelR::getScaleFactor, FInterpMatrixKernel.hpp:124-133).
#include "common.cuh"

#include <cstdlib>

namespace b200 {

namespace {

constexpr int SYM_THREADS = 512;

struct SymArgs {
  int R, rhs;
  double scale;
  long long nparents;
  const int *child;        // parents' [8] children at the target level
  const int *ilist;        // [ntargets][189]
  const IListTable *itab;
  const double *Ut, *Vt;   // per-slot permuted factors, both [p^3][r]
  const long long *toff;   // [343]
  const int *trank;        // [343]
  const double *M;         // source multipoles at this level
  double *L;               // target locals at this level
  int max_rank;
};

constexpr int SYM_T = 16;  // targets per CTA (children of one type of SYM_T consecutive parents)

// Copies into shared memory with every load of a thread issued before its stores, so that the loads of one
// staging step are in flight together instead of one L2 round trip after another.
constexpr int STAGE_UNROLL = 16;

__device__ __forceinline__ void stage_block(double *dst, const double *__restrict__ src, int count) {
  for (int base = 0; base < count; base += STAGE_UNROLL * SYM_THREADS) {
    double v[STAGE_UNROLL];
#pragma unroll
    for (int u = 0; u < STAGE_UNROLL; ++u) {
      const int idx = base + u * SYM_THREADS + threadIdx.x;
      v[u] = idx < count ? __ldg(src + idx) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < STAGE_UNROLL; ++u) {
      const int idx = base + u * SYM_THREADS + threadIdx.x;
      if (idx < count) dst[idx] = v[u];
    }
  }
}

// Ms[k][m] = M[src[k]][rhs][m] (0 for a missing source)
template <int nn, int T>
__device__ __forceinline__ void stage_rows(double *Ms, const double *__restrict__ M, const int *src, int R, int rhs) {
  constexpr int count = T * nn;
  for (int base = 0; base < count; base += STAGE_UNROLL * SYM_THREADS) {
    double v[STAGE_UNROLL];
#pragma unroll
    for (int u = 0; u < STAGE_UNROLL; ++u) {
      const int idx = base + u * SYM_THREADS + threadIdx.x;
      v[u] = 0.0;
      if (idx < count) {
        const int k = idx / nn, m = idx - k * nn;
        const int sc = src[k];
        if (sc >= 0) v[u] = __ldg(M + ((long long)sc * R + rhs) * nn + m);
      }
    }
#pragma unroll
    for (int u = 0; u < STAGE_UNROLL; ++u) {
      const int idx = base + u * SYM_THREADS + threadIdx.x;
      if (idx < count) Ms[idx] = v[u];
    }
  }
}

// One CTA: the SYM_T targets of child type blockIdx.y among SYM_T consecutive parents.  For each of the 189
// transfer vectors of that child type: gather the source multipoles, stage V_t in shared memory (coalesced)
// and form Y = V_t^T M (rank r); stage U_t in the same buffer and add U_t Y to the targets' local sums, which
// stay in registers across all transfer vectors.
template <int P>
__global__ void __launch_bounds__(SYM_THREADS) m2l_sym_kernel(SymArgs a) {
  constexpr int nn = P * P * P, T = SYM_T;
  constexpr int nout = T * nn;
  constexpr int NACC = (nout + SYM_THREADS - 1) / SYM_THREADS;
  extern __shared__ double sh[];
  double *Ms = sh;                        // [T][nn] gathered source multipoles
  double *Y = Ms + T * nn;                // [T][max_rank]
  double *Op = Y + T * a.max_rank;        // [nn][r] V_t, then U_t
  __shared__ int tgt[T], src[T];
  __shared__ int any;
  const int ct = blockIdx.y;
  const long long p0 = (long long)blockIdx.x * T;
  if (threadIdx.x < T) {
    const long long p = p0 + threadIdx.x;
    tgt[threadIdx.x] = p < a.nparents ? a.child[p * 8 + ct] : -1;
  }
  double acc[NACC];
#pragma unroll
  for (int j = 0; j < NACC; ++j) acc[j] = 0.0;
  for (int e = 0; e < 189; ++e) {
    __syncthreads();
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    if (threadIdx.x < T) {
      const int tg = tgt[threadIdx.x];
      const int sc = tg >= 0 ? a.ilist[(long long)tg * 189 + e] : -1;
      src[threadIdx.x] = sc;
      if (sc >= 0) any = 1;
    }
    __syncthreads();
    if (!any) continue;
    const int t = a.itab->slot[ct][e];
    const int r = a.trank[t];
    const double *Ut = a.Ut + a.toff[t];
    const double *Vt = a.Vt + a.toff[t];
    stage_rows<nn, T>(Ms, a.M, src, a.R, a.rhs);
    stage_block(Op, Vt, nn * r);
    __syncthreads();
    for (int idx = threadIdx.x; idx < T * r; idx += blockDim.x) {
      const int k = idx / r, q = idx - k * r;
      const double *mk = Ms + k * nn;
      double s0 = 0.0, s1 = 0.0;
      int m = 0;
      for (; m + 1 < nn; m += 2) {
        s0 += Op[m * r + q] * mk[m];
        s1 += Op[(m + 1) * r + q] * mk[m + 1];
      }
      if (m < nn) s0 += Op[m * r + q] * mk[m];
      Y[k * a.max_rank + q] = s0 + s1;
    }
    __syncthreads();
    stage_block(Op, Ut, nn * r);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NACC; ++j) {
      const int o = threadIdx.x + j * SYM_THREADS;
      if (o < nout) {
        const int k = o / nn, n = o - k * nn;
        if (src[k] >= 0) {
          const double *u = Op + n * r;
          const double *y = Y + k * a.max_rank;
          double s0 = 0.0, s1 = 0.0;
          int q = 0;
          for (; q + 1 < r; q += 2) {
            s0 += u[q] * y[q];
            s1 += u[q + 1] * y[q + 1];
          }
          if (q < r) s0 += u[q] * y[q];
          acc[j] += s0 + s1;
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NACC; ++j) {
    const int o = threadIdx.x + j * SYM_THREADS;
    if (o < nout) {
      const int k = o / nn, n = o - k * nn;
      if (tgt[k] >= 0) a.L[((long long)tgt[k] * a.R + a.rhs) * nn + n] += a.scale * acc[j];
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
    // the two-GEMM form (m2l_sym64.cu); the per-target kernel below remains for trees whose largest level
    // would need more than the two-GEMM form's cap on Y, and on request (B200FMM_SYM64=0)
    const char *env = std::getenv("B200FMM_SYM64");
    if (c.s64 && !(env && env[0] == '0')) {
      const b200fmm_status st = run_m2l_sym64(c, level);
      if (st != B200FMM_ERR_UNSUPPORTED) return st;
    }
    SymArgs a;
    a.R = c.R;
    a.scale = scale;
    a.nparents = c.lv[level - 1].n;
    a.child = c.lv[level - 1].child;
    a.ilist = T.ilist;
    a.itab = c.d_itab;
    a.Ut = c.d_Ut;
    a.Vt = c.d_Vt;
    a.toff = c.d_toff;
    a.trank = c.d_trank;
    a.M = T.M;
    a.L = T.L;
    a.max_rank = c.max_rank;
    const int T = SYM_T;
    const size_t sh = sizeof(double) * ((size_t)T * c.nn + (size_t)T * c.max_rank + (size_t)c.nn * c.max_rank);
    if (sh > 227 * 1024) return fail(B200FMM_ERR_UNSUPPORTED, "compressed operators too large for the FP64 M2L kernel");
    const dim3 grid((unsigned)((a.nparents + T - 1) / T), 8);
    for (int r = 0; r < c.R; ++r) {
      a.rhs = r;
      switch (c.p) {
#define B200_SYM(PV)                                                                                        \
  case PV:                                                                                                  \
    B200_CUDA(cudaFuncSetAttribute(m2l_sym_kernel<PV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh)); \
    m2l_sym_kernel<PV><<<grid, SYM_THREADS, sh, c.stream>>>(a);                                             \
    break;
        B200_SYM(3) B200_SYM(4) B200_SYM(5) B200_SYM(6) B200_SYM(7) B200_SYM(8)
#undef B200_SYM
        default:
          return fail(B200FMM_ERR_UNSUPPORTED, "order not built");
      }
      ++c.launches;
    }
  } else {
    m2l_dense_kernel<<<(unsigned)T.n, 128, sizeof(double) * c.nn, c.stream>>>(
        c.p, c.R, scale, T.keys, T.ilist, c.d_itab, c.d_dense, T.M, T.L);
    ++c.launches;
  }
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

}  // namespace b200
