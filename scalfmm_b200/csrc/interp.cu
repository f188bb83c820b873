// P2M / M2M / L2L / L2P in FP64 for the Chebyshev and Lagrange bases.
//
//  P2M  M[n] += sum_particles q * prod_d S_{n_d}(x_d)      (FChebInterpolator::applyP2M,
//                                                            Src/Kernels/Chebyshev/FChebInterpolator.hpp:627-762)
//  M2M  parent[n] += sum_m prod_d S[c][d][n_d][m_d] child[m] (applyM2M, FChebInterpolator.hpp:560-584)
//  L2L  child[m]  += sum_n prod_d S[c][d][n_d][m_d] parent[n] (applyL2L, FChebInterpolator.hpp:587-611)
//  L2P  phi += sum_n L[n] prod_d S_{n_d}(x_d); F += q * grad (applyL2PTotal, FChebInterpolator.hpp:1222-1417)
// with x mapped to [-1,1] around the leaf centre (map_glob_loc, Src/Kernels/Interpolation/FInterpMapping.hpp:
// 101-114; leaf centre FAbstractChebKernel.hpp:54-59).  Lagrange: FUnifInterpolator.hpp:340-549.
// Every contraction is done one axis at a time (p^4 work per cell instead of p^6); leaves are handled one
// warp each, parent cells one CTA each with one warp per child.
#include "common.cuh"

namespace b200 {

namespace {


// S_j(x) and dS_j/dx for j < p.  Chebyshev: 1/p + 2/p sum_o T_o(x) T_o(xbar_j), dT_o = o U_{o-1}.
template <int P>
__device__ __forceinline__ void basis_eval(int kernel, double x, const double *__restrict__ roots,
                                           const double *__restrict__ Tr, double *S, double *dS) {
  constexpr int p = P;
  if (kernel == B200FMM_LAGRANGE) {
    if (x > 1.0) x = 1.0;
    if (x < -1.0) x = -1.0;
    for (int j = 0; j < p; ++j) {
      double num = 1.0, den = 1.0, dsum = 0.0;
      for (int m = 0; m < p; ++m) {
        if (m == j) continue;
        den *= roots[j] - roots[m];
        num *= x - roots[m];
      }
      if (dS) {
        for (int k = 0; k < p; ++k) {
          if (k == j) continue;
          double t = 1.0;
          for (int m = 0; m < p; ++m)
            if (m != j && m != k) t *= x - roots[m];
          dsum += t;
        }
        dS[j] = dsum / den;
      }
      S[j] = num / den;
    }
    return;
  }
  double T[P], U[P];
  T[0] = 1.0;
  T[1] = x;
  U[0] = 1.0;
  U[1] = 2.0 * x;
#pragma unroll
  for (int o = 2; o < p; ++o) {
    T[o] = 2.0 * x * T[o - 1] - T[o - 2];
    U[o] = 2.0 * x * U[o - 1] - U[o - 2];
  }
  const double ip = 1.0 / p;
#pragma unroll
  for (int j = 0; j < p; ++j) {
    double s = ip, ds = 0.0;
#pragma unroll
    for (int o = 1; o < p; ++o) {
      const double t = 2.0 * ip * Tr[o * p + j];
      s += T[o] * t;
      ds += (double)o * U[o - 1] * t;
    }
    S[j] = s;
    if (dS) dS[j] = ds;
  }
}

// ---- P2M: one warp per leaf ------------------------------------------------------------------------
// The lanes first evaluate the 1-D weights of 32 particles (one particle each) into shared memory; then each
// lane owns nodes n = lane, lane+32, ... and sums q * wx * wy * wz over those particles.
constexpr int LEAF_WARPS = 4;

template <int P>
__global__ void __launch_bounds__(LEAF_WARPS * 32) p2m_kernel(
    int kernel, int R, long long N, long long nleaves, const long long *__restrict__ keys,
    const long long *__restrict__ leaf_start, const double *__restrict__ x, const double *__restrict__ y,
    const double *__restrict__ z, const double *__restrict__ q, double cx0, double cy0, double cz0, double leaf_w,
    const double *__restrict__ roots, const double *__restrict__ Tr, double *__restrict__ M) {
  constexpr int p = P, nn = P * P * P, NK = (nn + 31) / 32;
  __shared__ double W[LEAF_WARPS][32][3][P];
  __shared__ double Q[LEAF_WARPS][32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long leaf = (long long)blockIdx.x * LEAF_WARPS + w;
  if (leaf >= nleaves) return;
  int ix, iy, iz;
  morton_decode3(keys[leaf], ix, iy, iz);
  const double ctr[3] = {cx0 + (ix + 0.5) * leaf_w, cy0 + (iy + 0.5) * leaf_w, cz0 + (iz + 0.5) * leaf_w};
  const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1];
  for (int r = 0; r < R; ++r) {
    double acc[NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) acc[k] = 0.0;
    for (long long b = s0; b < s1; b += 32) {
      const int cnt = (int)min((long long)32, s1 - b);
      __syncwarp();
      if (lane < cnt) {
        const long long i = b + lane;
        const double pos[3] = {x[i], y[i], z[i]};
        for (int d = 0; d < 3; ++d) {
          const double a = ctr[d] - leaf_w / 2, bb = ctr[d] + leaf_w / 2;
          double wv[P];
          basis_eval<P>(kernel, (2.0 * pos[d] - bb - a) / (bb - a), roots, Tr, wv, nullptr);
#pragma unroll
          for (int k = 0; k < p; ++k) W[w][lane][d][k] = wv[k];
        }
        Q[w][lane] = q[(long long)r * N + i];
      }
      __syncwarp();
#pragma unroll
      for (int k = 0; k < NK; ++k) {
        const int n = lane + 32 * k;
        if (n < nn) {
          const int nx = n % p, ny = (n / p) % p, nz = n / (p * p);
          double a = acc[k];
          for (int j = 0; j < cnt; ++j) a += Q[w][j] * W[w][j][0][nx] * W[w][j][1][ny] * W[w][j][2][nz];
          acc[k] = a;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      const int n = lane + 32 * k;
      if (n < nn) M[(leaf * R + r) * nn + n] += acc[k];
    }
  }
}

// ---- M2M / L2L: one warp per child ------------------------------------------------------------------
// Each warp applies the child's three 1-D interpolators, one axis at a time, in its own shared-memory
// buffers.  M2M: the 8 children's contributions to the parent are then added in child order (deterministic).
__device__ inline void warp_contract(int p, int d, const double *__restrict__ A, const double *in, double *out,
                                     bool transpose, int lane) {
  const int nn = p * p * p;
  const int stride = d == 0 ? 1 : (d == 1 ? p : p * p);
  for (int e = lane; e < nn; e += 32) {
    const int nd = (e / stride) % p;
    const int base = e - nd * stride;
    double s = 0.0;
    for (int m = 0; m < p; ++m) s += (transpose ? A[m * p + nd] : A[nd * p + m]) * in[base + m * stride];
    out[e] = s;
  }
}

__global__ void __launch_bounds__(256) m2m_kernel(int p, int R, long long nparents, const int *__restrict__ child,
                                                  const double *__restrict__ S, const double *__restrict__ Mc,
                                                  double *__restrict__ Mp) {
  extern __shared__ double sh[];
  const int nn = p * p * p;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *b0 = sh + (size_t)w * 2 * nn, *b1 = b0 + nn;  // per-warp buffers; b0 ends with the contribution
  const long long pc = blockIdx.x;
  const int ci = child[pc * 8 + w];
  for (int r = 0; r < R; ++r) {
    if (ci >= 0) {
      for (int e = lane; e < nn; e += 32) b0[e] = Mc[((long long)ci * R + r) * nn + e];
      __syncwarp();
      warp_contract(p, 0, S + (w * 3 + 0) * p * p, b0, b1, false, lane);
      __syncwarp();
      warp_contract(p, 1, S + (w * 3 + 1) * p * p, b1, b0, false, lane);
      __syncwarp();
      warp_contract(p, 2, S + (w * 3 + 2) * p * p, b0, b1, false, lane);
    } else {
      for (int e = lane; e < nn; e += 32) b1[e] = 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      double s = 0.0;
      for (int k = 0; k < 8; ++k) s += sh[(size_t)k * 2 * nn + nn + e];
      Mp[(pc * R + r) * nn + e] += s;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) l2l_kernel(int p, int R, long long nparents, const int *__restrict__ child,
                                                  const double *__restrict__ S, const double *__restrict__ Lp,
                                                  double *__restrict__ Lc) {
  extern __shared__ double sh[];
  const int nn = p * p * p;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *par = sh;                                   // parent local
  double *b0 = sh + nn + (size_t)w * 2 * nn, *b1 = b0 + nn;
  const long long pc = blockIdx.x;
  const int ci = child[pc * 8 + w];
  for (int r = 0; r < R; ++r) {
    __syncthreads();
    for (int e = threadIdx.x; e < nn; e += blockDim.x) par[e] = Lp[(pc * R + r) * nn + e];
    __syncthreads();
    if (ci < 0) continue;
    warp_contract(p, 0, S + (w * 3 + 0) * p * p, par, b0, true, lane);
    __syncwarp();
    warp_contract(p, 1, S + (w * 3 + 1) * p * p, b0, b1, true, lane);
    __syncwarp();
    const double *A = S + (w * 3 + 2) * p * p;
    for (int e = lane; e < nn; e += 32) {
      const int nz = e / (p * p), base = e - nz * p * p;
      double s = 0.0;
      for (int m = 0; m < p; ++m) s += A[m * p + nz] * b1[base + m * p * p];
      Lc[((long long)ci * R + r) * nn + e] += s;
    }
  }
}

// ---- L2P: one warp per leaf, one particle per lane ----------------------------------------------------
template <int P>
__global__ void __launch_bounds__(LEAF_WARPS * 32) l2p_kernel(
    int kernel, int R, long long N, long long nleaves, const long long *__restrict__ keys,
    const long long *__restrict__ leaf_start, const double *__restrict__ x, const double *__restrict__ y,
    const double *__restrict__ z, const double *__restrict__ q, double cx0, double cy0, double cz0, double leaf_w,
    const double *__restrict__ roots, const double *__restrict__ Tr, const double *__restrict__ L,
    double *__restrict__ phi, double *__restrict__ fx, double *__restrict__ fy, double *__restrict__ fz) {
  constexpr int p = P, nn = P * P * P;
  __shared__ double sL[LEAF_WARPS][nn];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long leaf = (long long)blockIdx.x * LEAF_WARPS + w;
  if (leaf >= nleaves) return;
  double *Lw = sL[w];
  int ix, iy, iz;
  morton_decode3(keys[leaf], ix, iy, iz);
  const double ctr[3] = {cx0 + (ix + 0.5) * leaf_w, cy0 + (iy + 0.5) * leaf_w, cz0 + (iz + 0.5) * leaf_w};
  const double jac = 2.0 / leaf_w;
  const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1];
  for (int r = 0; r < R; ++r) {
    __syncwarp();
    for (int e = lane; e < nn; e += 32) Lw[e] = L[(leaf * R + r) * nn + e];
    __syncwarp();
    for (long long i = s0 + lane; i < s1; i += 32) {
      const double pos[3] = {x[i], y[i], z[i]};
      double wv[3][P], dw[3][P];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double a = ctr[d] - leaf_w / 2, b = ctr[d] + leaf_w / 2;
        basis_eval<P>(kernel, (2.0 * pos[d] - b - a) / (b - a), roots, Tr, wv[d], dw[d]);
      }
      double pv = 0, gx = 0, gy = 0, gz = 0;
#pragma unroll 1
      for (int kz = 0; kz < p; ++kz) {
        double bz = 0, bzx = 0, bzy = 0;
#pragma unroll
        for (int ky = 0; ky < p; ++ky) {
          const double *row = Lw + (kz * p + ky) * p;
          double a = 0, ad = 0;
#pragma unroll
          for (int kx = 0; kx < p; ++kx) {
            a += wv[0][kx] * row[kx];
            ad += dw[0][kx] * row[kx];
          }
          bz += wv[1][ky] * a;
          bzx += wv[1][ky] * ad;
          bzy += dw[1][ky] * a;
        }
        pv += wv[2][kz] * bz;
        gx += wv[2][kz] * bzx;
        gy += wv[2][kz] * bzy;
        gz += dw[2][kz] * bz;
      }
      const long long j = (long long)r * N + i;
      const double qq = q[j];
      phi[j] += pv;
      fx[j] += gx * jac * qq;
      fy[j] += gy * jac * qq;
      fz[j] += gz * jac * qq;
    }
  }
}

}  // namespace

b200fmm_status run_p2m(Context &c) {
  const int LL = c.H - 1;
  const Level &L = c.lv[LL];
  if (L.n == 0) return B200FMM_OK;
  const double W = c.cfg.box_width;
#define B200_P2M(PV)                                                                                        \
  case PV:                                                                                                  \
    p2m_kernel<PV><<<grid_for(L.n, LEAF_WARPS), LEAF_WARPS * 32, 0, c.stream>>>(                             \
        c.cfg.kernel, c.R, c.N, L.n, L.keys, c.d_leaf_start, c.d_x, c.d_y, c.d_z, c.d_q, c.cfg.center[0] - W / 2, \
        c.cfg.center[1] - W / 2, c.cfg.center[2] - W / 2, W / (double)(1 << LL), c.d_roots, c.d_Troots, L.M);     \
    break;
  switch (c.p) {
    B200_P2M(3) B200_P2M(4) B200_P2M(5) B200_P2M(6) B200_P2M(7) B200_P2M(8)
    default: return fail(B200FMM_ERR_UNSUPPORTED, "order not built");
  }
#undef B200_P2M
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

b200fmm_status run_m2m(Context &c, int level) {
  if (level < 2 || level >= c.H - 1) return fail(B200FMM_ERR_INVALID, "m2m: parent level must be in [2, height-2]");
  const Level &P = c.lv[level], &C = c.lv[level + 1];
  if (P.n == 0) return B200FMM_OK;
  const size_t sh = sizeof(double) * 16 * c.nn;
  B200_CUDA(cudaFuncSetAttribute(m2m_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
  m2m_kernel<<<(unsigned)P.n, 256, sh, c.stream>>>(c.p, c.R, P.n, P.child, c.d_S, C.M, P.M);
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

b200fmm_status run_l2l(Context &c, int level) {
  if (level < 2 || level >= c.H - 1) return fail(B200FMM_ERR_INVALID, "l2l: parent level must be in [2, height-2]");
  const Level &P = c.lv[level], &C = c.lv[level + 1];
  if (P.n == 0) return B200FMM_OK;
  const size_t sh = sizeof(double) * 17 * c.nn;
  B200_CUDA(cudaFuncSetAttribute(l2l_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
  l2l_kernel<<<(unsigned)P.n, 256, sh, c.stream>>>(c.p, c.R, P.n, P.child, c.d_S, P.L, C.L);
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

b200fmm_status run_l2p(Context &c) {
  const int LL = c.H - 1;
  const Level &L = c.lv[LL];
  if (L.n == 0) return B200FMM_OK;
  const double W = c.cfg.box_width;
#define B200_L2P(PV)                                                                                         \
  case PV:                                                                                                   \
    l2p_kernel<PV><<<grid_for(L.n, LEAF_WARPS), LEAF_WARPS * 32, 0, c.stream>>>(                              \
        c.cfg.kernel, c.R, c.N, L.n, L.keys, c.d_leaf_start, c.d_x, c.d_y, c.d_z, c.d_q, c.cfg.center[0] - W / 2,  \
        c.cfg.center[1] - W / 2, c.cfg.center[2] - W / 2, W / (double)(1 << LL), c.d_roots, c.d_Troots, L.L,      \
        c.d_phi, c.d_fx, c.d_fy, c.d_fz);                                                                    \
    break;
  switch (c.p) {
    B200_L2P(3) B200_L2P(4) B200_L2P(5) B200_L2P(6) B200_L2P(7) B200_L2P(8)
    default: return fail(B200FMM_ERR_UNSUPPORTED, "order not built");
  }
#undef B200_L2P
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

}  // namespace b200
