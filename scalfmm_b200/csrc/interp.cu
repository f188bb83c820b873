// P2M / M2M / L2L / L2P in FP64 for the Chebyshev and Lagrange bases.
//
//  P2M  M[n] += sum_particles q * prod_d S_{n_d}(x_d)      (FChebInterpolator::applyP2M,
//                                                            Src/Kernels/Chebyshev/FChebInterpolator.hpp:627-762)
//  M2M  parent[n] += sum_m prod_d S[c][d][n_d][m_d] child[m] (applyM2M, FChebInterpolator.hpp:560-584)
//  L2L  child[m]  += sum_n prod_d S[c][d][n_d][m_d] parent[n] (applyL2L, FChebInterpolator.hpp:587-611)
//  L2P  phi += sum_n L[n] prod_d S_{n_d}(x_d); F += q * grad (applyL2PTotal, FChebInterpolator.hpp:1222-1417)
// with x mapped to [-1,1] around the leaf centre (map_glob_loc, Src/Kernels/Interpolation/FInterpMapping.hpp:
// 101-114; leaf centre FAbstractChebKernel.hpp:54-59).  Lagrange: FUnifInterpolator.hpp:340-549.
// Every contraction is done one axis at a time (p^4 work per cell instead of p^6).
#include "common.cuh"

namespace b200 {

namespace {

constexpr int P2M_CHUNK = 32;

// S_j(x) and dS_j/dx for j < p.  Chebyshev: 1/p + 2/p sum_o T_o(x) T_o(xbar_j), dT_o = o U_{o-1}.
__device__ inline void basis_eval(int kernel, int p, double x, const double *__restrict__ roots,
                                  const double *__restrict__ Tr, double *S, double *dS) {
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
  double T[kMaxOrder], U[kMaxOrder];
  T[0] = 1.0;
  T[1] = x;
  U[0] = 1.0;
  U[1] = 2.0 * x;
  for (int o = 2; o < p; ++o) {
    T[o] = 2.0 * x * T[o - 1] - T[o - 2];
    U[o] = 2.0 * x * U[o - 1] - U[o - 2];
  }
  const double ip = 1.0 / p;
  for (int j = 0; j < p; ++j) {
    double s = ip, ds = 0.0;
    for (int o = 1; o < p; ++o) {
      const double t = 2.0 * ip * Tr[o * p + j];
      s += T[o] * t;
      ds += (double)o * U[o - 1] * t;
    }
    S[j] = s;
    if (dS) dS[j] = ds;
  }
}

__global__ void p2m_kernel(int kernel, int p, int R, long long N, const long long *__restrict__ keys,
                           const long long *__restrict__ leaf_start, const double *__restrict__ x,
                           const double *__restrict__ y, const double *__restrict__ z, const double *__restrict__ q,
                           double cx0, double cy0, double cz0, double leaf_w, const double *__restrict__ roots,
                           const double *__restrict__ Tr, double *__restrict__ M) {
  __shared__ double W[P2M_CHUNK][3][kMaxOrder];
  __shared__ double Q[P2M_CHUNK];
  const long long leaf = blockIdx.x;
  const int nn = p * p * p;
  int ix, iy, iz;
  morton_decode3(keys[leaf], ix, iy, iz);
  const double ctr[3] = {cx0 + (ix + 0.5) * leaf_w, cy0 + (iy + 0.5) * leaf_w, cz0 + (iz + 0.5) * leaf_w};
  const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1];
  for (int r = 0; r < R; ++r) {
    double acc[4] = {0, 0, 0, 0};
    for (long long b = s0; b < s1; b += P2M_CHUNK) {
      const int cnt = (int)min((long long)P2M_CHUNK, s1 - b);
      __syncthreads();
      if (threadIdx.x < 3 * cnt) {
        const int j = threadIdx.x / 3, d = threadIdx.x % 3;
        const double pos = d == 0 ? x[b + j] : (d == 1 ? y[b + j] : z[b + j]);
        const double a = ctr[d] - leaf_w / 2, bb = ctr[d] + leaf_w / 2;
        double w[kMaxOrder];
        basis_eval(kernel, p, (2.0 * pos - bb - a) / (bb - a), roots, Tr, w, nullptr);
        for (int k = 0; k < p; ++k) W[j][d][k] = w[k];
        if (d == 0) Q[j] = q[(long long)r * N + b + j];
      }
      __syncthreads();
      for (int k = 0; k < 4; ++k) {
        const int n = threadIdx.x + k * blockDim.x;
        if (n >= nn) break;
        const int nx = n % p, ny = (n / p) % p, nz = n / (p * p);
        double a = acc[k];
        for (int j = 0; j < cnt; ++j) a += Q[j] * W[j][0][nx] * W[j][1][ny] * W[j][2][nz];
        acc[k] = a;
      }
    }
    for (int k = 0; k < 4; ++k) {
      const int n = threadIdx.x + k * blockDim.x;
      if (n < nn) M[(leaf * R + r) * nn + n] += acc[k];
    }
  }
}

// One axis contraction out[..] = sum_m A[n_d][m_d] in[..] over axis d (0:x, 1:y, 2:z).
// transpose=false: A index [n*p + m] (M2M, from child index m to parent index n);
// transpose=true : A index [m*p + n] (L2L, from parent index m to child index n).
__device__ inline void contract_axis(int p, int d, const double *__restrict__ A, const double *in, double *out,
                                     bool transpose) {
  const int nn = p * p * p;
  for (int e = threadIdx.x; e < nn; e += blockDim.x) {
    const int i0 = e % p, i1 = (e / p) % p, i2 = e / (p * p);
    const int nd = d == 0 ? i0 : (d == 1 ? i1 : i2);
    const int stride = d == 0 ? 1 : (d == 1 ? p : p * p);
    const int base = e - nd * stride;
    double s = 0.0;
    for (int m = 0; m < p; ++m) s += (transpose ? A[m * p + nd] : A[nd * p + m]) * in[base + m * stride];
    out[e] = s;
  }
}

__global__ void m2m_kernel(int p, int R, long long nparents, const int *__restrict__ child,
                           const double *__restrict__ S, const double *__restrict__ Mc, double *__restrict__ Mp) {
  extern __shared__ double sh[];
  const int nn = p * p * p;
  double *b0 = sh, *b1 = sh + nn;
  const long long pc = blockIdx.x;
  for (int r = 0; r < R; ++r) {
    double acc[4] = {0, 0, 0, 0};
    for (int ch = 0; ch < 8; ++ch) {
      const int ci = child[pc * 8 + ch];
      if (ci < 0) continue;
      __syncthreads();
      for (int e = threadIdx.x; e < nn; e += blockDim.x) b0[e] = Mc[((long long)ci * R + r) * nn + e];
      __syncthreads();
      contract_axis(p, 0, S + (ch * 3 + 0) * p * p, b0, b1, false);
      __syncthreads();
      contract_axis(p, 1, S + (ch * 3 + 1) * p * p, b1, b0, false);
      __syncthreads();
      for (int k = 0; k < 4; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e >= nn) break;
        const int nz = e / (p * p), base = e - nz * p * p;
        const double *A = S + (ch * 3 + 2) * p * p;
        double s = 0.0;
        for (int m = 0; m < p; ++m) s += A[nz * p + m] * b0[base + m * p * p];
        acc[k] += s;
      }
    }
    for (int k = 0; k < 4; ++k) {
      const int e = threadIdx.x + k * blockDim.x;
      if (e < nn) Mp[(pc * R + r) * nn + e] += acc[k];
    }
  }
}

__global__ void l2l_kernel(int p, int R, long long nchildren, const long long *__restrict__ ckeys,
                           const int *__restrict__ parent, const double *__restrict__ S, const double *__restrict__ Lp,
                           double *__restrict__ Lc) {
  extern __shared__ double sh[];
  const int nn = p * p * p;
  double *b0 = sh, *b1 = sh + nn;
  const long long ci = blockIdx.x;
  const int ch = (int)(ckeys[ci] & 7);
  const long long pi = parent[ci];
  for (int r = 0; r < R; ++r) {
    __syncthreads();
    for (int e = threadIdx.x; e < nn; e += blockDim.x) b0[e] = Lp[(pi * R + r) * nn + e];
    __syncthreads();
    contract_axis(p, 0, S + (ch * 3 + 0) * p * p, b0, b1, true);
    __syncthreads();
    contract_axis(p, 1, S + (ch * 3 + 1) * p * p, b1, b0, true);
    __syncthreads();
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      const int nz = e / (p * p), base = e - nz * p * p;
      const double *A = S + (ch * 3 + 2) * p * p;
      double s = 0.0;
      for (int m = 0; m < p; ++m) s += A[m * p + nz] * b0[base + m * p * p];
      Lc[(ci * R + r) * nn + e] += s;
    }
  }
}

__global__ void l2p_kernel(int kernel, int p, int R, long long N, const long long *__restrict__ keys,
                           const long long *__restrict__ leaf_start, const double *__restrict__ x,
                           const double *__restrict__ y, const double *__restrict__ z, const double *__restrict__ q,
                           double cx0, double cy0, double cz0, double leaf_w, const double *__restrict__ roots,
                           const double *__restrict__ Tr, const double *__restrict__ L, double *__restrict__ phi,
                           double *__restrict__ fx, double *__restrict__ fy, double *__restrict__ fz) {
  extern __shared__ double sL[];  // [R][nn]
  const long long leaf = blockIdx.x;
  const int nn = p * p * p;
  for (int e = threadIdx.x; e < R * nn; e += blockDim.x) sL[e] = L[leaf * R * nn + e];
  __syncthreads();
  int ix, iy, iz;
  morton_decode3(keys[leaf], ix, iy, iz);
  const double ctr[3] = {cx0 + (ix + 0.5) * leaf_w, cy0 + (iy + 0.5) * leaf_w, cz0 + (iz + 0.5) * leaf_w};
  const double jac = 2.0 / leaf_w;
  const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1];
  for (long long i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
    const double pos[3] = {x[i], y[i], z[i]};
    double w[3][kMaxOrder], dw[3][kMaxOrder];
    for (int d = 0; d < 3; ++d) {
      const double a = ctr[d] - leaf_w / 2, b = ctr[d] + leaf_w / 2;
      basis_eval(kernel, p, (2.0 * pos[d] - b - a) / (b - a), roots, Tr, w[d], dw[d]);
    }
    for (int r = 0; r < R; ++r) {
      const double *Lr = sL + r * nn;
      double pv = 0, gx = 0, gy = 0, gz = 0;
      for (int kz = 0; kz < p; ++kz) {
        double bz = 0, bzx = 0, bzy = 0;
        for (int ky = 0; ky < p; ++ky) {
          const double *row = Lr + (kz * p + ky) * p;
          double a = 0, ad = 0;
          for (int kx = 0; kx < p; ++kx) {
            a += w[0][kx] * row[kx];
            ad += dw[0][kx] * row[kx];
          }
          bz += w[1][ky] * a;
          bzx += w[1][ky] * ad;
          bzy += dw[1][ky] * a;
        }
        pv += w[2][kz] * bz;
        gx += w[2][kz] * bzx;
        gy += w[2][kz] * bzy;
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
  p2m_kernel<<<(unsigned)L.n, 128, 0, c.stream>>>(c.cfg.kernel, c.p, c.R, c.N, L.keys, c.d_leaf_start, c.d_x, c.d_y,
                                                 c.d_z, c.d_q, c.cfg.center[0] - W / 2, c.cfg.center[1] - W / 2,
                                                 c.cfg.center[2] - W / 2, W / (double)(1 << LL), c.d_roots,
                                                 c.d_Troots, L.M);
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

b200fmm_status run_m2m(Context &c, int level) {
  if (level < 2 || level >= c.H - 1) return fail(B200FMM_ERR_INVALID, "m2m: parent level must be in [2, height-2]");
  const Level &P = c.lv[level], &C = c.lv[level + 1];
  if (P.n == 0) return B200FMM_OK;
  m2m_kernel<<<(unsigned)P.n, 128, 2 * c.nn * sizeof(double), c.stream>>>(c.p, c.R, P.n, P.child, c.d_S, C.M, P.M);
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

b200fmm_status run_l2l(Context &c, int level) {
  if (level < 2 || level >= c.H - 1) return fail(B200FMM_ERR_INVALID, "l2l: parent level must be in [2, height-2]");
  const Level &P = c.lv[level], &C = c.lv[level + 1];
  if (C.n == 0) return B200FMM_OK;
  l2l_kernel<<<(unsigned)C.n, 128, 2 * c.nn * sizeof(double), c.stream>>>(c.p, c.R, C.n, C.keys, C.parent, c.d_S,
                                                                          P.L, C.L);
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

b200fmm_status run_l2p(Context &c) {
  const int LL = c.H - 1;
  const Level &L = c.lv[LL];
  if (L.n == 0) return B200FMM_OK;
  const double W = c.cfg.box_width;
  const size_t sh = sizeof(double) * c.R * c.nn;
  if (sh > 48 * 1024)
    B200_CUDA(cudaFuncSetAttribute(l2p_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
  l2p_kernel<<<(unsigned)L.n, 64, sh, c.stream>>>(c.cfg.kernel, c.p, c.R, c.N, L.keys, c.d_leaf_start, c.d_x, c.d_y,
                                                 c.d_z, c.d_q, c.cfg.center[0] - W / 2, c.cfg.center[1] - W / 2,
                                                 c.cfg.center[2] - W / 2, W / (double)(1 << LL), c.d_roots,
                                                 c.d_Troots, L.L, c.d_phi, c.d_fx, c.d_fy, c.d_fz);
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

}  // namespace b200
