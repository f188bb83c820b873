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

// Interpolation nodes of every built order (3..8) and basis (Chebyshev, Lagrange), and the Chebyshev values
// T_o(node_j): read by P2M and L2P as constant-bank operands, so that the tables hold no registers.  Set per
// device when a handle builds its tables (upload_basis_constants); every handle of an order and basis writes
// the same values.
__constant__ double c_roots[2][kMaxOrder - 2][kMaxOrder];      // [basis: 1 = Lagrange][p - 3][j]
__constant__ double c_Tr[kMaxOrder - 2][kMaxOrder * kMaxOrder];  // [p - 3][o * p + j], Chebyshev

// S_j(x) and dS_j/dx for j < p.  Chebyshev: 1/p + 2/p sum_o T_o(x) T_o(xbar_j), dT_o = o U_{o-1}.
// Lagrange (equispaced nodes): prod_{m != j} (x - x_m) / (x_j - x_m) and its derivative.  Compile-time order
// and basis, every loop unrolled, so that S and dS stay in registers.
template <int P, bool LAGR>
__device__ __forceinline__ void basis_eval(double x, double *S, double *dS) {
  constexpr int p = P;
  const double *roots = c_roots[LAGR ? 1 : 0][P - 3];
  if constexpr (LAGR) {
    if (x > 1.0) x = 1.0;
    if (x < -1.0) x = -1.0;
#pragma unroll
    for (int j = 0; j < p; ++j) {
      double num = 1.0, den = 1.0, dsum = 0.0;
#pragma unroll
      for (int m = 0; m < p; ++m) {
        if (m == j) continue;
        den *= roots[j] - roots[m];
        num *= x - roots[m];
      }
      if (dS) {
#pragma unroll
        for (int k = 0; k < p; ++k) {
          if (k == j) continue;
          double t = 1.0;
#pragma unroll
          for (int m = 0; m < p; ++m)
            if (m != j && m != k) t *= x - roots[m];
          dsum += t;
        }
        dS[j] = dsum / den;
      }
      S[j] = num / den;
    }
  } else {
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
        const double t = 2.0 * ip * c_Tr[P - 3][o * p + j];
        s += T[o] * t;
        ds += (double)o * U[o - 1] * t;
      }
      S[j] = s;
      if (dS) dS[j] = ds;
    }
  }
}

// Record the largest |value| a warp wrote (mx per lane; every lane of the warp calls it) into one of the
// level's kMmaxSlots slots, chosen by block: non-negative doubles order like their bit patterns.
__device__ __forceinline__ void record_max(unsigned long long *slots, double mx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0 && mx > 0.0)
    atomicMax(slots + blockIdx.x % kMmaxSlots, (unsigned long long)__double_as_longlong(mx));
}

// ---- P2M: one 64-thread block per leaf -------------------------------------------------------------
// M[nx,ny,nz] = sum_j q_j Sx_j[nx] Sy_j[ny] Sz_j[nz].  The threads first evaluate the 1-D weights of up to 64
// particles (one each) into shared memory; then thread t < p^2 owns the node line (ny, nz) = (t % p, t / p)
// and keeps its p sums over nx in registers: per particle one product q Sy Sz and p FMAs with the
// broadcast Sx row, instead of three shared-memory reads per node and particle.
constexpr int P2M_THREADS = 64;
constexpr int L2P_WARPS = 2;  // L2P: leaves per CTA, one warp each (static shared memory <= 48 KB at order 8)

template <int P, bool LAGR>
__global__ void __launch_bounds__(P2M_THREADS, 8) p2m_kernel(
    int R, long long N, long long nleaves, const long long *__restrict__ keys,
    const long long *__restrict__ leaf_start, const double *__restrict__ x, const double *__restrict__ y,
    const double *__restrict__ z, const double *__restrict__ q, double cx0, double cy0, double cz0, double leaf_w,
    double *__restrict__ M, unsigned long long *__restrict__ mmax) {
  constexpr int p = P, nn = P * P * P, PX = (P + 1) & ~1;  // Sx rows padded to 16 bytes
  __shared__ __align__(16) double Wx[P2M_THREADS][PX];
  __shared__ double Wy[P2M_THREADS][P], Wz[P2M_THREADS][P], Q[P2M_THREADS];
  const int t = threadIdx.x;
  const long long leaf = blockIdx.x;
  int ix, iy, iz;
  morton_decode3(keys[leaf], ix, iy, iz);
  const double ctr[3] = {cx0 + (ix + 0.5) * leaf_w, cy0 + (iy + 0.5) * leaf_w, cz0 + (iz + 0.5) * leaf_w};
  const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1];
  const int ny = t % p, nz = t / p;
  const bool owner = t < p * p;
  for (int r = 0; r < R; ++r) {
    double acc[P];
#pragma unroll
    for (int k = 0; k < p; ++k) acc[k] = 0.0;
    for (long long b = s0; b < s1; b += P2M_THREADS) {
      const int cnt = (int)min((long long)P2M_THREADS, s1 - b);
      __syncthreads();
      if (t < cnt) {
        const long long i = b + t;
        const double pos[3] = {x[i], y[i], z[i]};
        double wv[P];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double a = ctr[d] - leaf_w / 2, bb = ctr[d] + leaf_w / 2;
          basis_eval<P, LAGR>((2.0 * pos[d] - bb - a) / (bb - a), wv, nullptr);
          double *dst = d == 0 ? Wx[t] : (d == 1 ? Wy[t] : Wz[t]);
#pragma unroll
          for (int k = 0; k < p; ++k) dst[k] = wv[k];
        }
        Q[t] = q[(long long)r * N + i];
      }
      __syncthreads();
      if (owner) {
        for (int j = 0; j < cnt; ++j) {
          const double w = Q[j] * Wy[j][ny] * Wz[j][nz];
#pragma unroll
          for (int k = 0; k < p; ++k) acc[k] += w * Wx[j][k];
        }
      }
    }
    double mx = 0.0;
    if (owner) {
      double *out = M + (leaf * R + r) * nn + (nz * p + ny) * p;
#pragma unroll
      for (int k = 0; k < p; ++k) {
        const double v = out[k] + acc[k];
        out[k] = v;
        mx = fmax(mx, fabs(v));
      }
    }
    if (mmax) record_max(mmax, mx);
  }
}

// Copy NN doubles with T threads, all loads issued before the first store (one memory latency per copy
// instead of one per element); ADD adds into dst instead of overwriting.
template <int NN, int T, bool ADD = false>
__device__ __forceinline__ void copy_block(double *dst, const double *__restrict__ src, int tid) {
  constexpr int K = (NN + T - 1) / T;
  double v[K], d[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int e = tid + k * T;
    v[k] = e < NN ? src[e] : 0.0;
    if (ADD) d[k] = e < NN ? dst[e] : 0.0;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int e = tid + k * T;
    if (e < NN) dst[e] = ADD ? d[k] + v[k] : v[k];
  }
}

// ---- M2M / L2L: one warp per child ------------------------------------------------------------------
// Each warp applies the child's three 1-D interpolators, one axis at a time, in its own shared-memory
// buffers.  A lane owns whole lines along the axis: it loads the line's p values into registers and writes
// the p results, with the p x p interpolator in registers.  M2M: the 8 children's contributions to the
// parent are then added in child order (deterministic).
template <int P, bool TRANSPOSE>
__device__ __forceinline__ void warp_lines(const double *__restrict__ A, int d, const double *in, double *out,
                                           int lane) {
  constexpr int p = P, nl = P * P;
  double a[P][P];
#pragma unroll
  for (int i = 0; i < p; ++i)
#pragma unroll
    for (int m = 0; m < p; ++m) a[i][m] = TRANSPOSE ? A[m * p + i] : A[i * p + m];
  const int stride = d == 0 ? 1 : (d == 1 ? p : p * p);
  for (int l = lane; l < nl; l += 32) {
    // first element of line l: the two other indices of the line, in increasing axis order
    const int base = d == 0 ? l * p : (d == 1 ? (l % p) + (l / p) * p * p : l);
    double v[P];
#pragma unroll
    for (int m = 0; m < p; ++m) v[m] = in[base + m * stride];
#pragma unroll
    for (int i = 0; i < p; ++i) {
      double s = 0.0;
#pragma unroll
      for (int m = 0; m < p; ++m) s += a[i][m] * v[m];
      out[base + i * stride] = s;
    }
  }
}

template <int P>
__global__ void __launch_bounds__(256) m2m_kernel(int R, long long nparents, const int *__restrict__ child,
                                                  const double *__restrict__ S, const double *__restrict__ Mc,
                                                  double *__restrict__ Mp, unsigned long long *__restrict__ mmax) {
  constexpr int p = P, nn = P * P * P;
  extern __shared__ double sh[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *b0 = sh + (size_t)w * 2 * nn, *b1 = b0 + nn;  // per-warp buffers; b1 ends with the contribution
  const long long pc = blockIdx.x;
  const int ci = child[pc * 8 + w];
  for (int r = 0; r < R; ++r) {
    if (ci >= 0) {
      copy_block<nn, 32>(b0, Mc + ((long long)ci * R + r) * nn, lane);
      __syncwarp();
      warp_lines<P, false>(S + (w * 3 + 0) * p * p, 0, b0, b1, lane);
      __syncwarp();
      warp_lines<P, false>(S + (w * 3 + 1) * p * p, 1, b1, b0, lane);
      __syncwarp();
      warp_lines<P, false>(S + (w * 3 + 2) * p * p, 2, b0, b1, lane);
    } else {
      for (int e = lane; e < nn; e += 32) b1[e] = 0.0;
    }
    __syncthreads();
    double mx = 0.0;
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 8; ++k) s += sh[(size_t)k * 2 * nn + nn + e];
      const double v = Mp[(pc * R + r) * nn + e] + s;
      Mp[(pc * R + r) * nn + e] = v;
      mx = fmax(mx, fabs(v));
    }
    if (mmax) record_max(mmax, mx);
    __syncthreads();
  }
}

template <int P>
__global__ void __launch_bounds__(256) l2l_kernel(int R, long long nparents, const int *__restrict__ child,
                                                  const double *__restrict__ S, const double *__restrict__ Lp,
                                                  double *__restrict__ Lc) {
  constexpr int p = P, nn = P * P * P;
  extern __shared__ double sh[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *par = sh;  // parent local
  double *b0 = sh + nn + (size_t)w * 2 * nn, *b1 = b0 + nn;
  const long long pc = blockIdx.x;
  const int ci = child[pc * 8 + w];
  for (int r = 0; r < R; ++r) {
    __syncthreads();
    copy_block<nn, 256>(par, Lp + (pc * R + r) * nn, threadIdx.x);
    __syncthreads();
    if (ci < 0) continue;
    warp_lines<P, true>(S + (w * 3 + 0) * p * p, 0, par, b0, lane);
    __syncwarp();
    warp_lines<P, true>(S + (w * 3 + 1) * p * p, 1, b0, b1, lane);
    __syncwarp();
    warp_lines<P, true>(S + (w * 3 + 2) * p * p, 2, b1, b0, lane);
    __syncwarp();
    double *out = Lc + ((long long)ci * R + r) * nn;
    copy_block<nn, 32, true>(out, b0, lane);
  }
}

// ---- L2P: one warp per leaf, one particle per lane ----------------------------------------------------
// The leaf's local expansion sits in shared memory; each lane contracts it with its particle's weights one
// axis at a time: the x weights in registers, the y and z weights (and derivatives) in the lane's own
// shared-memory row, so that the loops over y and z need no register indexing and the kernel stays small.
template <int P, bool LAGR>
__global__ void __launch_bounds__(L2P_WARPS * 32) l2p_kernel(
    int R, long long N, long long nleaves, const long long *__restrict__ keys,
    const long long *__restrict__ leaf_start, const double *__restrict__ x, const double *__restrict__ y,
    const double *__restrict__ z, const double *__restrict__ q, double cx0, double cy0, double cz0, double leaf_w,
    const double *__restrict__ L,
    double *__restrict__ phi, double *__restrict__ fx, double *__restrict__ fy, double *__restrict__ fz,
    const long long *__restrict__ shard) {
  constexpr int p = P, nn = P * P * P;
  __shared__ double sL[L2P_WARPS][nn];
  __shared__ double sW[L2P_WARPS][32][4 * P + 1];  // wy, dwy, wz, dwz of each lane's particle (+1: banks)
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // every leaf, or the shard's [shard[0], shard[1])
  const long long leaf = (shard ? shard[0] : 0) + (long long)blockIdx.x * L2P_WARPS + w;
  if (leaf >= (shard ? shard[1] : nleaves)) return;
  double *Lw = sL[w];
  double *wy = sW[w][lane], *dwy = wy + P, *wz = wy + 2 * P, *dwz = wy + 3 * P;
  int ix, iy, iz;
  morton_decode3(keys[leaf], ix, iy, iz);
  const double cx = cx0 + (ix + 0.5) * leaf_w, cy = cy0 + (iy + 0.5) * leaf_w, cz = cz0 + (iz + 0.5) * leaf_w;
  const double jac = 2.0 / leaf_w;
  const long long s0 = leaf_start[leaf], s1 = leaf_start[leaf + 1];
  for (int r = 0; r < R; ++r) {
    __syncwarp();
    copy_block<nn, 32>(Lw, L + (leaf * R + r) * nn, lane);
    __syncwarp();
    for (long long i = s0 + lane; i < s1; i += 32) {
      double wx[P], dwx[P];
      {
        double t[P], dt[P];
        basis_eval<P, LAGR>((2.0 * y[i] - 2.0 * cy) / leaf_w, t, dt);
#pragma unroll
        for (int k = 0; k < p; ++k) {
          wy[k] = t[k];
          dwy[k] = dt[k];
        }
        basis_eval<P, LAGR>((2.0 * z[i] - 2.0 * cz) / leaf_w, t, dt);
#pragma unroll
        for (int k = 0; k < p; ++k) {
          wz[k] = t[k];
          dwz[k] = dt[k];
        }
      }
      basis_eval<P, LAGR>((2.0 * x[i] - 2.0 * cx) / leaf_w, wx, dwx);
      double pv = 0, gx = 0, gy = 0, gz = 0;
#pragma unroll 1
      for (int kz = 0; kz < p; ++kz) {
        double bz = 0, bzx = 0, bzy = 0;
#pragma unroll 1
        for (int ky = 0; ky < p; ++ky) {
          const double *row = Lw + (kz * p + ky) * p;
          double a = 0, ad = 0;
#pragma unroll
          for (int kx = 0; kx < p; ++kx) {
            const double v = row[kx];
            a += wx[kx] * v;
            ad += dwx[kx] * v;
          }
          const double yk = wy[ky];
          bz += yk * a;
          bzx += yk * ad;
          bzy += dwy[ky] * a;
        }
        const double zk = wz[kz];
        pv += zk * bz;
        gx += zk * bzx;
        gy += zk * bzy;
        gz += dwz[kz] * bz;
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

b200fmm_status upload_basis_constants(const Context &c, const double *roots, const double *Tr) {
  const int p = c.p;
  if (p < 3 || p > kMaxOrder) return B200FMM_OK;  // no P2M / L2P kernel is built for this order
  const int lag = c.cfg.kernel == B200FMM_LAGRANGE ? 1 : 0;
  B200_CUDA(cudaMemcpyToSymbol(c_roots, roots, sizeof(double) * p,
                               sizeof(double) * ((size_t)(lag * (kMaxOrder - 2) + p - 3) * kMaxOrder)));
  if (!lag)
    B200_CUDA(cudaMemcpyToSymbol(c_Tr, Tr, sizeof(double) * p * p, sizeof(double) * (size_t)(p - 3) * kMaxOrder * kMaxOrder));
  return B200FMM_OK;
}

b200fmm_status run_p2m(Context &c) {
  const int LL = c.H - 1;
  const Level &L = c.lv[LL];
  if (L.n == 0) return B200FMM_OK;
  const double W = c.cfg.box_width;
  const double x0 = c.cfg.center[0] - W / 2, y0 = c.cfg.center[1] - W / 2, z0 = c.cfg.center[2] - W / 2;
  const double lw = W / (double)(1 << LL);
  const bool lagr = c.cfg.kernel == B200FMM_LAGRANGE;
  unsigned long long *mmax = c.mmax_out ? c.mmax_out + (size_t)LL * kMmaxSlots : nullptr;
#define B200_P2M(PV)                                                                                        \
  case PV:                                                                                                  \
    if (lagr)                                                                                               \
      p2m_kernel<PV, true><<<(unsigned)L.n, P2M_THREADS, 0, c.stream>>>(                                     \
          c.R, c.N, L.n, L.keys, c.d_leaf_start, c.d_x, c.d_y, c.d_z, c.d_q, x0, y0, z0, lw, L.M, mmax);              \
    else                                                                                                    \
      p2m_kernel<PV, false><<<(unsigned)L.n, P2M_THREADS, 0, c.stream>>>(                                    \
          c.R, c.N, L.n, L.keys, c.d_leaf_start, c.d_x, c.d_y, c.d_z, c.d_q, x0, y0, z0, lw, L.M, mmax);              \
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
  unsigned long long *mmax = c.mmax_out ? c.mmax_out + (size_t)level * kMmaxSlots : nullptr;
#define B200_M2M(PV)                                                                                        \
  case PV:                                                                                                  \
    B200_CUDA(cudaFuncSetAttribute(m2m_kernel<PV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));   \
    m2m_kernel<PV><<<(unsigned)P.n, 256, sh, c.stream>>>(c.R, P.n, P.child, c.d_S, C.M, P.M, mmax);         \
    break;
  switch (c.p) {
    B200_M2M(3) B200_M2M(4) B200_M2M(5) B200_M2M(6) B200_M2M(7) B200_M2M(8)
    default: return fail(B200FMM_ERR_UNSUPPORTED, "order not built");
  }
#undef B200_M2M
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

b200fmm_status run_l2l(Context &c, int level) {
  if (level < 2 || level >= c.H - 1) return fail(B200FMM_ERR_INVALID, "l2l: parent level must be in [2, height-2]");
  const Level &P = c.lv[level], &C = c.lv[level + 1];
  if (P.n == 0) return B200FMM_OK;
  const size_t sh = sizeof(double) * 17 * c.nn;
#define B200_L2L(PV)                                                                                        \
  case PV:                                                                                                  \
    B200_CUDA(cudaFuncSetAttribute(l2l_kernel<PV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));   \
    l2l_kernel<PV><<<(unsigned)P.n, 256, sh, c.stream>>>(c.R, P.n, P.child, c.d_S, P.L, C.L);               \
    break;
  switch (c.p) {
    B200_L2L(3) B200_L2L(4) B200_L2L(5) B200_L2L(6) B200_L2L(7) B200_L2L(8)
    default: return fail(B200FMM_ERR_UNSUPPORTED, "order not built");
  }
#undef B200_L2L
  ++c.launches;
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

b200fmm_status run_l2p(Context &c, const long long *shard) {
  const int LL = c.H - 1;
  const Level &L = c.lv[LL];
  if (L.n == 0) return B200FMM_OK;
  const double W = c.cfg.box_width;
  const double x0 = c.cfg.center[0] - W / 2, y0 = c.cfg.center[1] - W / 2, z0 = c.cfg.center[2] - W / 2;
  const double lw = W / (double)(1 << LL);
  const bool lagr = c.cfg.kernel == B200FMM_LAGRANGE;
#define B200_L2P(PV)                                                                                         \
  case PV:                                                                                                   \
    if (lagr)                                                                                                \
      l2p_kernel<PV, true><<<grid_for(L.n, L2P_WARPS), L2P_WARPS * 32, 0, c.stream>>>(                      \
          c.R, c.N, L.n, L.keys, c.d_leaf_start, c.d_x, c.d_y, c.d_z, c.d_q, x0, y0, z0, lw, L.L, c.d_phi,       \
          c.d_fx, c.d_fy, c.d_fz, shard);                                          \
    else                                                                                                     \
      l2p_kernel<PV, false><<<grid_for(L.n, L2P_WARPS), L2P_WARPS * 32, 0, c.stream>>>(                     \
          c.R, c.N, L.n, L.keys, c.d_leaf_start, c.d_x, c.d_y, c.d_z, c.d_q, x0, y0, z0, lw, L.L, c.d_phi,       \
          c.d_fx, c.d_fy, c.d_fz, shard);                                          \
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
