// Symmetric M2L operator compression on the GPU, in FP64.
//
// FChebSymM2LHandler::ComputeAndCompress (Src/Kernels/Chebyshev/FChebSymM2LHandler.hpp:39-281) compresses the
// weighted kernel matrix of each of the 16 canonical transfer vectors: a partially pivoted ACA
// (Src/Utils/FAca.hpp:141-225) gives K ~ U V^T of some rank k, a QR of both factors and an SVD of Ru Rv^T
// recompress it, and the rank rule of FSvd::getRank (Src/Utils/FSvd.hpp:53-64) cuts it at the target
// accuracy.  Here every step runs on the device, one CTA per class:
//   aca_kernel   the ACA loop (row residual, column pivot, column residual, row pivot, Frobenius-norm update,
//                stop test), one thread per node;
//   qr_kernel    Householder QR of the p^3 x k factors (grid: class x factor), explicit Q;
//   svd_kernel   Ru Rv^T, a one-sided Jacobi SVD with the round-robin pair order (k/2 disjoint rotations at
//                a time, one warp each), singular values sorted descending, the rank rule, and the output
//                factors U = Qu Ur diag(s) / w, V = Qv Vr / w (the un-weighting of
//                FChebSymM2LHandler.hpp:257-261).
// Every sum has a fixed order, so results repeat bit for bit from run to run.  The ACA's sums run in node
// order without fused multiply-adds, as a sequential CPU loop computes them: its stop test decides the number
// of terms, and with it the final rank, at the last bit for some classes.
#include "common.cuh"

#include <algorithm>

namespace b200 {

namespace {

constexpr int CT = 512;  // threads per CTA: one per interpolation node up to order 8
constexpr int CW = CT / 32;

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// sum over the CTA, the same value in every thread
__device__ double block_sum(double x, double *red) {
  x = warp_sum(x);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < CW; ++i) s += red[i];
  return s;
}

// index of the largest a > 0 over the CTA (ties: the smallest index), or -1 when no a is > 0; entries that
// take no part pass a = -1
__device__ int block_argmax(double a, int i, double *red, int *redi) {
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const double oa = __shfl_xor_sync(0xffffffffu, a, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (oa > a || (oa == a && oi < i)) {
      a = oa;
      i = oi;
    }
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = a;
    redi[threadIdx.x >> 5] = i;
  }
  __syncthreads();
  double ba = red[0];
  int bi = redi[0];
  for (int w = 1; w < CW; ++w)
    if (red[w] > ba || (red[w] == ba && redi[w] < bi)) {
      ba = red[w];
      bi = redi[w];
    }
  return ba > 0.0 ? bi : -1;
}

// Partially pivoted ACA of the class matrix A (row-major, A[t * nn + s]); the factor vectors are written as
// rows of U and V ([l][nn]).  kout = the number of terms, status 1 = zero pivot.
__global__ void __launch_bounds__(CT) aca_kernel(int nn, const double *__restrict__ Aall, double eps2,
                                                 double *__restrict__ Uall, double *__restrict__ Vall,
                                                 int *__restrict__ kout, int *__restrict__ status) {
  __shared__ double red[CW];
  __shared__ int redi[CW];
  __shared__ double coef[CT], ab[CT], sv[CT], su[CT];
  __shared__ char rfree[CT], cfree[CT];
  const int ci = blockIdx.x, t = threadIdx.x;
  const double *A = Aall + (size_t)ci * nn * nn;
  double *U = Uall + (size_t)ci * nn * nn, *V = Vall + (size_t)ci * nn * nn;
  if (t < nn) rfree[t] = cfree[t] = 1;
  int I = 0, J = 0, k = 0;
  double norm2S = 0.0;
  for (;;) {
    __syncthreads();
    // row residual v = A[I, :] - sum_l U_l[I] V_l
    if (t < k) coef[t] = U[(size_t)t * nn + I];
    if (t == 0) rfree[I] = 0;
    __syncthreads();
    double vj = 0.0;
    if (t < nn) {
      vj = A[(size_t)I * nn + t];
      for (int l = 0; l < k; ++l) vj = __dsub_rn(vj, __dmul_rn(coef[l], V[(size_t)l * nn + t]));
    }
    const int Jn = block_argmax((t < nn && cfree[t]) ? fabs(vj) : -1.0, t, red, redi);
    if (Jn >= 0) J = Jn;
    if (t < nn) sv[t] = vj;
    __syncthreads();
    const double vJ = sv[J];
    if (vJ == 0.0) {
      if (t == 0) status[ci] = 1;
      return;
    }
    vj = __dmul_rn(vj, 1.0 / vJ);
    __syncthreads();
    // column residual u = A[:, J] - sum_l V_l[J] U_l
    if (t < nn) sv[t] = vj;
    if (t < k) coef[t] = V[(size_t)t * nn + J];
    if (t == 0) cfree[J] = 0;
    __syncthreads();
    double ui = 0.0;
    if (t < nn) {
      ui = A[(size_t)t * nn + J];
      for (int l = 0; l < k; ++l) ui = __dsub_rn(ui, __dmul_rn(coef[l], U[(size_t)l * nn + t]));
    }
    const int In = block_argmax((t < nn && rfree[t]) ? fabs(ui) : -1.0, t, red, redi);
    if (In >= 0) I = In;
    if (t < nn) su[t] = ui;
    __syncthreads();
    // cross terms of the norm update, sum_l (u . U_l)(V_l . v), and |u|^2, |v|^2: one thread per sum, each
    // summed in node order without fused multiply-adds.  The stop test of the ACA is sensitive to rounding at
    // the last bit (one more or one fewer term changes the final rank), and this order reproduces the
    // reference's ranks.
    if (t < k) {
      double a = 0.0, b = 0.0;
      for (int i = 0; i < nn; ++i) a = __dadd_rn(a, __dmul_rn(su[i], U[(size_t)t * nn + i]));
      for (int i = 0; i < nn; ++i) b = __dadd_rn(b, __dmul_rn(V[(size_t)t * nn + i], sv[i]));
      ab[t] = __dmul_rn(a, b);
    } else if (t == CT - 1) {  // k < nn <= CT, so this thread has no cross term
      double q = 0.0, r = 0.0;
      for (int i = 0; i < nn; ++i) q = __dadd_rn(q, __dmul_rn(su[i], su[i]));
      for (int i = 0; i < nn; ++i) r = __dadd_rn(r, __dmul_rn(sv[i], sv[i]));
      red[0] = q;
      red[1] = r;
    }
    __syncthreads();
    const double uu = red[0], vv = red[1];
    double cross = 0.0;
    for (int l = 0; l < k; ++l) cross = __dadd_rn(cross, ab[l]);
    const double n2 = __dmul_rn(uu, vv);
    norm2S = __dadd_rn(norm2S, __dadd_rn(n2, 2.0 * cross));
    if (t < nn) {
      U[(size_t)k * nn + t] = ui;
      V[(size_t)k * nn + t] = vj;
    }
    ++k;
    if (!(n2 > __dmul_rn(eps2, norm2S)) || k >= nn) break;
  }
  if (t == 0) kout[ci] = k;
}

// Householder QR of the nn x k factor (columns = the rows l of U or V): R (k x k, column-major) and the
// explicit Q (k columns of nn).  grid (class, factor).
__global__ void __launch_bounds__(CT) qr_kernel(int nn, int kmax, const int *__restrict__ kk,
                                                double *__restrict__ Uall, double *__restrict__ Vall,
                                                double *__restrict__ Hall, double *__restrict__ Qall,
                                                double *__restrict__ Rall) {
  __shared__ double red[CW];
  __shared__ double beta[CT];
  const int ci = blockIdx.x, f = blockIdx.y, t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int k = kk[ci];
  double *A = (f == 0 ? Uall : Vall) + (size_t)ci * nn * nn;
  const size_t slot = (size_t)ci * 2 + f;
  double *H = Hall + slot * kmax * nn, *Q = Qall + slot * kmax * nn, *R = Rall + slot * kmax * kmax;
  for (int j = 0; j < k; ++j) {
    const double a = (t >= j && t < nn) ? A[(size_t)j * nn + t] : 0.0;
    const double norm = sqrt(block_sum(a * a, red));
    const double a0 = A[(size_t)j * nn + j];
    const double alpha = a0 >= 0 ? -norm : norm;
    const double h = (t >= j && t < nn) ? a - (t == j ? alpha : 0.0) : 0.0;
    const double hn2 = block_sum(h * h, red);
    const double bj = hn2 > 0 ? 2.0 / hn2 : 0.0;
    if (t < nn) H[(size_t)j * nn + t] = h;
    if (t == 0) beta[j] = bj;
    __syncthreads();
    for (int c = j + w; c < k; c += CW) {
      double d = 0.0;
      for (int i = j + lane; i < nn; i += 32) d += H[(size_t)j * nn + i] * A[(size_t)c * nn + i];
      d = warp_sum(d) * bj;
      for (int i = j + lane; i < nn; i += 32) A[(size_t)c * nn + i] -= d * H[(size_t)j * nn + i];
    }
    __syncthreads();
  }
  for (int e = t; e < k * k; e += CT) {
    const int c = e / k, i = e % k;
    R[e] = i <= c ? A[(size_t)c * nn + i] : 0.0;
  }
  for (int e = t; e < k * nn; e += CT) Q[e] = (e % nn == e / nn) ? 1.0 : 0.0;
  __syncthreads();
  for (int j = k - 1; j >= 0; --j) {
    for (int c = w; c < k; c += CW) {
      double d = 0.0;
      for (int i = j + lane; i < nn; i += 32) d += H[(size_t)j * nn + i] * Q[(size_t)c * nn + i];
      d = warp_sum(d) * beta[j];
      for (int i = j + lane; i < nn; i += 32) Q[(size_t)c * nn + i] -= d * H[(size_t)j * nn + i];
    }
    __syncthreads();
  }
}

// SVD of Ru Rv^T by one-sided Jacobi, the rank rule, and the un-weighted output factors:
// out[ci][0][r][i] = U row r, out[ci][1][r][i] = V row r, r < rank.  status 2 = no convergence, 3 = rank 0.
__global__ void __launch_bounds__(CT) svd_kernel(int nn, int kmax, const int *__restrict__ kk, double eps,
                                                 const double *__restrict__ Rall, const double *__restrict__ Qall,
                                                 const double *__restrict__ wgt, double *__restrict__ Pall,
                                                 double *__restrict__ Vmall, double *__restrict__ Sall,
                                                 double *__restrict__ out, int *__restrict__ rank_out,
                                                 int *__restrict__ status) {
  __shared__ double sv[CT], ss[CT];
  __shared__ int pos[CT];
  __shared__ int rotated, rank_sh;
  const int ci = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int k = kk[ci];
  const double *Ru = Rall + (size_t)ci * 2 * kmax * kmax, *Rv = Ru + (size_t)kmax * kmax;
  const double *Qu = Qall + (size_t)ci * 2 * kmax * nn, *Qv = Qu + (size_t)kmax * nn;
  double *P = Pall + (size_t)ci * kmax * kmax, *Vm = Vmall + (size_t)ci * kmax * kmax;
  double *Us = Sall + (size_t)ci * 2 * kmax * kmax, *Vs = Us + (size_t)kmax * kmax;
  // P = Ru Rv^T (column-major): P[b][a] = sum_l Ru[l][a] Rv[l][b]
  for (int e = t; e < k * k; e += CT) {
    const int b = e / k, a = e % k;
    double s = 0.0;
    for (int l = 0; l < k; ++l) s += Ru[(size_t)l * k + a] * Rv[(size_t)l * k + b];
    P[e] = s;
    Vm[e] = a == b ? 1.0 : 0.0;
  }
  const int kp = k + (k & 1);  // players of the round-robin, one dummy when k is odd
  bool converged = false;
  for (int sweep = 0; sweep < 80 && !converged; ++sweep) {
    if (t == 0) rotated = 0;
    __syncthreads();
    for (int r = 0; r < kp - 1; ++r) {
      for (int q = w; q < kp / 2; q += CW) {
        int a, b;
        if (q == 0) {
          a = r;
          b = kp - 1;
        } else {
          a = (r + q) % (kp - 1);
          b = (r - q + kp - 1) % (kp - 1);
        }
        if (a > b) {
          const int x = a;
          a = b;
          b = x;
        }
        if (b >= k) continue;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i = lane; i < k; i += 32) {
          const double x = P[(size_t)a * k + i], y = P[(size_t)b * k + i];
          al += x * x;
          be += y * y;
          ga += x * y;
        }
        al = warp_sum(al);
        be = warp_sum(be);
        ga = warp_sum(ga);
        if (fabs(ga) <= 1e-15 * sqrt(al * be) || ga == 0.0) continue;
        if (lane == 0) rotated = 1;
        const double zeta = (be - al) / (2.0 * ga);
        const double tn = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + tn * tn), sn = cs * tn;
        for (int i = lane; i < k; i += 32) {
          const double x = P[(size_t)a * k + i], y = P[(size_t)b * k + i];
          P[(size_t)a * k + i] = cs * x - sn * y;
          P[(size_t)b * k + i] = sn * x + cs * y;
          const double vx = Vm[(size_t)a * k + i], vy = Vm[(size_t)b * k + i];
          Vm[(size_t)a * k + i] = cs * vx - sn * vy;
          Vm[(size_t)b * k + i] = sn * vx + cs * vy;
        }
      }
      __syncthreads();
    }
    converged = rotated == 0;
    __syncthreads();
  }
  if (!converged) {
    if (t == 0) status[ci] = 2;
    return;
  }
  // singular values (column norms), sorted descending, ties in column order
  for (int j = w; j < k; j += CW) {
    double s = 0.0;
    for (int i = lane; i < k; i += 32) s += P[(size_t)j * k + i] * P[(size_t)j * k + i];
    s = warp_sum(s);
    if (lane == 0) sv[j] = sqrt(s);
  }
  __syncthreads();
  if (t < k) {
    int n = 0;
    for (int i = 0; i < k; ++i) n += (sv[i] > sv[t] || (sv[i] == sv[t] && i < t)) ? 1 : 0;
    pos[t] = n;
    ss[n] = sv[t];
  }
  __syncthreads();
  for (int e = t; e < k * k; e += CT) {
    const int j = e / k, i = e % k, jj = pos[j];
    Us[(size_t)jj * k + i] = sv[j] > 0 ? P[e] / sv[j] : 0.0;
    Vs[(size_t)jj * k + i] = Vm[e];
  }
  if (t == 0) {
    double nrm2 = 0.0;
    for (int i = 0; i < k; ++i) nrm2 += ss[i] * ss[i];
    int rank = 0;
    double acc = 0.0;
    for (int i = k; i > 0; --i) {
      acc += ss[i - 1] * ss[i - 1];
      if (acc > eps * eps * nrm2) {
        rank = i;
        break;
      }
    }
    rank_sh = rank;
    rank_out[ci] = rank;
    if (rank == 0) status[ci] = 3;
  }
  __syncthreads();
  const int rank = rank_sh;
  double *Uo = out + (size_t)ci * 2 * kmax * nn, *Vo = Uo + (size_t)kmax * nn;
  for (int e = t; e < rank * nn; e += CT) {
    const int r = e / nn, i = e % nn;
    double su = 0.0, sw = 0.0;
    for (int l = 0; l < k; ++l) {
      su += Qu[(size_t)l * nn + i] * Us[(size_t)r * k + l];
      sw += Qv[(size_t)l * nn + i] * Vs[(size_t)r * k + l];
    }
    Uo[e] = su * ss[r] / wgt[i];
    Vo[e] = sw / wgt[i];
  }
}

}  // namespace

b200fmm_status compress_classes(Context &c, int ncls, const double *dA, const double *dw, double eps,
                                std::vector<int> &ranks, std::vector<double> &uv) {
  const int nn = c.nn;
  if (nn > CT) return fail(B200FMM_ERR_UNSUPPORTED, "compression: order too high");
  double *dU = nullptr, *dV = nullptr, *dH = nullptr, *dQ = nullptr, *dR = nullptr, *dP = nullptr,
         *dVm = nullptr, *dS = nullptr, *dout = nullptr;
  int *dk = nullptr, *drank = nullptr, *dst = nullptr;
  std::vector<void *> owned;
  auto alloc = [&](auto **p, size_t bytes) {
    const bool ok = cudaMalloc((void **)p, std::max<size_t>(bytes, 16)) == cudaSuccess;
    if (ok) owned.push_back((void *)*p);
    return ok;
  };
  auto release = [&]() {
    for (void *p : owned) cudaFree(p);
    owned.clear();
  };
  const size_t mat = (size_t)ncls * nn * nn;
  if (!alloc(&dU, sizeof(double) * mat) || !alloc(&dV, sizeof(double) * mat) || !alloc(&dk, sizeof(int) * ncls) ||
      !alloc(&drank, sizeof(int) * ncls) || !alloc(&dst, sizeof(int) * ncls)) {
    release();
    return fail(B200FMM_ERR_OOM, "compression scratch");
  }
  if (cudaMemset(dst, 0, sizeof(int) * ncls) != cudaSuccess) {
    release();
    return fail(B200FMM_ERR_CUDA, "compression scratch");
  }
  aca_kernel<<<ncls, CT>>>(nn, dA, eps * eps, dU, dV, dk, dst);
  std::vector<int> k(ncls), st(ncls);
  if (cudaGetLastError() != cudaSuccess || cudaMemcpy(st.data(), dst, sizeof(int) * ncls, cudaMemcpyDeviceToHost) ||
      cudaMemcpy(k.data(), dk, sizeof(int) * ncls, cudaMemcpyDeviceToHost)) {
    release();
    return fail(B200FMM_ERR_CUDA, "ACA kernel failed");
  }
  for (int s : st)
    if (s) {
      release();
      return fail(B200FMM_ERR_NUMERIC, "ACA breakdown (zero pivot)");
    }
  const int kmax = *std::max_element(k.begin(), k.end());
  const size_t sq = (size_t)ncls * kmax * kmax, tall = (size_t)ncls * 2 * kmax * nn;
  if (!alloc(&dH, sizeof(double) * tall) || !alloc(&dQ, sizeof(double) * tall) ||
      !alloc(&dR, sizeof(double) * 2 * sq) || !alloc(&dP, sizeof(double) * sq) || !alloc(&dVm, sizeof(double) * sq) ||
      !alloc(&dS, sizeof(double) * 2 * sq) || !alloc(&dout, sizeof(double) * tall)) {
    release();
    return fail(B200FMM_ERR_OOM, "compression scratch");
  }
  qr_kernel<<<dim3(ncls, 2), CT>>>(nn, kmax, dk, dU, dV, dH, dQ, dR);
  svd_kernel<<<ncls, CT>>>(nn, kmax, dk, eps, dR, dQ, dw, dP, dVm, dS, dout, drank, dst);
  std::vector<int> rk(ncls);
  if (cudaGetLastError() != cudaSuccess || cudaMemcpy(st.data(), dst, sizeof(int) * ncls, cudaMemcpyDeviceToHost) ||
      cudaMemcpy(rk.data(), drank, sizeof(int) * ncls, cudaMemcpyDeviceToHost)) {
    release();
    return fail(B200FMM_ERR_CUDA, "QR / SVD kernels failed");
  }
  for (int s : st)
    if (s) {
      release();
      return fail(B200FMM_ERR_NUMERIC, s == 2 ? "SVD did not converge" : "rank rule failed");
    }
  ranks = rk;
  uv.clear();
  for (int ci = 0; ci < ncls; ++ci) {
    const size_t off = uv.size(), n = (size_t)rk[ci] * nn;
    uv.resize(off + 2 * n);
    const double *src = dout + (size_t)ci * 2 * kmax * nn;
    if (cudaMemcpy(uv.data() + off, src, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(uv.data() + off + n, src + (size_t)kmax * nn, sizeof(double) * n, cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
      release();
      return fail(B200FMM_ERR_CUDA, "compression readback");
    }
  }
  release();
  return B200FMM_OK;
}

}  // namespace b200
