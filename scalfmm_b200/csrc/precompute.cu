// Interpolation tables and M2L operator precompute (FP64).
//
//  * nodes and 1-D interpolators: Chebyshev roots (Src/Kernels/Chebyshev/FChebRoots.hpp:31-36), equispaced
//    Lagrange roots (Src/Kernels/Uniform/FUnifRoots.hpp:35-39); child->parent interpolators
//    (FChebInterpolator::initTensorM2MandL2L, Src/Kernels/Chebyshev/FChebInterpolator.hpp:300-338).
//  * symmetric compression (Src/Kernels/Chebyshev/FChebSymM2LHandler.hpp:39-281): the weighted kernel
//    matrices of the 16 canonical transfer vectors are evaluated on the GPU and compressed there
//    (compress.cu: partially pivoted ACA, Householder QR of both factors, Jacobi SVD, rank rule), all in FP64.
//  * symmetry tables (Src/Kernels/Interpolation/FInterpSymmetries.hpp:18-125).
//  * dense per-transfer-vector operators K(X_m, Y_n) at reference width 2
//    (FChebDenseM2LHandler::Compute, Src/Kernels/Chebyshev/FChebDenseM2LHandler.hpp:178-215), evaluated on
//    the GPU.
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace b200 {

namespace {

void roots_for(int kernel, int p, double *r) {
  if (kernel == B200FMM_LAGRANGE) {
    for (int j = 0; j < p; ++j) r[j] = -1.0 + 2.0 * j / (double)(p - 1);
  } else {
    for (int j = 0; j < p; ++j) r[j] = -std::cos(M_PI * (2.0 * j + 1.0) / (2.0 * p));
  }
}

// 1-D basis S_j(x), j < p (Chebyshev: FChebInterpolator.hpp:466-485; Lagrange: FUnifRoots.hpp:49-83)
void basis_host(int kernel, int p, const double *roots, double x, double *S) {
  if (kernel == B200FMM_LAGRANGE) {
    for (int j = 0; j < p; ++j) {
      double v = 1.0;
      for (int m = 0; m < p; ++m)
        if (m != j) v *= (x - roots[m]) / (roots[j] - roots[m]);
      S[j] = v;
    }
    return;
  }
  double T[kMaxOrder];
  T[0] = 1.0;
  if (p > 1) T[1] = x;
  for (int o = 2; o < p; ++o) T[o] = 2.0 * x * T[o - 1] - T[o - 2];
  for (int j = 0; j < p; ++j) {
    double s = 1.0 / p;
    for (int o = 1; o < p; ++o) s += 2.0 / p * T[o] * std::cos(o * std::acos(roots[j]));
    S[j] = s;
  }
}

void build_itab(IListTable &t) {
  for (int c = 0; c < 8; ++c) {
    const int cb[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
    int k = 0;
    for (int px = -1; px <= 1; ++px)
      for (int py = -1; py <= 1; ++py)
        for (int pz = -1; pz <= 1; ++pz) {
          if (!(px || py || pz)) continue;
          for (int ch = 0; ch < 8; ++ch) {
            const int d[3] = {2 * px + ((ch >> 2) & 1) - cb[0], 2 * py + ((ch >> 1) & 1) - cb[1],
                              2 * pz + (ch & 1) - cb[2]};
            if (std::abs(d[0]) > 1 || std::abs(d[1]) > 1 || std::abs(d[2]) > 1) {
              for (int a = 0; a < 3; ++a) t.off[c][k][a] = (signed char)d[a];
              t.slot[c][k] = (short)(((d[0] + 3) * 7 + (d[1] + 3)) * 7 + (d[2] + 3));
              ++k;
            }
          }
        }
    t.n[c] = k;
  }
}

// FInterpSymmetries::getPermutationArrayAndIndex (FInterpSymmetries.hpp:102-125)
void sym_tables(int p, std::vector<int> &pind, std::vector<int> &pvec) {
  const int nn = p * p * p;
  pind.assign(343, 0);
  pvec.assign(343 * nn, 0);
  std::vector<int> quads(8 * nn), cones(8 * nn);
  for (int i = 0; i < p; ++i)
    for (int j = 0; j < p; ++j)
      for (int k = 0; k < p; ++k) {
        const int idx = k * p * p + j * p + i;
        for (int q = 0; q < 8; ++q) {
          const int ii = (q & 1) ? p - 1 - i : i, jj = (q & 2) ? p - 1 - j : j, kk = (q & 4) ? p - 1 - k : k;
          quads[q * nn + idx] = kk * p * p + jj * p + ii;
        }
        cones[0 * nn + idx] = k * p * p + j * p + i;
        cones[1 * nn + idx] = j * p * p + k * p + i;
        cones[3 * nn + idx] = j * p * p + i * p + k;
        cones[4 * nn + idx] = k * p * p + i * p + j;
        cones[6 * nn + idx] = i * p * p + k * p + j;
        cones[7 * nn + idx] = i * p * p + j * p + k;
      }
  static const int perms[8][3] = {{0, 1, 2}, {0, 2, 1}, {0, 0, 0}, {2, 0, 1}, {1, 0, 2}, {0, 0, 0}, {1, 2, 0}, {2, 1, 0}};
  for (int i = -3; i <= 3; ++i)
    for (int j = -3; j <= 3; ++j)
      for (int k = -3; k <= 3; ++k) {
        const int t = ((i + 3) * 7 + (j + 3)) * 7 + (k + 3);
        if (!(std::abs(i) > 1 || std::abs(j) > 1 || std::abs(k) > 1)) continue;
        const int q = (i < 0 ? 1 : 0) | (j < 0 ? 2 : 0) | (k < 0 ? 4 : 0);
        const int u[3] = {std::abs(i), std::abs(j), std::abs(k)};
        const int cidx = ((u[1] > u[0]) << 2) | ((u[2] > u[0]) << 1) | (u[2] > u[1]);
        for (int n = 0; n < nn; ++n) pvec[t * nn + n] = cones[cidx * nn + quads[q * nn + n]];
        pind[t] = (u[perms[cidx][0]] + 3) * 49 + (u[perms[cidx][1]] + 3) * 7 + (u[perms[cidx][2]] + 3);
      }
}

// ---- GPU kernel evaluation -------------------------------------------------------------------------

// Weighted kernel matrices of the 16 class slots: A[c][t][s] = w_t w_s / |X_t - Y_s|, X = nodes of the
// width-2 cell at the origin, Y = nodes of the width-2 cell centred at 2*(i,j,k).
__global__ void eval_weighted_classes(int p, const double *__restrict__ roots, const int *__restrict__ cls,
                                      const double *__restrict__ w, double *__restrict__ A) {
  const int nn = p * p * p;
  const int c = blockIdx.y;
  const int slot = cls[c];
  const int ci = slot / 49 - 3, cj = (slot / 7) % 7 - 3, ck = slot % 7 - 3;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)nn * nn) return;
  const int t = (int)(e / nn), s = (int)(e % nn);
  const double dx = roots[t % p] - (2.0 * ci + roots[s % p]);
  const double dy = roots[(t / p) % p] - (2.0 * cj + roots[(s / p) % p]);
  const double dz = roots[t / (p * p)] - (2.0 * ck + roots[s / (p * p)]);
  A[(long long)c * nn * nn + e] = w[t] * w[s] * (1.0 / sqrt(dx * dx + dy * dy + dz * dz));
}

// Dense operators for every far slot: K[t][n][m] = 1/|X_m - Y_n| (zero for the 27 near slots).
__global__ void eval_dense(int p, const double *__restrict__ roots, double *__restrict__ K) {
  const int nn = p * p * p;
  const int t = blockIdx.y;
  const int i = t / 49 - 3, j = (t / 7) % 7 - 3, k = t % 7 - 3;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)nn * nn) return;
  double v = 0.0;
  if (abs(i) > 1 || abs(j) > 1 || abs(k) > 1) {
    const int n = (int)(e / nn), m = (int)(e % nn);  // stored [t][n][m]: coalesced over the target node m
    const double dx = roots[m % p] - (2.0 * i + roots[n % p]);
    const double dy = roots[(m / p) % p] - (2.0 * j + roots[(n / p) % p]);
    const double dz = roots[m / (p * p)] - (2.0 * k + roots[n / (p * p)]);
    v = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
  }
  K[(long long)t * nn * nn + e] = v;
}

}  // namespace

b200fmm_status build_tables(Context &c) {
  const int p = c.p;
  std::vector<double> roots(p), Tr(p * p), S(8 * 3 * p * p);
  roots_for(c.cfg.kernel, p, roots.data());
  for (int o = 0; o < p; ++o)
    for (int j = 0; j < p; ++j) Tr[o * p + j] = std::cos(o * std::acos(roots[j]));
  for (int ch = 0; ch < 8; ++ch) {
    const double sg[3] = {(ch >> 2) & 1 ? 0.5 : -0.5, (ch >> 1) & 1 ? 0.5 : -0.5, ch & 1 ? 0.5 : -0.5};
    for (int d = 0; d < 3; ++d)
      for (int m = 0; m < p; ++m) {
        double w[kMaxOrder];
        basis_host(c.cfg.kernel, p, roots.data(), sg[d] + 0.5 * roots[m], w);
        for (int n = 0; n < p; ++n) S[((ch * 3 + d) * p + n) * p + m] = w[n];
      }
  }
  B200_CUDA(cudaMalloc(&c.d_roots, sizeof(double) * p));
  B200_CUDA(cudaMalloc(&c.d_S, sizeof(double) * S.size()));
  B200_CUDA(cudaMemcpy(c.d_roots, roots.data(), sizeof(double) * p, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_S, S.data(), sizeof(double) * S.size(), cudaMemcpyHostToDevice));
  B200_CHECK(upload_basis_constants(c, roots.data(), Tr.data()));
  build_itab(c.itab);
  B200_CUDA(cudaMalloc(&c.d_itab, sizeof(IListTable)));
  B200_CUDA(cudaMemcpy(c.d_itab, &c.itab, sizeof(IListTable), cudaMemcpyHostToDevice));
  return B200FMM_OK;
}

b200fmm_status compress_sym_operators(Context &c) {
  const int p = c.p, nn = c.nn;
  const double eps = c.cfg.epsilon > 0 ? c.cfg.epsilon : std::pow(10.0, -p);
  std::vector<double> roots(p);
  roots_for(B200FMM_CHEB_SYM, p, roots.data());
  // root of the tensor Chebyshev weights (FChebTensor::setRootOfWeights, FChebTensor.hpp:42-55)
  std::vector<double> w1(p), w(nn);
  for (int o = 0; o < p; ++o) w1[o] = M_PI / p * std::sqrt(1.0 - roots[o] * roots[o]);
  for (int n = 0; n < nn; ++n) w[n] = std::sqrt(w1[n % p] * w1[(n / p) % p] * w1[n / (p * p)]);
  std::vector<int> cls;
  for (int i = 2; i <= 3; ++i)
    for (int j = 0; j <= i; ++j)
      for (int k = 0; k <= j; ++k) cls.push_back((i + 3) * 49 + (j + 3) * 7 + (k + 3));
  const int ncls = (int)cls.size();
  double *dA = nullptr, *dr = nullptr, *dw = nullptr;
  int *dc = nullptr;
  B200_CUDA(cudaMalloc(&dA, sizeof(double) * ncls * nn * nn));
  B200_CUDA(cudaMalloc(&dr, sizeof(double) * p));
  B200_CUDA(cudaMalloc(&dw, sizeof(double) * nn));
  B200_CUDA(cudaMalloc(&dc, sizeof(int) * ncls));
  B200_CUDA(cudaMemcpy(dr, roots.data(), sizeof(double) * p, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(dw, w.data(), sizeof(double) * nn, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(dc, cls.data(), sizeof(int) * ncls, cudaMemcpyHostToDevice));
  eval_weighted_classes<<<dim3(grid_for((long long)nn * nn, 256), ncls), 256>>>(p, dr, dc, dw, dA);
  b200fmm_status st = cudaGetLastError() == cudaSuccess ? B200FMM_OK : fail(B200FMM_ERR_CUDA, "class matrices");
  std::vector<int> ranks;
  if (st == B200FMM_OK) st = compress_classes(c, ncls, dA, dw, eps, ranks, c.sym_uv);
  cudaFree(dA);
  cudaFree(dr);
  cudaFree(dw);
  cudaFree(dc);
  if (st != B200FMM_OK) return st;
  c.sym_ranks.assign(343, 0);
  for (int ci = 0; ci < ncls; ++ci) c.sym_ranks[cls[ci]] = ranks[ci];
  return B200FMM_OK;
}

// the class slot and node permutation of every slot (sym_tables), for the other files of the library
void slot_symmetry_tables(int p, std::vector<int> &pind, std::vector<int> &pvec) { sym_tables(p, pind, pvec); }

// Per-slot permuted factors on the host: Ut[t][n][a] = U_c[pvec_t[n]][a], Vt[t][m][a] = V_c[pvec_t[m]][a]
// (row-major p^3 x r, r = rank of the slot's class), at toff[t] for every far slot t (-1 for near slots).
b200fmm_status sym_slot_factors(const Context &c, std::vector<double> &Ut, std::vector<double> &Vt,
                                std::vector<long long> &toff, std::vector<int> &trank) {
  const int nn = c.nn;
  std::vector<int> pind, pvec;
  sym_tables(c.p, pind, pvec);
  std::vector<long long> off(343, -1);
  std::vector<int> rk(343, 0);
  long long o = 0, used = 0;
  for (int t = 0; t < 343; ++t)
    if (c.sym_ranks[t] > 0) {
      off[t] = o;
      rk[t] = c.sym_ranks[t];
      o += (long long)rk[t] * nn;
    }
  // every far slot must map to a class slot that has an operator
  for (int t = 0; t < 343; ++t) {
    const int i = t / 49 - 3, j = (t / 7) % 7 - 3, k = t % 7 - 3;
    if ((std::abs(i) > 1 || std::abs(j) > 1 || std::abs(k) > 1) && rk[pind[t]] == 0)
      return fail(B200FMM_ERR_INVALID, "symmetric operators: a class slot has rank 0");
  }
  std::vector<double> U(o), V(o);
  for (int t = 0; t < 343; ++t)
    if (rk[t] > 0) {
      const double *src = c.sym_uv.data() + used;
      std::memcpy(U.data() + off[t], src, sizeof(double) * rk[t] * nn);
      std::memcpy(V.data() + off[t], src + (size_t)rk[t] * nn, sizeof(double) * rk[t] * nn);
      used += 2LL * rk[t] * nn;
    }
  toff.assign(343, -1);
  trank.assign(343, 0);
  long long tot = 0;
  for (int t = 0; t < 343; ++t) {
    const int i = t / 49 - 3, j = (t / 7) % 7 - 3, k = t % 7 - 3;
    if (!(std::abs(i) > 1 || std::abs(j) > 1 || std::abs(k) > 1)) continue;
    toff[t] = tot;
    trank[t] = rk[pind[t]];
    tot += (long long)trank[t] * nn;
  }
  Ut.assign(tot, 0.0);
  Vt.assign(tot, 0.0);
  for (int t = 0; t < 343; ++t) {
    if (toff[t] < 0) continue;
    const int cls = pind[t], r = trank[t];
    const double *Uc = U.data() + off[cls], *Vc = V.data() + off[cls];  // [a][j] = U_c[j][a]
    const int *pv = pvec.data() + (size_t)t * nn;
    for (int n = 0; n < nn; ++n)
      for (int a = 0; a < r; ++a) {
        Ut[toff[t] + (size_t)n * r + a] = Uc[(size_t)a * nn + pv[n]];
        Vt[toff[t] + (size_t)n * r + a] = Vc[(size_t)a * nn + pv[n]];
      }
  }
  return B200FMM_OK;
}

b200fmm_status upload_sym_operators(Context &c) {
  const int nn = c.nn;
  std::vector<int> pind, pvec;
  sym_tables(c.p, pind, pvec);
  std::vector<long long> off(343, -1);
  std::vector<int> rk(343, 0);
  long long o = 0, used = 0;
  c.max_rank = 0;
  for (int t = 0; t < 343; ++t)
    if (c.sym_ranks[t] > 0) {
      off[t] = o;
      rk[t] = c.sym_ranks[t];
      o += (long long)rk[t] * nn;
      c.max_rank = std::max(c.max_rank, rk[t]);
    }
  // every far slot must map to a class slot that has an operator
  for (int t = 0; t < 343; ++t) {
    const int i = t / 49 - 3, j = (t / 7) % 7 - 3, k = t % 7 - 3;
    if ((std::abs(i) > 1 || std::abs(j) > 1 || std::abs(k) > 1) && rk[pind[t]] == 0)
      return fail(B200FMM_ERR_INVALID, "symmetric operators: a class slot has rank 0");
  }
  std::vector<double> U(o), V(o);
  for (int t = 0; t < 343; ++t)
    if (rk[t] > 0) {
      const double *src = c.sym_uv.data() + used;
      std::memcpy(U.data() + off[t], src, sizeof(double) * rk[t] * nn);
      std::memcpy(V.data() + off[t], src + (size_t)rk[t] * nn, sizeof(double) * rk[t] * nn);
      used += 2LL * rk[t] * nn;
    }
  for (void *p : {(void *)c.d_pindices, (void *)c.d_pvec, (void *)c.d_symU, (void *)c.d_symV, (void *)c.d_symoff,
                  (void *)c.d_symrank, (void *)c.d_Ut, (void *)c.d_Vt, (void *)c.d_toff, (void *)c.d_trank})
    if (p) cudaFree(p);
  // per-slot permuted factors (FChebSymKernel::M2L applies the permutation around the class operator;
  // folding it into the factors once gives plain per-slot operators)
  std::vector<long long> toff;
  std::vector<int> trank;
  std::vector<double> Ut, Vt;
  B200_CHECK(sym_slot_factors(c, Ut, Vt, toff, trank));
  const long long tot = (long long)Ut.size();
  B200_CUDA(cudaMalloc(&c.d_Ut, sizeof(double) * std::max<long long>(tot, 1)));
  B200_CUDA(cudaMalloc(&c.d_Vt, sizeof(double) * std::max<long long>(tot, 1)));
  B200_CUDA(cudaMalloc(&c.d_toff, sizeof(long long) * 343));
  B200_CUDA(cudaMalloc(&c.d_trank, sizeof(int) * 343));
  B200_CUDA(cudaMemcpy(c.d_Ut, Ut.data(), sizeof(double) * tot, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_Vt, Vt.data(), sizeof(double) * tot, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_toff, toff.data(), sizeof(long long) * 343, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_trank, trank.data(), sizeof(int) * 343, cudaMemcpyHostToDevice));
  B200_CHECK(sym64_prepare(c, c.d_Ut, c.d_Vt, toff, trank));
  B200_CUDA(cudaMalloc(&c.d_pindices, sizeof(int) * 343));
  B200_CUDA(cudaMalloc(&c.d_pvec, sizeof(int) * 343 * nn));
  B200_CUDA(cudaMalloc(&c.d_symU, sizeof(double) * std::max<long long>(o, 1)));
  B200_CUDA(cudaMalloc(&c.d_symV, sizeof(double) * std::max<long long>(o, 1)));
  B200_CUDA(cudaMalloc(&c.d_symoff, sizeof(long long) * 343));
  B200_CUDA(cudaMalloc(&c.d_symrank, sizeof(int) * 343));
  B200_CUDA(cudaMemcpy(c.d_pindices, pind.data(), sizeof(int) * 343, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_pvec, pvec.data(), sizeof(int) * 343 * nn, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_symU, U.data(), sizeof(double) * o, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_symV, V.data(), sizeof(double) * o, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_symoff, off.data(), sizeof(long long) * 343, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_symrank, rk.data(), sizeof(int) * 343, cudaMemcpyHostToDevice));
  // per child type, the interaction-list entries ordered by symmetry class (the reference batches the
  // M2L of one target by class, FChebSymKernel.hpp:216-285)
  std::vector<int> order(8 * 189);
  for (int ct = 0; ct < 8; ++ct) {
    std::vector<int> e(189);
    for (int k = 0; k < 189; ++k) e[k] = k;
    std::stable_sort(e.begin(), e.end(),
                     [&](int a, int b) { return pind[c.itab.slot[ct][a]] < pind[c.itab.slot[ct][b]]; });
    for (int k = 0; k < 189; ++k) order[ct * 189 + k] = e[k];
  }
  std::vector<int> bounds(8 * 17, 0);  // [child type][class ordinal 0..16] start offsets into the order
  std::vector<int> cls_slots;
  for (int t = 0; t < 343; ++t)
    if (rk[t] > 0) cls_slots.push_back(t);
  for (int ct = 0; ct < 8; ++ct) {
    int k = 0;
    for (int ci = 0; ci < (int)cls_slots.size() && ci < 16; ++ci) {
      bounds[ct * 17 + ci] = k;
      while (k < 189 && pind[c.itab.slot[ct][order[ct * 189 + k]]] == cls_slots[ci]) ++k;
    }
    bounds[ct * 17 + 16] = k;
    if (k != 189) return fail(B200FMM_ERR_INVALID, "symmetric operators: class table mismatch");
  }
  if (c.d_class_order) cudaFree(c.d_class_order);
  if (c.d_cls_bounds) cudaFree(c.d_cls_bounds);
  B200_CUDA(cudaMalloc(&c.d_class_order, sizeof(int) * 8 * 189));
  B200_CUDA(cudaMalloc(&c.d_cls_bounds, sizeof(int) * 8 * 17));
  B200_CUDA(cudaMemcpy(c.d_class_order, order.data(), sizeof(int) * 8 * 189, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(c.d_cls_bounds, bounds.data(), sizeof(int) * 8 * 17, cudaMemcpyHostToDevice));
  c.cls_slots = cls_slots;
  if (c.d_cls_slots) cudaFree(c.d_cls_slots);
  B200_CUDA(cudaMalloc(&c.d_cls_slots, sizeof(int) * 16));
  B200_CUDA(cudaMemcpy(c.d_cls_slots, cls_slots.data(), sizeof(int) * 16, cudaMemcpyHostToDevice));
  return B200FMM_OK;
}

b200fmm_status build_dense_operators(Context &c) {
  const int nn = c.nn;
  if (c.d_dense) return B200FMM_OK;
  B200_CUDA(cudaMalloc(&c.d_dense, sizeof(double) * 343 * (size_t)nn * nn));
  eval_dense<<<dim3(grid_for((long long)nn * nn, 256), 343), 256>>>(c.p, c.d_roots, c.d_dense);
  B200_CUDA(cudaGetLastError());
  B200_CUDA(cudaDeviceSynchronize());
  return B200FMM_OK;
}

}  // namespace b200
