// FP64 M2L for the symmetric Chebyshev operators (parity form), as two dense FP64 GEMMs per level.
//
// FChebSymKernel::M2L (Src/Kernels/Chebyshev/FChebSymKernel.hpp:210-328) applies, for each target and each of
// its <= 189 far neighbours at transfer vector t, the compressed operator of t's symmetry class through t's
// permutation: L += scale * P_t^T U_c V_c^T P_t M.  With the permutation folded into per-slot factors
// U_t = P_t^T U_c, V_t = P_t^T V_c (precompute.cu), the product splits into
//   Y_t(s) = V_t^T M_s        -- depends on the source cell s and the slot only,
//   L(c)  += scale * sum_t U_t Y_t(c + d_t).
// Both halves are dense GEMMs with FP64 operands and FP64 accumulation:
//   * phase 1, per source parity sp: every slot that cells of parity sp feed (as sources of some target) is
//     stacked into one operator Vs_sp = [V_t^T]_t (sum of ranks ~ 4,200 rows at order 7, K = p^3); one GEMM
//     Y = Vs_sp * [M_s]_s over all cells of that parity gives every Y_t(s) the level needs;
//   * phase 2, per child type ct (the target parity, which fixes the 189 transfer vectors and their order):
//     Uc_ct = [U_t]_e concatenated along the rank (K ~ 4,200), and L(c) += scale * Uc_ct * [Y_t(s_e(c))]_e with
//     the B operand gathered through the interaction list (a missing source contributes zero).
// Each output element is computed by one thread over the whole K range in a fixed order, so results do not
// depend on the work order.  The reference sums the same products in a different order; the tests hold the
// two to 1e-12 relative.
#include "common.cuh"

#include <algorithm>
#include <cmath>

namespace b200 {

struct Sym64 {
  int ysum[8] = {0};                 // rows of Vs_sp (sum of the ranks of the slots parity sp feeds)
  long long vs_off[8] = {0};         // element offset of Vs_sp in d_vs
  int kct[8] = {0};                  // K of Uc_ct
  long long uc_off[8] = {0};         // element offset of Uc_ct in d_uc
  long long km_off[8] = {0};         // entry offset of ct's K map in d_kmap
  int ystride = 0;                   // max ysum (row stride of Y)
  double *d_vs = nullptr;            // [sp][ysum][nn] row-major
  double *d_uc = nullptr;            // [ct][nn][kct] row-major
  int2 *d_kmap = nullptr;            // [ct][kct]: (interaction-list entry e, row of Y)
  // per tree
  long long list_serial = -1;
  int *d_plist = nullptr;            // cells of every level grouped by parity
  int *d_pcnt = nullptr;             // [kMaxHeight][8] counts, then [kMaxHeight][8] cursors
  long long *h_loff = nullptr;       // host: first list entry of each level
  size_t cap_list = 0;
  double *d_y = nullptr;             // [ncells][ystride] of the level in work
  size_t cap_y = 0;
};

namespace {

constexpr int G_BM = 128, G_BN = 128, G_BK = 8, G_THREADS = 256;
constexpr int G_TM = 8, G_TN = 8;  // outputs per thread: rows ty*8 + i, columns tx + 16 j

// cells of levels 2..LL grouped by parity (child type = key & 7): counts, then placement with per-parity cursors
struct ListArgs {
  const long long *keys[kMaxHeight];
  long long n[kMaxHeight];
  long long loff[kMaxHeight];
  int l0, l1;
};

__global__ void parity_count_kernel(const __grid_constant__ ListArgs a, int *__restrict__ cnt) {
  for (int l = a.l0; l <= a.l1; ++l)
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n[l];
         i += (long long)gridDim.x * blockDim.x)
      atomicAdd(cnt + l * 8 + (int)(a.keys[l][i] & 7), 1);
}

__global__ void parity_place_kernel(const __grid_constant__ ListArgs a, int *__restrict__ cnt, int *__restrict__ list) {
  for (int l = a.l0; l <= a.l1; ++l) {
    int base[8];
    int s = 0;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      base[p] = s;
      s += cnt[l * 8 + p];
    }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n[l];
         i += (long long)gridDim.x * blockDim.x) {
      const int p = (int)(a.keys[l][i] & 7);
      const int k = atomicAdd(cnt + kMaxHeight * 8 + l * 8 + p, 1);
      list[a.loff[l] + base[p] + k] = (int)i;
    }
  }
}

struct GemmArgs {
  int nn, R, rhs, ystride;
  double scale;
  const int *list;       // this level's cells grouped by parity
  const int *cnt;        // [8] cells per parity at this level
  // phase 1
  const double *vs;      // Vs_sp at vs + vs_off[sp]
  long long vs_off[8];
  int ysum[8];
  const double *M;       // [ncells][R][nn]
  double *Y;             // [ncells][ystride]
  // phase 2
  const double *uc;      // Uc_ct at uc + uc_off[ct]
  long long uc_off[8];
  int kct[8];
  const int2 *kmap;
  long long km_off[8];
  const int *ilist;      // [ncells][189]
  double *L;             // [ncells][R][nn]
};

// One 128 x 128 tile of C = A B over K, A row-major [M][K] (ld = K), B delivered by the caller's loader.
// The K loop keeps two shared-memory stages; the next stage's values are loaded into registers while the
// current one is multiplied.
template <class LoadB>
__device__ __forceinline__ void gemm_tile(const double *__restrict__ A, int Mrows, int K, int m0, LoadB loadB,
                                          double (&acc)[G_TM][G_TN], double (*As)[G_BK][G_BM],
                                          double (*Bs)[G_BK][G_BN]) {
  const int t = threadIdx.x;
  const int tx = t & 15, ty = t >> 4;
  // loaders: A row am = t / 2, k = (t & 1) * 4 + 0..3; B column bn = t & 127, k = (t >> 7) * 4 + 0..3
  const int am = t >> 1, ak = (t & 1) * 4;
  const int bn = t & 127, bk = (t >> 7) * 4;
  const bool arow = m0 + am < Mrows;
  const double *Arow = A + (long long)(m0 + am) * K;
  double ra[4], rb[4];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = k0 + ak + u;
      ra[u] = (arow && k < K) ? __ldg(Arow + k) : 0.0;
    }
    loadB(k0 + bk, bn, rb);
  };
  auto store = [&](int s) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      As[s][ak + u][am] = ra[u];
      Bs[s][bk + u][bn] = rb[u];
    }
  };
#pragma unroll
  for (int i = 0; i < G_TM; ++i)
#pragma unroll
    for (int j = 0; j < G_TN; ++j) acc[i][j] = 0.0;
  const int nk = (K + G_BK - 1) / G_BK;
  fetch(0);
  store(0);
  __syncthreads();
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt & 1;
    if (kt + 1 < nk) fetch((kt + 1) * G_BK);
#pragma unroll
    for (int k = 0; k < G_BK; ++k) {
      double a[G_TM], b[G_TN];
#pragma unroll
      for (int i = 0; i < G_TM; ++i) a[i] = As[s][k][ty * G_TM + i];
#pragma unroll
      for (int j = 0; j < G_TN; ++j) b[j] = Bs[s][k][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < G_TM; ++i)
#pragma unroll
        for (int j = 0; j < G_TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (kt + 1 < nk) store(s ^ 1);
    __syncthreads();
  }
}

// Phase 1, persistent over items (parity, cell tile, row tile): Y[cell][m] = sum_k Vs_sp[m][k] M[cell][rhs][k].
__global__ void __launch_bounds__(G_THREADS, 1) sym64_y_kernel(const __grid_constant__ GemmArgs a) {
  __shared__ __align__(16) double As[2][G_BK][G_BM];
  __shared__ __align__(16) double Bs[2][G_BK][G_BN];
  int nt[8], mt[8], first[9];
  int cstart[8];
  first[0] = 0;
  int s = 0;
  for (int p = 0; p < 8; ++p) {
    cstart[p] = s;
    s += a.cnt[p];
    nt[p] = (a.cnt[p] + G_BN - 1) / G_BN;
    mt[p] = (a.ysum[p] + G_BM - 1) / G_BM;
    first[p + 1] = first[p] + nt[p] * mt[p];
  }
  for (int item = blockIdx.x; item < first[8]; item += gridDim.x) {
    int p = 0;
    while (item >= first[p + 1]) ++p;
    const int r = item - first[p];
    const int m0 = (r % mt[p]) * G_BM, n0 = (r / mt[p]) * G_BN;
    const int ncol = min(G_BN, a.cnt[p] - n0);
    const int *cells = a.list + cstart[p] + n0;
    auto loadB = [&](int k, int n, double (&v)[4]) {
      const bool ok = n < ncol;
      const double *Mc = ok ? a.M + ((long long)cells[n] * a.R + a.rhs) * a.nn : a.M;
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = (ok && k + u < a.nn) ? __ldg(Mc + k + u) : 0.0;
    };
    double acc[G_TM][G_TN];
    gemm_tile(a.vs + a.vs_off[p], a.ysum[p], a.nn, m0, loadB, acc, As, Bs);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int j = 0; j < G_TN; ++j) {
      const int n = tx + 16 * j;
      if (n >= ncol) continue;
      double *Yc = a.Y + (long long)cells[n] * a.ystride;
#pragma unroll
      for (int i = 0; i < G_TM; ++i) {
        const int m = m0 + ty * G_TM + i;
        if (m < a.ysum[p]) Yc[m] = acc[i][j];
      }
    }
  }
}

// Phase 2, persistent over items (child type, target tile, node tile):
// L[c][rhs][m] += scale * sum_k Uc_ct[m][k] Y[ilist[c][e_k]][row_k].
__global__ void __launch_bounds__(G_THREADS, 1) sym64_l_kernel(const __grid_constant__ GemmArgs a) {
  __shared__ __align__(16) double As[2][G_BK][G_BM];
  __shared__ __align__(16) double Bs[2][G_BK][G_BN];
  int nt[8], first[9], cstart[8];
  const int mt = (a.nn + G_BM - 1) / G_BM;
  first[0] = 0;
  int s = 0;
  for (int p = 0; p < 8; ++p) {
    cstart[p] = s;
    s += a.cnt[p];
    nt[p] = (a.cnt[p] + G_BN - 1) / G_BN;
    first[p + 1] = first[p] + nt[p] * mt;
  }
  for (int item = blockIdx.x; item < first[8]; item += gridDim.x) {
    int ct = 0;
    while (item >= first[ct + 1]) ++ct;
    const int r = item - first[ct];
    const int m0 = (r % mt) * G_BM, n0 = (r / mt) * G_BN;
    const int ncol = min(G_BN, a.cnt[ct] - n0);
    const int *cells = a.list + cstart[ct] + n0;
    const int2 *km = a.kmap + a.km_off[ct];
    const int K = a.kct[ct];
    auto loadB = [&](int k, int n, double (&v)[4]) {
      const int *il = n < ncol ? a.ilist + (long long)cells[n] * 189 : nullptr;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        v[u] = 0.0;
        if (il && k + u < K) {
          const int2 e = km[k + u];
          const int src = il[e.x];
          if (src >= 0) v[u] = a.Y[(long long)src * a.ystride + e.y];
        }
      }
    };
    double acc[G_TM][G_TN];
    gemm_tile(a.uc + a.uc_off[ct], a.nn, K, m0, loadB, acc, As, Bs);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int j = 0; j < G_TN; ++j) {
      const int n = tx + 16 * j;
      if (n >= ncol) continue;
      double *Lc = a.L + ((long long)cells[n] * a.R + a.rhs) * a.nn;
#pragma unroll
      for (int i = 0; i < G_TM; ++i) {
        const int m = m0 + ty * G_TM + i;
        if (m < a.nn) Lc[m] += a.scale * acc[i][j];
      }
    }
  }
}

// out[row][m] = Vt[foff + m * rank + q] for the row's (foff, rank, q)
__global__ void gather_vs_kernel(long long nrows, int nn, const int3 *__restrict__ rows, const double *__restrict__ Vt,
                                 double *__restrict__ out) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= nrows * nn) return;
  const int3 r = rows[g / nn];
  out[g] = Vt[r.x + (long long)(g % nn) * r.y + r.z];
}
// out[m][k] = Ut[foff + m * rank + q] for column k's (foff, rank, q)
__global__ void gather_uc_kernel(int K, int nn, const int3 *__restrict__ cols, const double *__restrict__ Ut,
                                 double *__restrict__ out) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= (long long)nn * K) return;
  const int k = (int)(g % K), m = (int)(g / K);
  const int3 col = cols[k];
  out[g] = Ut[col.x + (long long)m * col.y + col.z];
}

int sm_count(const Context &c) {
  int v = 148;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, c.device);
  return v > 0 ? v : 148;
}

}  // namespace

void sym64_free(Context &c) {
  Sym64 *s = c.s64;
  if (!s) return;
  for (void *p : {(void *)s->d_vs, (void *)s->d_uc, (void *)s->d_kmap, (void *)s->d_plist, (void *)s->d_pcnt,
                  (void *)s->d_y})
    if (p) cudaFree(p);
  delete[] s->h_loff;
  delete s;
  c.s64 = nullptr;
}

// The stacked operators of both phases, gathered on the device from the per-slot factors (d_Ut, d_Vt: row-major
// p^3 x r each, at the slot's offset toff).
b200fmm_status sym64_prepare(Context &c, const double *d_Ut, const double *d_Vt, const std::vector<long long> &toff,
                             const std::vector<int> &trank) {
  sym64_free(c);
  Sym64 *s = new Sym64();
  s->h_loff = new long long[kMaxHeight]();
  c.s64 = s;
  const int nn = c.nn;
  // the slots each source parity feeds: entry e of child type ct reads the cell at offset itab.off[ct][e],
  // whose parity is ct's parity plus that offset, per axis
  std::vector<int> ybase(8 * 343, -1);
  long long vs_total = 0;
  for (int sp = 0; sp < 8; ++sp) {
    std::vector<char> fed(343, 0);
    for (int ct = 0; ct < 8; ++ct)
      for (int e = 0; e < c.itab.n[ct]; ++e) {
        const int px = (((ct >> 2) & 1) + c.itab.off[ct][e][0]) & 1, py = (((ct >> 1) & 1) + c.itab.off[ct][e][1]) & 1,
                  pz = ((ct & 1) + c.itab.off[ct][e][2]) & 1;
        if (((px << 2) | (py << 1) | pz) == sp) fed[c.itab.slot[ct][e]] = 1;
      }
    int rows = 0;
    for (int t = 0; t < 343; ++t)
      if (fed[t]) {
        if (toff[t] < 0) return fail(B200FMM_ERR_INVALID, "symmetric operators: a far slot has no factor");
        ybase[sp * 343 + t] = rows;
        rows += trank[t];
      }
    s->ysum[sp] = rows;
    s->vs_off[sp] = vs_total;
    vs_total += (long long)rows * nn;
    s->ystride = std::max(s->ystride, rows);
  }
  // rows of the stacked V (gathered on the device): row (sp, ybase + q) is column q of V_t
  std::vector<int3> vrows((size_t)(vs_total / nn));
  for (int sp = 0; sp < 8; ++sp)
    for (int t = 0; t < 343; ++t) {
      const int b = ybase[sp * 343 + t];
      if (b < 0) continue;
      for (int q = 0; q < trank[t]; ++q)
        vrows[(size_t)(s->vs_off[sp] / nn) + b + q] = make_int3((int)toff[t], trank[t], q);
    }
  long long uc_total = 0, km_total = 0;
  for (int ct = 0; ct < 8; ++ct) {
    int K = 0;
    for (int e = 0; e < c.itab.n[ct]; ++e) K += trank[c.itab.slot[ct][e]];
    s->kct[ct] = K;
    s->uc_off[ct] = uc_total;
    s->km_off[ct] = km_total;
    uc_total += (long long)K * nn;
    km_total += K;
  }
  // columns of the concatenated U (gathered on the device): column k of Uc_ct is column q of U_t of entry e
  std::vector<int3> ucols((size_t)km_total);
  std::vector<int2> km((size_t)km_total);
  for (int ct = 0; ct < 8; ++ct) {
    int k = 0;
    for (int e = 0; e < c.itab.n[ct]; ++e) {
      const int t = c.itab.slot[ct][e], r = trank[t];
      const int px = (((ct >> 2) & 1) + c.itab.off[ct][e][0]) & 1, py = (((ct >> 1) & 1) + c.itab.off[ct][e][1]) & 1,
                pz = ((ct & 1) + c.itab.off[ct][e][2]) & 1;
      const int yb = ybase[((px << 2) | (py << 1) | pz) * 343 + t];
      for (int q = 0; q < r; ++q, ++k) {
        km[(size_t)s->km_off[ct] + k] = make_int2(e, yb + q);
        ucols[(size_t)s->km_off[ct] + k] = make_int3((int)toff[t], r, q);
      }
    }
  }
  int3 *d_vrows = nullptr, *d_ucols = nullptr;
  B200_CUDA(cudaMalloc(&s->d_vs, sizeof(double) * std::max<long long>(vs_total, 1)));
  B200_CUDA(cudaMalloc(&s->d_uc, sizeof(double) * std::max<long long>(uc_total, 1)));
  B200_CUDA(cudaMalloc(&s->d_kmap, sizeof(int2) * std::max<long long>(km_total, 1)));
  B200_CUDA(cudaMalloc(&s->d_pcnt, sizeof(int) * 2 * kMaxHeight * 8));
  B200_CUDA(cudaMalloc(&d_vrows, sizeof(int3) * std::max<size_t>(vrows.size(), 1)));
  B200_CUDA(cudaMalloc(&d_ucols, sizeof(int3) * std::max<size_t>(ucols.size(), 1)));
  B200_CUDA(cudaMemcpy(s->d_kmap, km.data(), sizeof(int2) * km_total, cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(d_vrows, vrows.data(), sizeof(int3) * vrows.size(), cudaMemcpyHostToDevice));
  B200_CUDA(cudaMemcpy(d_ucols, ucols.data(), sizeof(int3) * ucols.size(), cudaMemcpyHostToDevice));
  gather_vs_kernel<<<grid_for(vs_total, 256), 256>>>((long long)vrows.size(), nn, d_vrows, d_Vt, s->d_vs);
  for (int ct = 0; ct < 8; ++ct)
    if (s->kct[ct] > 0)
      gather_uc_kernel<<<grid_for((long long)nn * s->kct[ct], 256), 256>>>(s->kct[ct], nn, d_ucols + s->km_off[ct],
                                                                         d_Ut, s->d_uc + s->uc_off[ct]);
  B200_CUDA(cudaGetLastError());
  B200_CUDA(cudaDeviceSynchronize());
  cudaFree(d_vrows);
  cudaFree(d_ucols);
  return B200FMM_OK;
}

bool sym64_fed_ranks(const Context &c, double *fed) {
  if (!c.s64) return false;
  for (int p = 0; p < 8; ++p) fed[p] = c.s64->ysum[p];
  return true;
}

// Parity lists of the current tree (once per tree) and room for Y of the largest level.  Returns
// B200FMM_ERR_UNSUPPORTED when Y of that level would exceed the cap, so that the caller keeps the per-target
// kernel.
static b200fmm_status sym64_tree(Context &c) {
  Sym64 &s = *c.s64;
  const int LL = c.H - 1;
  long long total = 0, nmax = 0;
  ListArgs la{};
  la.l0 = 2;
  la.l1 = LL;
  for (int l = 2; l <= LL; ++l) {
    la.keys[l] = c.lv[l].keys;
    la.n[l] = c.lv[l].n;
    la.loff[l] = total;
    s.h_loff[l] = total;
    total += c.lv[l].n;
    nmax = std::max(nmax, c.lv[l].n);
  }
  const size_t ybytes = sizeof(double) * (size_t)nmax * s.ystride;
  if (ybytes > (size_t)16 << 30) return fail(B200FMM_ERR_UNSUPPORTED, "FP64 M2L: Y of the largest level exceeds 16 GiB");
  if (s.list_serial == c.tree_serial) return B200FMM_OK;
  if (s.cap_list < (size_t)total) {
    if (s.d_plist) cudaFree(s.d_plist);
    s.d_plist = nullptr;
    s.cap_list = 0;
    B200_CUDA(cudaMalloc(&s.d_plist, sizeof(int) * std::max<long long>(total, 1)));
    s.cap_list = (size_t)total;
  }
  if (s.cap_y < ybytes) {
    if (s.d_y) cudaFree(s.d_y);
    s.d_y = nullptr;
    s.cap_y = 0;
    B200_CUDA(cudaMalloc(&s.d_y, std::max<size_t>(ybytes, 8)));
    s.cap_y = ybytes;
  }
  B200_CUDA(cudaMemsetAsync(s.d_pcnt, 0, sizeof(int) * 2 * kMaxHeight * 8, c.stream));
  const unsigned g = grid_for(std::min<long long>(nmax, 1 << 20), 256);
  parity_count_kernel<<<g, 256, 0, c.stream>>>(la, s.d_pcnt);
  parity_place_kernel<<<g, 256, 0, c.stream>>>(la, s.d_pcnt, s.d_plist);
  c.launches += 2;
  B200_CUDA(cudaGetLastError());
  s.list_serial = c.tree_serial;
  return B200FMM_OK;
}

b200fmm_status run_m2l_sym64(Context &c, int level) {
  Sym64 &s = *c.s64;
  const Level &T = c.lv[level];
  if (T.n == 0) return B200FMM_OK;
  B200_CHECK(sym64_tree(c));
  GemmArgs a{};
  a.nn = c.nn;
  a.R = c.R;
  a.ystride = s.ystride;
  a.scale = 2.0 / (c.cfg.box_width / (double)(1LL << level));
  a.list = s.d_plist + s.h_loff[level];
  a.cnt = s.d_pcnt + level * 8;
  a.vs = s.d_vs;
  a.uc = s.d_uc;
  a.kmap = s.d_kmap;
  for (int p = 0; p < 8; ++p) {
    a.vs_off[p] = s.vs_off[p];
    a.ysum[p] = s.ysum[p];
    a.uc_off[p] = s.uc_off[p];
    a.kct[p] = s.kct[p];
    a.km_off[p] = s.km_off[p];
  }
  a.M = T.M;
  a.L = T.L;
  a.Y = s.d_y;
  a.ilist = T.ilist;
  // items per phase bound the grid: (cells / 128 + 8) tiles per parity times the row tiles
  const long long ct_tiles = (T.n + G_BN - 1) / G_BN + 8;
  const long long items1 = ct_tiles * ((s.ystride + G_BM - 1) / G_BM);
  const long long items2 = ct_tiles * ((c.nn + G_BM - 1) / G_BM);
  const int sms = sm_count(c);
  for (int r = 0; r < c.R; ++r) {
    a.rhs = r;
    sym64_y_kernel<<<(unsigned)std::min<long long>(items1, sms), G_THREADS, 0, c.stream>>>(a);
    sym64_l_kernel<<<(unsigned)std::min<long long>(items2, sms), G_THREADS, 0, c.stream>>>(a);
    c.launches += 2;
  }
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

}  // namespace b200
