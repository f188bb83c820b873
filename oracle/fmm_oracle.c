/* CPU restatement of the ScalFMM FMM hot path in FP64 -- TEST INFRASTRUCTURE ONLY (see fmm_oracle.h).
 *
 * The math follows the reference routine cited at each function; the loop structure is written for
 * clarity (direct tensor-product sums instead of the reference's BLAS factorisations), which changes
 * results only at rounding level (~1e-15 relative).
 */
#define _GNU_SOURCE
#include "fmm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXP 12

/* ------------------------------------------------------------------------------------------------
 * Morton keys and tree coordinates
 * ---------------------------------------------------------------------------------------------- */

/* FTreeCoordinate::getMortonIndex (FTreeCoordinate.hpp:91-113): bit b of z -> bit 3b, of y -> 3b+1,
 * of x -> 3b+2. */
long long orc_morton_encode(int ix, int iy, int iz) {
  long long key = 0;
  for (int b = 0; b < 21; ++b) {
    key |= (long long)((iz >> b) & 1) << (3 * b);
    key |= (long long)((iy >> b) & 1) << (3 * b + 1);
    key |= (long long)((ix >> b) & 1) << (3 * b + 2);
  }
  return key;
}

/* FTreeCoordinate::setPositionFromMorton (FTreeCoordinate.hpp:127-143). */
void orc_morton_decode(long long key, int *ix, int *iy, int *iz) {
  int x = 0, y = 0, z = 0;
  for (int b = 0; b < 21; ++b) {
    z |= (int)((key >> (3 * b)) & 1) << b;
    y |= (int)((key >> (3 * b + 1)) & 1) << b;
    x |= (int)((key >> (3 * b + 2)) & 1) << b;
  }
  *ix = x;
  *iy = y;
  *iz = z;
}

/* FCoordinateComputer::GetTreeCoordinate (FCoordinateComputer.hpp:16-25): int(rel/leafWidth), and a
 * position exactly on the upper face maps to the last cell. */
static int tree_coordinate(double rel, double box_width, double leaf_width, int height) {
  if (rel == box_width) return (1 << (height - 1)) - 1;
  return (int)(rel / leaf_width);
}

int orc_morton_keys(long long n, const double *x, const double *y, const double *z, double box_width,
                    const double *center, int height, long long *keys) {
  const double leaf_width = box_width / (double)(1 << (height - 1));
  const double cx = center[0] - box_width / 2, cy = center[1] - box_width / 2, cz = center[2] - box_width / 2;
  for (long long i = 0; i < n; ++i) {
    const double rx = x[i] - cx, ry = y[i] - cy, rz = z[i] - cz;
    if (!(rx >= 0 && rx <= box_width && ry >= 0 && ry <= box_width && rz >= 0 && rz <= box_width)) return -1;
    keys[i] = orc_morton_encode(tree_coordinate(rx, box_width, leaf_width, height),
                                tree_coordinate(ry, box_width, leaf_width, height),
                                tree_coordinate(rz, box_width, leaf_width, height));
  }
  return 0;
}

/* FTreeCoordinate::getNeighborsIndexes (FTreeCoordinate.hpp:189-216). */
int orc_leaf_neighbors(int ix, int iy, int iz, int height, long long *keys, int *positions) {
  const int lim = 1 << (height - 1);
  int k = 0;
  for (int dx = -1; dx <= 1; ++dx) {
    if (ix + dx < 0 || ix + dx >= lim) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      if (iy + dy < 0 || iy + dy >= lim) continue;
      for (int dz = -1; dz <= 1; ++dz) {
        if (iz + dz < 0 || iz + dz >= lim) continue;
        if (dx || dy || dz) {
          keys[k] = orc_morton_encode(ix + dx, iy + dy, iz + dz);
          positions[k] = ((dx + 1) * 3 + (dy + 1)) * 3 + (dz + 1);
          ++k;
        }
      }
    }
  }
  return k;
}

/* FTreeCoordinate::getInteractionNeighbors (FTreeCoordinate.hpp:219-264), separation 1. */
int orc_interaction_list(int ix, int iy, int iz, int level, long long *keys, int *positions) {
  const int px = ix >> 1, py = iy >> 1, pz = iz >> 1;
  const int lim = 1 << (level - 1);
  int k = 0;
  for (int dx = -1; dx <= 1; ++dx) {
    if (px + dx < 0 || px + dx >= lim) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      if (py + dy < 0 || py + dy >= lim) continue;
      for (int dz = -1; dz <= 1; ++dz) {
        if (pz + dz < 0 || pz + dz >= lim) continue;
        if (!(dx || dy || dz)) continue;
        const int ox = px + dx, oy = py + dy, oz = pz + dz;
        const long long pkey = orc_morton_encode(ox, oy, oz);
        for (int c = 0; c < 8; ++c) {
          const int xd = ((ox << 1) | ((c >> 2) & 1)) - ix;
          const int yd = ((oy << 1) | ((c >> 1) & 1)) - iy;
          const int zd = ((oz << 1) | (c & 1)) - iz;
          if (abs(xd) > 1 || abs(yd) > 1 || abs(zd) > 1) {
            positions[k] = ((xd + 3) * 7 + (yd + 3)) * 7 + zd + 3;
            keys[k] = (pkey << 3) | c;
            ++k;
          }
        }
      }
    }
  }
  return k;
}

/* ------------------------------------------------------------------------------------------------
 * Interpolation bases
 * ---------------------------------------------------------------------------------------------- */

/* Chebyshev roots in ascending order, xbar_j = -cos(pi (2j+1) / (2p))  (FChebRoots.hpp:31-36; the
 * reference tabulates the same values to 15 digits, FChebRoots.hpp:84-300). */
void orc_cheb_roots(int order, double *roots) {
  for (int j = 0; j < order; ++j) roots[j] = -cos(M_PI * (2.0 * j + 1.0) / (2.0 * order));
}

static double cheb_T(int n, double x) { /* FChebRoots::T, FChebRoots.hpp:45-56 */
  if (x > 1.0) x = 1.0;
  if (x < -1.0) x = -1.0;
  return cos(n * acos(x));
}

/* Uniform (Lagrange) roots, xbar_n = -1 + 2n/(p-1)  (FUnifRoots.hpp:35-39). */
static void unif_roots(int order, double *roots) {
  for (int j = 0; j < order; ++j) roots[j] = -1.0 + 2.0 * j / (double)(order - 1);
}

/* Lagrange polynomial L_n(x) on equispaced nodes (FUnifRoots::L, FUnifRoots.hpp:49-83). */
static double unif_L(int order, int n, double x) {
  if (x > 1.0) x = 1.0;
  if (x < -1.0) x = -1.0;
  double scale = ((order - n - 1) % 2) ? -1.0 : 1.0;
  double fn = 1.0, fm = 1.0;
  for (int k = 2; k <= n; ++k) fn *= k;
  for (int k = 2; k <= order - n - 1; ++k) fm *= k;
  scale /= pow(2.0, order - 1) * fn * fm;
  double L = 1.0;
  for (int m = 0; m < order; ++m)
    if (m != n) L *= (double)(order - 1) * (x + 1.0) - 2.0 * m;
  return L * scale;
}

/* dL_n/dx (FUnifRoots::dL, FUnifRoots.hpp:92-121). */
static double unif_dL(int order, const double *roots, int n, double x) {
  if (x > 1.0) x = 1.0;
  if (x < -1.0) x = -1.0;
  double num = 0.0, den = 1.0;
  for (int p = 0; p < order; ++p) {
    if (p == n) continue;
    double t = 1.0;
    for (int m = 0; m < order; ++m)
      if (m != n && m != p) t *= x - roots[m];
    num += t;
    den *= roots[n] - roots[p];
  }
  return num / den;
}

typedef struct {
  int kind, p, nn;
  double roots[MAXP];
  double Troot[MAXP][MAXP]; /* Chebyshev: T_o(root_j) */
} basis_t;

static void basis_init(basis_t *b, int kind, int p) {
  b->kind = kind;
  b->p = p;
  b->nn = p * p * p;
  if (kind == ORC_LAGRANGE)
    unif_roots(p, b->roots);
  else
    orc_cheb_roots(p, b->roots);
  for (int o = 0; o < p; ++o)
    for (int j = 0; j < p; ++j) b->Troot[o][j] = cheb_T(o, b->roots[j]);
}

/* One-dimensional interpolation weights S_j(x) and their derivatives for j = 0..p-1, x in [-1,1].
 * Chebyshev: S_j(x) = 1/p + 2/p sum_{o>=1} T_o(x) T_o(xbar_j)   (FChebInterpolator.hpp:466-485), with
 * T_o(x) by the three-term recurrence and dT_o/dx = o U_{o-1}(x) (FChebInterpolator.hpp:1310-1336).
 * Lagrange: S_j(x) = L_j(x), dS_j = dL_j (FUnifInterpolator.hpp:340-390). */
static void basis_weights(const basis_t *b, double x, double *S, double *dS) {
  const int p = b->p;
  if (b->kind == ORC_LAGRANGE) {
    for (int j = 0; j < p; ++j) {
      S[j] = unif_L(p, j, x);
      if (dS) dS[j] = unif_dL(p, b->roots, j, x);
    }
    return;
  }
  double T[MAXP], U[MAXP];
  T[0] = 1.0;
  T[1] = x;
  U[0] = 1.0;
  U[1] = 2.0 * x;
  for (int o = 2; o < p; ++o) {
    T[o] = 2.0 * x * T[o - 1] - T[o - 2];
    U[o] = 2.0 * x * U[o - 1] - U[o - 2];
  }
  for (int j = 0; j < p; ++j) {
    double s = 1.0 / p, ds = 0.0;
    for (int o = 1; o < p; ++o) {
      s += 2.0 / p * T[o] * b->Troot[o][j];
      ds += 2.0 / p * (double)o * U[o - 1] * b->Troot[o][j];
    }
    S[j] = s;
    if (dS) dS[j] = ds;
  }
}

/* Child->parent 1-D interpolators for the 8 children (FChebInterpolator::initTensorM2MandL2L,
 * FChebInterpolator.hpp:300-338): the child's roots expressed in the parent frame are
 * +-0.5 + 0.5*xbar_m, and S[c][d][n*p+m] = S_n(child root m along axis d). */
static void child_interpolators(const basis_t *b, double *S /* [8][3][p*p] */) {
  const int p = b->p;
  for (int c = 0; c < 8; ++c) {
    const double sgn[3] = {(c >> 2) & 1 ? 0.5 : -0.5, (c >> 1) & 1 ? 0.5 : -0.5, c & 1 ? 0.5 : -0.5};
    for (int d = 0; d < 3; ++d) {
      for (int m = 0; m < p; ++m) {
        double w[MAXP];
        basis_weights(b, sgn[d] + 0.5 * b->roots[m], w, NULL);
        for (int n = 0; n < p; ++n) S[((c * 3 + d) * p + n) * p + m] = w[n];
      }
    }
  }
}

/* ------------------------------------------------------------------------------------------------
 * Symmetries (FInterpSymmetries.hpp:18-125)
 * ---------------------------------------------------------------------------------------------- */
int orc_sym_tables(int order, unsigned *pindices, unsigned *pvectors) {
  const int p = order, nn = p * p * p;
  if (p < 2 || p > MAXP) return -1;
  unsigned *quads = (unsigned *)malloc(sizeof(unsigned) * 8 * nn);
  unsigned *cones = (unsigned *)malloc(sizeof(unsigned) * 8 * nn);
  unsigned evn[MAXP], odd[MAXP];
  for (int o = 0; o < p; ++o) {
    evn[o] = o;
    odd[o] = p - 1 - o;
  }
  for (int i = 0; i < p; ++i)
    for (int j = 0; j < p; ++j)
      for (int k = 0; k < p; ++k) {
        const int idx = k * p * p + j * p + i;
        for (int q = 0; q < 8; ++q) {
          const unsigned ii = (q & 1) ? odd[i] : evn[i];
          const unsigned jj = (q & 2) ? odd[j] : evn[j];
          const unsigned kk = (q & 4) ? odd[k] : evn[k];
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
        pindices[t] = 0;
        for (int n = 0; n < nn; ++n) pvectors[(long)t * nn + n] = 0;
        if (!(abs(i) > 1 || abs(j) > 1 || abs(k) > 1)) continue;
        const int qidx = (i < 0 ? 1 : 0) | (j < 0 ? 2 : 0) | (k < 0 ? 4 : 0);
        const int u[3] = {abs(i), abs(j), abs(k)};
        const int cidx = ((u[1] > u[0]) << 2) | ((u[2] > u[0]) << 1) | (u[2] > u[1]);
        for (int n = 0; n < nn; ++n) pvectors[(long)t * nn + n] = cones[cidx * nn + quads[qidx * nn + n]];
        pindices[t] = (u[perms[cidx][0]] + 3) * 49 + (u[perms[cidx][1]] + 3) * 7 + (u[perms[cidx][2]] + 3);
      }
  free(quads);
  free(cones);
  return 0;
}

/* ------------------------------------------------------------------------------------------------
 * Direct sum
 * ---------------------------------------------------------------------------------------------- */

/* FP2PR::NonMutualParticles (FP2PR.hpp:45-69): phi += q_s/r, F += -q_t q_s (x_t-x_s)/r^3. */
static inline void pair_nonmutual(double tx, double ty, double tz, double tq, double sx, double sy, double sz,
                                  double sq, double *p, double *gx, double *gy, double *gz) {
  double dx = tx - sx, dy = ty - sy, dz = tz - sz;
  double inv2 = 1.0 / (dx * dx + dy * dy + dz * dz);
  const double inv = sqrt(inv2);
  inv2 *= inv;
  inv2 *= tq * sq;
  *gx += -dx * inv2;
  *gy += -dy * inv2;
  *gz += -dz * inv2;
  *p += inv * sq;
}

int orc_direct(long long n, const double *x, const double *y, const double *z, const double *q,
               long long ntargets, const long long *targets, int nthreads, double *phi, double *fx, double *fy,
               double *fz) {
  const long long nt = ntargets < 0 ? n : ntargets;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 64)
  for (long long k = 0; k < nt; ++k) {
    const long long i = ntargets < 0 ? k : targets[k];
    double p = 0, gx = 0, gy = 0, gz = 0;
    for (long long j = 0; j < n; ++j)
      if (j != i) pair_nonmutual(x[i], y[i], z[i], q[i], x[j], y[j], z[j], q[j], &p, &gx, &gy, &gz);
    phi[k] = p;
    fx[k] = gx;
    fy[k] = gy;
    fz[k] = gz;
  }
  return 0;
}

/* ------------------------------------------------------------------------------------------------
 * Tree
 * ---------------------------------------------------------------------------------------------- */
typedef struct {
  int height, nlevels;
  long long *ncells;   /* per level */
  long long **keys;    /* per level, sorted unique Morton keys of non-empty cells */
  long long *leaf_start, *leaf_end; /* per leaf (level height-1), into the sorted particle order */
  long long *perm;     /* sorted position -> original particle index */
} tree_t;

static const long long *g_sort_keys;
static int cmp_idx(const void *a, const void *b) {
  const long long ia = *(const long long *)a, ib = *(const long long *)b;
  const long long ka = g_sort_keys[ia], kb = g_sort_keys[ib];
  if (ka != kb) return ka < kb ? -1 : 1;
  return ia < ib ? -1 : (ia > ib); /* stable: insertion order inside a leaf (FOctree::insert appends) */
}

static long long find_key(const long long *keys, long long n, long long key) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long mid = (lo + hi) / 2;
    if (keys[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < n && keys[lo] == key) ? lo : -1;
}

static int tree_build(tree_t *t, const long long *pkeys, long long n, int height) {
  t->height = height;
  t->nlevels = height;
  t->perm = (long long *)malloc(sizeof(long long) * (n > 0 ? n : 1));
  for (long long i = 0; i < n; ++i) t->perm[i] = i;
  g_sort_keys = pkeys;
  qsort(t->perm, n, sizeof(long long), cmp_idx);
  t->ncells = (long long *)calloc(height, sizeof(long long));
  t->keys = (long long **)calloc(height, sizeof(long long *));
  const int L = height - 1;
  long long nleaves = 0;
  for (long long i = 0; i < n; ++i)
    if (i == 0 || pkeys[t->perm[i]] != pkeys[t->perm[i - 1]]) ++nleaves;
  t->keys[L] = (long long *)malloc(sizeof(long long) * (nleaves ? nleaves : 1));
  t->leaf_start = (long long *)malloc(sizeof(long long) * (nleaves ? nleaves : 1));
  t->leaf_end = (long long *)malloc(sizeof(long long) * (nleaves ? nleaves : 1));
  long long k = -1;
  for (long long i = 0; i < n; ++i) {
    const long long key = pkeys[t->perm[i]];
    if (i == 0 || key != pkeys[t->perm[i - 1]]) {
      ++k;
      t->keys[L][k] = key;
      t->leaf_start[k] = i;
    }
    t->leaf_end[k] = i + 1;
  }
  t->ncells[L] = nleaves;
  for (int l = L - 1; l >= 0; --l) {
    const long long nc = t->ncells[l + 1];
    t->keys[l] = (long long *)malloc(sizeof(long long) * (nc ? nc : 1));
    long long m = 0;
    for (long long i = 0; i < nc; ++i) {
      const long long pk = t->keys[l + 1][i] >> 3;
      if (m == 0 || t->keys[l][m - 1] != pk) t->keys[l][m++] = pk;
    }
    t->ncells[l] = m;
  }
  return 0;
}

static void tree_free(tree_t *t) {
  for (int l = 0; l < t->nlevels; ++l) free(t->keys[l]);
  free(t->keys);
  free(t->ncells);
  free(t->leaf_start);
  free(t->leaf_end);
  free(t->perm);
}

/* ------------------------------------------------------------------------------------------------
 * FMM passes
 * ---------------------------------------------------------------------------------------------- */

/* Tensor-product evaluation helpers: w[d][j] per axis. */
static inline double tensor3(const double *wx, const double *wy, const double *wz, int n, int p) {
  return wx[n % p] * wy[(n / p) % p] * wz[n / (p * p)];
}

int orc_fmm(const orc_config *cfg, long long n, const double *x, const double *y, const double *z,
            const double *q, unsigned ops, double *phi, double *fx, double *fy, double *fz, orc_dump *dump) {
  const int p = cfg->order, H = cfg->height, R = cfg->nrhs > 0 ? cfg->nrhs : 1;
  if (p < 2 || p > MAXP || H < 2 || H > 21) return -1;
  if (cfg->kind == ORC_CHEB_SYM && (!cfg->sym_ranks || !cfg->sym_uv)) return -2;
#ifdef _OPENMP
  if (cfg->nthreads > 0) omp_set_num_threads(cfg->nthreads);
#endif
  const int nn = p * p * p;
  const double W = cfg->box_width;
  const double corner[3] = {cfg->center[0] - W / 2, cfg->center[1] - W / 2, cfg->center[2] - W / 2};
  basis_t B;
  basis_init(&B, cfg->kind, p);

  long long *pkeys = (long long *)malloc(sizeof(long long) * (n > 0 ? n : 1));
  if (orc_morton_keys(n, x, y, z, W, cfg->center, H, pkeys) != 0) {
    free(pkeys);
    return -3;
  }
  tree_t T;
  tree_build(&T, pkeys, n, H);
  free(pkeys);
  const int LL = H - 1;

  /* expansions per level: [ncells][R][nn] */
  double **M = (double **)calloc(H, sizeof(double *));
  double **Lc = (double **)calloc(H, sizeof(double *));
  for (int l = 0; l < H; ++l) {
    M[l] = (double *)calloc((size_t)(T.ncells[l] ? T.ncells[l] : 1) * R * nn, sizeof(double));
    Lc[l] = (double *)calloc((size_t)(T.ncells[l] ? T.ncells[l] : 1) * R * nn, sizeof(double));
  }
  for (long long i = 0; i < (long long)R * n; ++i) phi[i] = fx[i] = fy[i] = fz[i] = 0.0;

  const double leaf_w = W / (double)(1 << LL);

  /* P2M: FChebSymKernel::P2M (FChebSymKernel.hpp:181-188) -> applyP2M (FChebInterpolator.hpp:627-762):
   * M[n] = sum_particles q * prod_d S_{n_d}(x_d), x mapped to [-1,1] by map_glob_loc
   * (FInterpMapping.hpp:101-114) around the leaf centre (FAbstractChebKernel.hpp:54-59). */
  if (ops & ORC_P2M) {
#pragma omp parallel for schedule(dynamic, 4)
    for (long long c = 0; c < T.ncells[LL]; ++c) {
      int ix, iy, iz;
      orc_morton_decode(T.keys[LL][c], &ix, &iy, &iz);
      const double ctr[3] = {corner[0] + (ix + 0.5) * leaf_w, corner[1] + (iy + 0.5) * leaf_w,
                             corner[2] + (iz + 0.5) * leaf_w};
      for (long long s = T.leaf_start[c]; s < T.leaf_end[c]; ++s) {
        const long long i = T.perm[s];
        const double pos[3] = {x[i], y[i], z[i]};
        double w[3][MAXP];
        for (int d = 0; d < 3; ++d) {
          const double a = ctr[d] - leaf_w / 2, b = ctr[d] + leaf_w / 2;
          basis_weights(&B, (2.0 * pos[d] - b - a) / (b - a), w[d], NULL);
        }
        for (int r = 0; r < R; ++r) {
          const double qq = q[(long long)r * n + i];
          double *m = M[LL] + ((size_t)c * R + r) * nn;
          for (int k = 0; k < nn; ++k) m[k] += qq * tensor3(w[0], w[1], w[2], k, p);
        }
      }
    }
  }

  double *S = (double *)malloc(sizeof(double) * 8 * 3 * p * p);
  child_interpolators(&B, S);

  /* M2M: levels H-2 .. 2 (FFmmAlgorithmThread.hpp:204-254), FChebSymKernel::M2M (FChebSymKernel.hpp:192-206)
   * -> applyM2M (FChebInterpolator.hpp:560-584): parent[n] += sum_m prod_d S[c][d][n_d, m_d] child[m]. */
  if (ops & ORC_M2M) {
    for (int l = LL - 1; l >= 2; --l) {
#pragma omp parallel for schedule(dynamic, 4)
      for (long long c = 0; c < T.ncells[l]; ++c) {
        const long long pk = T.keys[l][c];
        for (int ch = 0; ch < 8; ++ch) {
          const long long ci = find_key(T.keys[l + 1], T.ncells[l + 1], (pk << 3) | ch);
          if (ci < 0) continue;
          const double *Sx = S + (ch * 3 + 0) * p * p, *Sy = S + (ch * 3 + 1) * p * p, *Sz = S + (ch * 3 + 2) * p * p;
          for (int r = 0; r < R; ++r) {
            const double *src = M[l + 1] + ((size_t)ci * R + r) * nn;
            double *dst = M[l] + ((size_t)c * R + r) * nn;
            for (int nI = 0; nI < nn; ++nI) {
              const int a = nI % p, b = (nI / p) % p, cc = nI / (p * p);
              double acc = 0.0;
              for (int mI = 0; mI < nn; ++mI)
                acc += Sx[a * p + mI % p] * Sy[b * p + (mI / p) % p] * Sz[cc * p + mI / (p * p)] * src[mI];
              dst[nI] += acc;
            }
          }
        }
      }
    }
  }

  /* M2L: levels 2..H-1 (FFmmAlgorithmThread.hpp:271-322) over the interaction list.
   *  - ORC_CHEB_SYM: FChebSymKernel::M2L (FChebSymKernel.hpp:210-328) with the compressed 16-class
   *    operators and permutation vectors: L[n] += scale * (U (V^T M'))[pvec[n]], M'[pvec[n]] = M[n].
   *  - ORC_CHEB_DENSE / ORC_LAGRANGE: L[m] += scale * sum_n K(X_m, Y_n) M[n] with X the target nodes of
   *    a width-2 cell at the origin and Y the source nodes centred at 2*(dx,dy,dz)
   *    (FChebDenseM2LHandler.hpp:178-215; the FFT-diagonalised FUnifM2LHandler applies the same
   *    Toeplitz operator, FUnifM2LHandler.hpp:26-124).
   *  scale = 2 / cell width (FInterpMatrixKernel.hpp:124-133). */
  if (ops & ORC_M2L) {
    unsigned *pind = NULL, *pvec = NULL;
    const double **Uk = NULL, **Vk = NULL;
    double *Kd = NULL; /* dense operators, only the slots that occur, computed lazily per slot */
    unsigned char *Kd_ready = NULL;
    if (cfg->kind == ORC_CHEB_SYM) {
      pind = (unsigned *)malloc(sizeof(unsigned) * 343);
      pvec = (unsigned *)malloc(sizeof(unsigned) * 343 * nn);
      orc_sym_tables(p, pind, pvec);
      Uk = (const double **)calloc(343, sizeof(double *));
      Vk = (const double **)calloc(343, sizeof(double *));
      long long off = 0;
      for (int t = 0; t < 343; ++t)
        if (cfg->sym_ranks[t] > 0) {
          Uk[t] = cfg->sym_uv + off;
          Vk[t] = cfg->sym_uv + off + (long long)cfg->sym_ranks[t] * nn;
          off += 2LL * cfg->sym_ranks[t] * nn;
        }
    } else {
      Kd = (double *)malloc(sizeof(double) * 343 * (size_t)nn * nn);
      Kd_ready = (unsigned char *)calloc(343, 1);
      double X[MAXP * MAXP * MAXP][3];
      for (int m = 0; m < nn; ++m) {
        X[m][0] = B.roots[m % p];
        X[m][1] = B.roots[(m / p) % p];
        X[m][2] = B.roots[m / (p * p)];
      }
      for (int t = 0; t < 343; ++t) {
        const int i = t / 49 - 3, j = (t / 7) % 7 - 3, k = t % 7 - 3;
        if (!(abs(i) > 1 || abs(j) > 1 || abs(k) > 1)) continue;
        for (int m = 0; m < nn; ++m)
          for (int nI = 0; nI < nn; ++nI) {
            const double dx = X[m][0] - (2.0 * i + X[nI][0]);
            const double dy = X[m][1] - (2.0 * j + X[nI][1]);
            const double dz = X[m][2] - (2.0 * k + X[nI][2]);
            Kd[((size_t)t * nn + m) * nn + nI] = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
          }
        Kd_ready[t] = 1;
      }
    }
    for (int l = 2; l <= LL; ++l) {
      const double scale = 2.0 / (W / (double)(1LL << l));
#pragma omp parallel
      {
        double *mp = (double *)malloc(sizeof(double) * nn);
        double *lp = (double *)malloc(sizeof(double) * nn);
        double *yc = (double *)malloc(sizeof(double) * nn);
        long long nkeys[343];
        int npos[343];
#pragma omp for schedule(dynamic, 4)
        for (long long c = 0; c < T.ncells[l]; ++c) {
          int ix, iy, iz;
          orc_morton_decode(T.keys[l][c], &ix, &iy, &iz);
          const int cnt = orc_interaction_list(ix, iy, iz, l, nkeys, npos);
          for (int e = 0; e < cnt; ++e) {
            const long long si = find_key(T.keys[l], T.ncells[l], nkeys[e]);
            if (si < 0) continue;
            const int t = npos[e];
            for (int r = 0; r < R; ++r) {
              const double *Ms = M[l] + ((size_t)si * R + r) * nn;
              double *Lt = Lc[l] + ((size_t)c * R + r) * nn;
              if (cfg->kind == ORC_CHEB_SYM) {
                const unsigned cls = pind[t];
                const int rk = cfg->sym_ranks[cls];
                const unsigned *pv = pvec + (size_t)t * nn;
                for (int m = 0; m < nn; ++m) mp[pv[m]] = Ms[m];
                for (int a = 0; a < rk; ++a) {
                  double acc = 0.0;
                  const double *v = Vk[cls] + (size_t)a * nn;
                  for (int m = 0; m < nn; ++m) acc += v[m] * mp[m];
                  yc[a] = acc;
                }
                for (int m = 0; m < nn; ++m) {
                  double acc = 0.0;
                  for (int a = 0; a < rk; ++a) acc += Uk[cls][(size_t)a * nn + m] * yc[a];
                  lp[m] = scale * acc;
                }
                for (int m = 0; m < nn; ++m) Lt[m] += lp[pv[m]];
              } else {
                const double *K = Kd + (size_t)t * nn * nn;
                for (int m = 0; m < nn; ++m) {
                  double acc = 0.0;
                  for (int nI = 0; nI < nn; ++nI) acc += K[(size_t)m * nn + nI] * Ms[nI];
                  Lt[m] += scale * acc;
                }
              }
            }
          }
        }
        free(mp);
        free(lp);
        free(yc);
      }
    }
    free(pind);
    free(pvec);
    free(Uk);
    free(Vk);
    free(Kd);
    free(Kd_ready);
  }

  /* L2L: parents at levels 2..H-2 (FFmmAlgorithmThread.hpp:329-373), applyL2L
   * (FChebInterpolator.hpp:587-611): child[m] += sum_n prod_d S[c][d][n_d, m_d] parent[n]. */
  if (ops & ORC_L2L) {
    for (int l = 2; l <= LL - 1; ++l) {
#pragma omp parallel for schedule(dynamic, 4)
      for (long long ci = 0; ci < T.ncells[l + 1]; ++ci) {
        const long long ck = T.keys[l + 1][ci];
        const long long pi = find_key(T.keys[l], T.ncells[l], ck >> 3);
        const int ch = (int)(ck & 7);
        const double *Sx = S + (ch * 3 + 0) * p * p, *Sy = S + (ch * 3 + 1) * p * p, *Sz = S + (ch * 3 + 2) * p * p;
        for (int r = 0; r < R; ++r) {
          const double *src = Lc[l] + ((size_t)pi * R + r) * nn;
          double *dst = Lc[l + 1] + ((size_t)ci * R + r) * nn;
          for (int mI = 0; mI < nn; ++mI) {
            const int a = mI % p, b = (mI / p) % p, cc = mI / (p * p);
            double acc = 0.0;
            for (int nI = 0; nI < nn; ++nI)
              acc += Sx[(nI % p) * p + a] * Sy[((nI / p) % p) * p + b] * Sz[(nI / (p * p)) * p + cc] * src[nI];
            dst[mI] += acc;
          }
        }
      }
    }
  }

  /* L2P (FChebInterpolator::applyL2PTotal, FChebInterpolator.hpp:1222-1417): phi += sum_n L[n] S_n(x),
   * F += q * grad_x (sum_n L[n] S_n(x)) with the Jacobian 2/leaf width. */
  if (ops & ORC_L2P) {
#pragma omp parallel for schedule(dynamic, 4)
    for (long long c = 0; c < T.ncells[LL]; ++c) {
      int ix, iy, iz;
      orc_morton_decode(T.keys[LL][c], &ix, &iy, &iz);
      const double ctr[3] = {corner[0] + (ix + 0.5) * leaf_w, corner[1] + (iy + 0.5) * leaf_w,
                             corner[2] + (iz + 0.5) * leaf_w};
      const double jac = 2.0 / leaf_w;
      for (long long s = T.leaf_start[c]; s < T.leaf_end[c]; ++s) {
        const long long i = T.perm[s];
        const double pos[3] = {x[i], y[i], z[i]};
        double w[3][MAXP], dw[3][MAXP];
        for (int d = 0; d < 3; ++d) {
          const double a = ctr[d] - leaf_w / 2, b = ctr[d] + leaf_w / 2;
          basis_weights(&B, (2.0 * pos[d] - b - a) / (b - a), w[d], dw[d]);
        }
        for (int r = 0; r < R; ++r) {
          const double *Lt = Lc[LL] + ((size_t)c * R + r) * nn;
          double pv = 0, gx = 0, gy = 0, gz = 0;
          for (int k = 0; k < nn; ++k) {
            const int a = k % p, b = (k / p) % p, cc = k / (p * p);
            pv += Lt[k] * w[0][a] * w[1][b] * w[2][cc];
            gx += Lt[k] * dw[0][a] * w[1][b] * w[2][cc];
            gy += Lt[k] * w[0][a] * dw[1][b] * w[2][cc];
            gz += Lt[k] * w[0][a] * w[1][b] * dw[2][cc];
          }
          const long long j = (long long)r * n + i;
          const double qq = q[j];
          phi[j] += pv;
          fx[j] += gx * jac * qq;
          fy[j] += gy * jac * qq;
          fz[j] += gz * jac * qq;
        }
      }
    }
  }

  /* P2P over the leaf and its <=26 neighbours (FChebSymKernel::P2P, FChebSymKernel.hpp:453-478; the
   * mutual half-shell evaluation there computes the same ordered pairs as this target-stationary sum). */
  if (ops & ORC_P2P) {
#pragma omp parallel for schedule(dynamic, 4)
    for (long long c = 0; c < T.ncells[LL]; ++c) {
      int ix, iy, iz;
      orc_morton_decode(T.keys[LL][c], &ix, &iy, &iz);
      long long nk[27];
      int np[27];
      const int cnt = orc_leaf_neighbors(ix, iy, iz, H, nk, np);
      nk[cnt] = T.keys[LL][c];
      long long srcs[27];
      int ns = 0;
      for (int e = 0; e <= cnt; ++e) {
        const long long si = find_key(T.keys[LL], T.ncells[LL], nk[e]);
        if (si >= 0) srcs[ns++] = si;
      }
      for (long long s = T.leaf_start[c]; s < T.leaf_end[c]; ++s) {
        const long long i = T.perm[s];
        for (int r = 0; r < R; ++r) {
          const double *qr = q + (long long)r * n;
          double pv = 0, gx = 0, gy = 0, gz = 0;
          for (int e = 0; e < ns; ++e)
            for (long long u = T.leaf_start[srcs[e]]; u < T.leaf_end[srcs[e]]; ++u) {
              const long long j = T.perm[u];
              if (j == i) continue;
              pair_nonmutual(x[i], y[i], z[i], qr[i], x[j], y[j], z[j], qr[j], &pv, &gx, &gy, &gz);
            }
          const long long jj = (long long)r * n + i;
          phi[jj] += pv;
          fx[jj] += gx;
          fy[jj] += gy;
          fz[jj] += gz;
        }
      }
    }
  }

  if (dump) {
    long long k = 0;
    for (int l = 0; l < H; ++l)
      for (long long c = 0; c < T.ncells[l]; ++c, ++k) {
        if (k >= dump->cap) continue;
        dump->levels[k] = l;
        dump->mortons[k] = T.keys[l][c];
        memcpy(dump->multipoles + (size_t)k * R * nn, M[l] + (size_t)c * R * nn, sizeof(double) * R * nn);
        memcpy(dump->locals + (size_t)k * R * nn, Lc[l] + (size_t)c * R * nn, sizeof(double) * R * nn);
      }
    dump->count = k;
  }

  free(S);
  for (int l = 0; l < H; ++l) {
    free(M[l]);
    free(Lc[l]);
  }
  free(M);
  free(Lc);
  tree_free(&T);
  return 0;
}
