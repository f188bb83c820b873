// ScalFMM's C user API (Addons/CKernelApi/Src/CScalfmmApi.h) forwarded to one b200fmm handle, and the
// .fma / .bfma particle files of FFmaGenericLoader / FFmaGenericWriter (Src/Files/FFmaGenericLoader.hpp).
//
// The shim keeps the particles in insertion order on the host (positions, charges, potentials, forces) and hands
// them to the handle at execute time: new or moved particles rebuild the tree (b200fmm_set_particles), new charges
// alone replace them on the current tree (b200fmm_set_charges).  The computed potentials and forces come back in
// insertion order and are added to the host copies, the reference's containers' "+=" semantics.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/b200fmm.h"
#include "../../include/b200fmm_capi.h"

namespace {

struct CapiHandle {
  scalfmm_kernel_type kernel = chebyshev;
  scalfmm_algorithm algo = multi_thread;
  int precision = B200FMM_FP64;
  int height = 0;
  double width = 0, center[3] = {0, 0, 0};
  b200fmm_handle h = nullptr;
  std::vector<double> x, y, z, q, phi, fx, fy, fz;
  bool tree_dirty = true;     // positions changed since the handle last saw them
  bool charges_dirty = true;  // charges changed since the handle last saw them
  b200fmm_status status = B200FMM_OK;
  double timers_s[9] = {0};
};

CapiHandle *as_handle(scalfmm_handle h) { return static_cast<CapiHandle *>(h); }

// Failures print one line (the reference would abort) and stay readable through b200fmm_capi_status.
void report(CapiHandle *c, b200fmm_status st, const char *where, const char *what = nullptr) {
  if (st == B200FMM_OK) return;
  if (c) c->status = st;
  std::fprintf(stderr, "b200fmm C API: %s: %s\n", where, what ? what : b200fmm_last_error());
}

bool check(CapiHandle *c, const char *where) {
  if (!c) {
    std::fprintf(stderr, "b200fmm C API: %s: null handle\n", where);
    return false;
  }
  return true;
}

// An index list of the _npart variants, checked against the particle count.
bool check_indices(CapiHandle *c, int n, const int *idx, const char *where) {
  if (n < 0 || (n > 0 && !idx)) {
    report(c, B200FMM_ERR_INVALID, where, "bad particle index list");
    return false;
  }
  for (int k = 0; k < n; ++k)
    if (idx[k] < 0 || (size_t)idx[k] >= c->x.size()) {
      report(c, B200FMM_ERR_INVALID, where, "particle index out of range");
      return false;
    }
  return true;
}

bool check_count(CapiHandle *c, int n, const char *where) {
  if (n < 0 || (size_t)n != c->x.size()) {
    report(c, B200FMM_ERR_INVALID, where, "count differs from the number of inserted particles");
    return false;
  }
  return true;
}

void append(CapiHandle *c, int n, const double *X, const double *Y, const double *Z, long long sx, long long sy,
            long long sz) {
  for (int i = 0; i < n; ++i) {
    c->x.push_back(X[i * sx]);
    c->y.push_back(Y[i * sy]);
    c->z.push_back(Z[i * sz]);
    c->q.push_back(0.0);
    c->phi.push_back(0.0);
    c->fx.push_back(0.0);
    c->fy.push_back(0.0);
    c->fz.push_back(0.0);
  }
  c->tree_dirty = c->charges_dirty = true;
}

void execute(CapiHandle *c, unsigned ops, const char *where) {
  if (!c->h) return report(c, B200FMM_ERR_STATE, where, "scalfmm_build_tree was not called");
  const long long n = (long long)c->x.size();
  if (n == 0) return report(c, B200FMM_ERR_STATE, where, "no particles inserted");
  b200fmm_status st = B200FMM_OK;
  if (c->tree_dirty) {
    st = b200fmm_set_particles(c->h, n, c->x.data(), c->y.data(), c->z.data(), c->q.data(), 0);
    if (st == B200FMM_OK) c->tree_dirty = c->charges_dirty = false;
  } else if (c->charges_dirty) {
    st = b200fmm_set_charges(c->h, c->q.data(), 0);
    if (st == B200FMM_OK) c->charges_dirty = false;
  }
  if (st == B200FMM_OK) st = b200fmm_execute(c->h, ops);
  std::vector<double> r((size_t)4 * n);
  if (st == B200FMM_OK) st = b200fmm_get_results(c->h, r.data(), r.data() + n, r.data() + 2 * n, r.data() + 3 * n, 0);
  if (st != B200FMM_OK) return report(c, st, where);
  for (long long i = 0; i < n; ++i) {
    c->phi[i] += r[i];
    c->fx[i] += r[n + i];
    c->fy[i] += r[2 * n + i];
    c->fz[i] += r[3 * n + i];
  }
  double ms[8];
  if (b200fmm_last_timings(c->h, ms) == B200FMM_OK) {
    // P2M, M2M, M2L, L2L, L2P, P2P, NearField (P2P + L2P), M2P, P2L
    const double t[9] = {ms[1], ms[2], ms[3], ms[4], ms[5], ms[6], ms[5] + ms[6], 0.0, 0.0};
    for (int k = 0; k < 9; ++k) c->timers_s[k] = 1e-3 * t[k];
  }
}

}  // namespace

extern "C" {

scalfmm_handle scalfmm_init(scalfmm_kernel_type KernelType, scalfmm_algorithm algo) {
  if (KernelType != chebyshev && KernelType != lagrange) {
    report(nullptr, B200FMM_ERR_UNSUPPORTED, "scalfmm_init",
           "only the built-in interpolation kernels (chebyshev, lagrange) run on this library");
    return nullptr;
  }
  CapiHandle *c = new CapiHandle();
  c->kernel = KernelType;
  scalfmm_algorithm_config(c, algo);
  return c;
}

void scalfmm_algorithm_config(scalfmm_handle Handle, scalfmm_algorithm config) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_algorithm_config")) return;
  if (config != sequential && config != multi_thread)
    return report(c, B200FMM_ERR_UNSUPPORTED, "scalfmm_algorithm_config",
                  "only the sequential and multi_thread algorithms are available");
  c->algo = config;
}

b200fmm_status b200fmm_capi_set_precision(scalfmm_handle handle, int precision) {
  CapiHandle *c = as_handle(handle);
  if (!c) return B200FMM_ERR_INVALID;
  if (precision != B200FMM_FP64 && precision != B200FMM_MIXED) return B200FMM_ERR_INVALID;
  if (c->h) return B200FMM_ERR_STATE;
  c->precision = precision;
  return B200FMM_OK;
}

b200fmm_status b200fmm_capi_status(scalfmm_handle handle) {
  CapiHandle *c = as_handle(handle);
  return c ? c->status : B200FMM_ERR_INVALID;
}

void scalfmm_build_tree(scalfmm_handle handle, int TreeHeight, double BoxWidth, double *BoxCenter,
                        Scalfmm_Cell_Descriptor, Scalfmm_Leaf_Descriptor) {
  CapiHandle *c = as_handle(handle);
  if (!check(c, "scalfmm_build_tree")) return;
  if (!BoxCenter) return report(c, B200FMM_ERR_INVALID, "scalfmm_build_tree", "null box centre");
  if (c->h) b200fmm_destroy(c->h);
  c->h = nullptr;
  b200fmm_config cfg{};
  cfg.kernel = c->kernel == chebyshev ? B200FMM_CHEB_SYM : B200FMM_LAGRANGE;
  cfg.order = 7;  // FScalfmmApiInit.cpp:44: FChebSymKernel<..., 7>
  cfg.height = TreeHeight;
  cfg.nrhs = 1;
  cfg.precision = c->precision;
  cfg.box_width = BoxWidth;
  for (int d = 0; d < 3; ++d) cfg.center[d] = BoxCenter[d];
  cfg.epsilon = 0.0;
  cfg.stream = nullptr;
  cfg.device = -1;
  const b200fmm_status st = b200fmm_create(&cfg, &c->h);
  if (st != B200FMM_OK) return report(c, st, "scalfmm_build_tree");
  c->height = TreeHeight;
  c->width = BoxWidth;
  for (int d = 0; d < 3; ++d) c->center[d] = BoxCenter[d];
  c->tree_dirty = c->charges_dirty = true;
}

void scalfmm_tree_abstract_insert(scalfmm_handle Handle, int NbPartToInsert, int nbAttributeToInsert,
                                  int *strideForEachAtt, double *rawDatas) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_tree_abstract_insert")) return;
  if (NbPartToInsert < 0 || nbAttributeToInsert < 3 || !strideForEachAtt || (NbPartToInsert && !rawDatas))
    return report(c, B200FMM_ERR_INVALID, "scalfmm_tree_abstract_insert", "bad arguments");
  // one record per particle, the attribute a at offset strideForEachAtt[a]; the record length is one past
  // the largest offset; the fourth attribute, when given, is the physical value
  int rec = 0;
  for (int a = 0; a < nbAttributeToInsert; ++a) rec = std::max(rec, strideForEachAtt[a] + 1);
  const size_t first = c->x.size();
  append(c, NbPartToInsert, rawDatas + strideForEachAtt[0], rawDatas + strideForEachAtt[1],
         rawDatas + strideForEachAtt[2], rec, rec, rec);
  if (nbAttributeToInsert > 3)
    for (int i = 0; i < NbPartToInsert; ++i) c->q[first + i] = rawDatas[(size_t)i * rec + strideForEachAtt[3]];
}

void scalfmm_tree_insert_particles(scalfmm_handle Handle, int NbPositions, double *arrayX, double *arrayY,
                                   double *arrayZ, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_tree_insert_particles")) return;
  if (NbPositions < 0 || (NbPositions && (!arrayX || !arrayY || !arrayZ)))
    return report(c, B200FMM_ERR_INVALID, "scalfmm_tree_insert_particles", "bad arguments");
  append(c, NbPositions, arrayX, arrayY, arrayZ, 1, 1, 1);
}

void scalfmm_tree_insert_particles_xyz(scalfmm_handle Handle, int NbPositions, double *XYZ, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_tree_insert_particles_xyz")) return;
  if (NbPositions < 0 || (NbPositions && !XYZ))
    return report(c, B200FMM_ERR_INVALID, "scalfmm_tree_insert_particles_xyz", "bad arguments");
  append(c, NbPositions, XYZ, XYZ + 1, XYZ + 2, 3, 3, 3);
}

// ---- per-particle values ------------------------------------------------------------------------------
void scalfmm_set_physical_values(scalfmm_handle Handle, int n, double *v, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_set_physical_values") || !check_count(c, n, "scalfmm_set_physical_values")) return;
  std::memcpy(c->q.data(), v, sizeof(double) * n);
  c->charges_dirty = true;
}
void scalfmm_get_physical_values(scalfmm_handle Handle, int n, double *v, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_physical_values") || !check_count(c, n, "scalfmm_get_physical_values")) return;
  std::memcpy(v, c->q.data(), sizeof(double) * n);
}
void scalfmm_set_physical_values_npart(scalfmm_handle Handle, int n, int *idx, double *v, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_set_physical_values_npart") || !check_indices(c, n, idx, "scalfmm_set_physical_values_npart"))
    return;
  for (int k = 0; k < n; ++k) c->q[idx[k]] = v[k];
  c->charges_dirty = true;
}
void scalfmm_get_physical_values_npart(scalfmm_handle Handle, int n, int *idx, double *v, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_physical_values_npart") || !check_indices(c, n, idx, "scalfmm_get_physical_values_npart"))
    return;
  for (int k = 0; k < n; ++k) v[k] = c->q[idx[k]];
}

void scalfmm_get_forces_xyz(scalfmm_handle Handle, int n, double *f, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_forces_xyz") || !check_count(c, n, "scalfmm_get_forces_xyz")) return;
  for (int i = 0; i < n; ++i) {
    f[3 * i] = c->fx[i];
    f[3 * i + 1] = c->fy[i];
    f[3 * i + 2] = c->fz[i];
  }
}
void scalfmm_get_forces_xyz_npart(scalfmm_handle Handle, int n, int *idx, double *f, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_forces_xyz_npart") || !check_indices(c, n, idx, "scalfmm_get_forces_xyz_npart")) return;
  for (int k = 0; k < n; ++k) {
    f[3 * k] = c->fx[idx[k]];
    f[3 * k + 1] = c->fy[idx[k]];
    f[3 * k + 2] = c->fz[idx[k]];
  }
}
void scalfmm_get_forces(scalfmm_handle Handle, int n, double *fX, double *fY, double *fZ, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_forces") || !check_count(c, n, "scalfmm_get_forces")) return;
  std::memcpy(fX, c->fx.data(), sizeof(double) * n);
  std::memcpy(fY, c->fy.data(), sizeof(double) * n);
  std::memcpy(fZ, c->fz.data(), sizeof(double) * n);
}
void scalfmm_get_forces_npart(scalfmm_handle Handle, int n, int *idx, double *fX, double *fY, double *fZ, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_forces_npart") || !check_indices(c, n, idx, "scalfmm_get_forces_npart")) return;
  for (int k = 0; k < n; ++k) {
    fX[k] = c->fx[idx[k]];
    fY[k] = c->fy[idx[k]];
    fZ[k] = c->fz[idx[k]];
  }
}
void scalfmm_set_forces_xyz(scalfmm_handle Handle, int n, double *f, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_set_forces_xyz") || !check_count(c, n, "scalfmm_set_forces_xyz")) return;
  for (int i = 0; i < n; ++i) {
    c->fx[i] = f[3 * i];
    c->fy[i] = f[3 * i + 1];
    c->fz[i] = f[3 * i + 2];
  }
}
void scalfmm_set_forces_xyz_npart(scalfmm_handle Handle, int n, int *idx, double *f, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_set_forces_xyz_npart") || !check_indices(c, n, idx, "scalfmm_set_forces_xyz_npart")) return;
  for (int k = 0; k < n; ++k) {
    c->fx[idx[k]] = f[3 * k];
    c->fy[idx[k]] = f[3 * k + 1];
    c->fz[idx[k]] = f[3 * k + 2];
  }
}
void scalfmm_set_forces(scalfmm_handle Handle, int n, double *fX, double *fY, double *fZ, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_set_forces") || !check_count(c, n, "scalfmm_set_forces")) return;
  std::memcpy(c->fx.data(), fX, sizeof(double) * n);
  std::memcpy(c->fy.data(), fY, sizeof(double) * n);
  std::memcpy(c->fz.data(), fZ, sizeof(double) * n);
}
void scalfmm_set_forces_npart(scalfmm_handle Handle, int n, int *idx, double *fX, double *fY, double *fZ, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_set_forces_npart") || !check_indices(c, n, idx, "scalfmm_set_forces_npart")) return;
  for (int k = 0; k < n; ++k) {
    c->fx[idx[k]] = fX[k];
    c->fy[idx[k]] = fY[k];
    c->fz[idx[k]] = fZ[k];
  }
}
void scalfmm_get_potentials(scalfmm_handle Handle, int n, double *v, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_potentials") || !check_count(c, n, "scalfmm_get_potentials")) return;
  std::memcpy(v, c->phi.data(), sizeof(double) * n);
}
void scalfmm_set_potentials(scalfmm_handle Handle, int n, double *v, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_set_potentials") || !check_count(c, n, "scalfmm_set_potentials")) return;
  std::memcpy(c->phi.data(), v, sizeof(double) * n);
}
void scalfmm_get_potentials_npart(scalfmm_handle Handle, int n, int *idx, double *v, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_potentials_npart") || !check_indices(c, n, idx, "scalfmm_get_potentials_npart")) return;
  for (int k = 0; k < n; ++k) v[k] = c->phi[idx[k]];
}
void scalfmm_set_potentials_npart(scalfmm_handle Handle, int n, int *idx, double *v, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_set_potentials_npart") || !check_indices(c, n, idx, "scalfmm_set_potentials_npart")) return;
  for (int k = 0; k < n; ++k) c->phi[idx[k]] = v[k];
}

// ---- moving particles ---------------------------------------------------------------------------------
static void move(CapiHandle *c, int n, const int *idx, const double *X, const double *Y, const double *Z, int stride,
                 bool add) {
  for (int k = 0; k < n; ++k) {
    const int i = idx ? idx[k] : k;
    if (add) {
      c->x[i] += X[(size_t)k * stride];
      c->y[i] += Y[(size_t)k * stride];
      c->z[i] += Z[(size_t)k * stride];
    } else {
      c->x[i] = X[(size_t)k * stride];
      c->y[i] = Y[(size_t)k * stride];
      c->z[i] = Z[(size_t)k * stride];
    }
  }
  c->tree_dirty = true;
}
void scalfmm_add_to_positions_xyz(scalfmm_handle Handle, int n, double *d, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_add_to_positions_xyz") && check_count(c, n, "scalfmm_add_to_positions_xyz"))
    move(c, n, nullptr, d, d + 1, d + 2, 3, true);
}
void scalfmm_add_to_positions(scalfmm_handle Handle, int n, double *X, double *Y, double *Z, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_add_to_positions") && check_count(c, n, "scalfmm_add_to_positions"))
    move(c, n, nullptr, X, Y, Z, 1, true);
}
void scalfmm_add_to_positions_xyz_npart(scalfmm_handle Handle, int n, int *idx, double *d, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_add_to_positions_xyz_npart") && check_indices(c, n, idx, "scalfmm_add_to_positions_xyz_npart"))
    move(c, n, idx, d, d + 1, d + 2, 3, true);
}
void scalfmm_add_to_positions_npart(scalfmm_handle Handle, int n, int *idx, double *X, double *Y, double *Z, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_add_to_positions_npart") && check_indices(c, n, idx, "scalfmm_add_to_positions_npart"))
    move(c, n, idx, X, Y, Z, 1, true);
}
void scalfmm_set_positions_xyz(scalfmm_handle Handle, int n, double *d, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_set_positions_xyz") && check_count(c, n, "scalfmm_set_positions_xyz"))
    move(c, n, nullptr, d, d + 1, d + 2, 3, false);
}
void scalfmm_set_positions(scalfmm_handle Handle, int n, double *X, double *Y, double *Z, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_set_positions") && check_count(c, n, "scalfmm_set_positions"))
    move(c, n, nullptr, X, Y, Z, 1, false);
}
void scalfmm_set_positions_xyz_npart(scalfmm_handle Handle, int n, int *idx, double *d, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_set_positions_xyz_npart") && check_indices(c, n, idx, "scalfmm_set_positions_xyz_npart"))
    move(c, n, idx, d, d + 1, d + 2, 3, false);
}
void scalfmm_set_positions_npart(scalfmm_handle Handle, int n, int *idx, double *X, double *Y, double *Z, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_set_positions_npart") && check_indices(c, n, idx, "scalfmm_set_positions_npart"))
    move(c, n, idx, X, Y, Z, 1, false);
}
void scalfmm_update_tree(scalfmm_handle handle) {
  // the tree of the moved particles is built on the GPU at the next execute
  CapiHandle *c = as_handle(handle);
  if (check(c, "scalfmm_update_tree")) c->tree_dirty = true;
}
void scalfmm_get_positions_xyz(scalfmm_handle Handle, int n, double *p, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_positions_xyz") || !check_count(c, n, "scalfmm_get_positions_xyz")) return;
  for (int i = 0; i < n; ++i) {
    p[3 * i] = c->x[i];
    p[3 * i + 1] = c->y[i];
    p[3 * i + 2] = c->z[i];
  }
}
void scalfmm_get_positions(scalfmm_handle Handle, int n, double *X, double *Y, double *Z, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_positions") || !check_count(c, n, "scalfmm_get_positions")) return;
  std::memcpy(X, c->x.data(), sizeof(double) * n);
  std::memcpy(Y, c->y.data(), sizeof(double) * n);
  std::memcpy(Z, c->z.data(), sizeof(double) * n);
}
void scalfmm_get_positions_xyz_npart(scalfmm_handle Handle, int n, int *idx, double *p, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_positions_xyz_npart") || !check_indices(c, n, idx, "scalfmm_get_positions_xyz_npart"))
    return;
  for (int k = 0; k < n; ++k) {
    p[3 * k] = c->x[idx[k]];
    p[3 * k + 1] = c->y[idx[k]];
    p[3 * k + 2] = c->z[idx[k]];
  }
}
void scalfmm_get_positions_npart(scalfmm_handle Handle, int n, int *idx, double *X, double *Y, double *Z, PartType) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_get_positions_npart") || !check_indices(c, n, idx, "scalfmm_get_positions_npart")) return;
  for (int k = 0; k < n; ++k) {
    X[k] = c->x[idx[k]];
    Y[k] = c->y[idx[k]];
    Z[k] = c->z[idx[k]];
  }
}

// ---- execution -----------------------------------------------------------------------------------------
void scalfmm_user_kernel_config(scalfmm_handle Handle, Scalfmm_Kernel_Descriptor, void *) {
  report(as_handle(Handle), B200FMM_ERR_UNSUPPORTED, "scalfmm_user_kernel_config",
         "user-defined kernels are not part of this library");
}
void scalfmm_execute_fmm(scalfmm_handle Handle) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_execute_fmm")) execute(c, B200FMM_ALL, "scalfmm_execute_fmm");
}
void scalfmm_execute_fmm_far_field(scalfmm_handle Handle) {
  CapiHandle *c = as_handle(Handle);
  if (check(c, "scalfmm_execute_fmm_far_field")) execute(c, B200FMM_FAR_FIELD, "scalfmm_execute_fmm_far_field");
}

void scalfmm_apply_on_leaf(scalfmm_handle Handle, Callback_apply_on_leaf function) {
  CapiHandle *c = as_handle(Handle);
  if (!check(c, "scalfmm_apply_on_leaf")) return;
  if (!function) return report(c, B200FMM_ERR_INVALID, "scalfmm_apply_on_leaf", "null callback");
  if (!c->h) return report(c, B200FMM_ERR_STATE, "scalfmm_apply_on_leaf", "scalfmm_build_tree was not called");
  const long long n = (long long)c->x.size();
  if (n == 0) return;
  b200fmm_status st = B200FMM_OK;
  if (c->tree_dirty) {
    st = b200fmm_set_particles(c->h, n, c->x.data(), c->y.data(), c->z.data(), c->q.data(), 0);
    if (st == B200FMM_OK) c->tree_dirty = c->charges_dirty = false;
  }
  std::vector<long long> ncells(c->height), perm(n);
  long long np = 0;
  if (st == B200FMM_OK) st = b200fmm_tree_info(c->h, ncells.data(), &np);
  const int LL = c->height - 1;
  const long long nleaves = st == B200FMM_OK ? ncells[LL] : 0;
  std::vector<long long> keys(nleaves), start(nleaves + 1);
  if (st == B200FMM_OK) st = b200fmm_get_cells(c->h, LL, keys.data(), nullptr, nullptr);
  if (st == B200FMM_OK) st = b200fmm_get_leaf_ranges(c->h, start.data());
  if (st == B200FMM_OK) st = b200fmm_get_permutation(c->h, perm.data());
  if (st != B200FMM_OK) return report(c, st, "scalfmm_apply_on_leaf");
  const double lw = c->width / (double)(1LL << LL);
  std::vector<FSize> idx;
  for (long long leaf = 0; leaf < nleaves; ++leaf) {
    int g[3] = {0, 0, 0};  // the leaf's cell coordinates from its Morton key (x is the high bit of each triple)
    for (int b = 0; b < 21; ++b)
      for (int a = 0; a < 3; ++a) g[a] |= (int)((keys[leaf] >> (3 * b + 2 - a)) & 1) << b;
    double llc[3];
    for (int a = 0; a < 3; ++a) llc[a] = c->center[a] - c->width / 2 + g[a] * lw;
    idx.assign(perm.begin() + start[leaf], perm.begin() + start[leaf + 1]);
    function(LL, (FSize)idx.size(), idx.data(), keys[leaf], llc, nullptr, nullptr, nullptr);
  }
}

// ---- release, monitoring, utilities ----------------------------------------------------------------------
void scalfmm_dealloc_handle(scalfmm_handle handle, Callback_free_cell) {
  CapiHandle *c = as_handle(handle);
  if (!c) return;
  if (c->h) b200fmm_destroy(c->h);
  delete c;
}
void scalfmm_apply_on_cell(scalfmm_handle handle, Callback_apply_on_cell) {
  // the built-in kernels' cells hold no user data (FScalFMMEngine::apply_on_cell does nothing for them)
  check(as_handle(handle), "scalfmm_apply_on_cell");
}
int scalfmm_get_nb_timers(scalfmm_handle) { return 9; }
void scalfmm_get_timers(scalfmm_handle handle, double *Timers) {
  CapiHandle *c = as_handle(handle);
  if (!check(c, "scalfmm_get_timers") || !Timers) return;
  for (int k = 0; k < 9; ++k) Timers[k] = c->timers_s[k];
}
void scalfmm_set_upper_limit(scalfmm_handle handle, int upperLimit) {
  CapiHandle *c = as_handle(handle);
  if (check(c, "scalfmm_set_upper_limit") && upperLimit != 2)
    report(c, B200FMM_ERR_UNSUPPORTED, "scalfmm_set_upper_limit", "the interpolation kernels use upper limit 2");
}
void scalfmm_utils_parentChildPosition(int childPosition, int *childFullPosition) {
  // child index bits (x y z) -> -1 / +1 per axis
  childFullPosition[0] = ((childPosition >> 2) & 1) ? 1 : -1;
  childFullPosition[1] = ((childPosition >> 1) & 1) ? 1 : -1;
  childFullPosition[2] = (childPosition & 1) ? 1 : -1;
}
void scalfmm_utils_interactionPosition(int interactionPosition, int *srcPosition) {
  // ((dx+3)*7 + (dy+3))*7 + (dz+3) -> (dx, dy, dz)
  srcPosition[0] = interactionPosition / 49 - 3;
  srcPosition[1] = (interactionPosition / 7) % 7 - 3;
  srcPosition[2] = interactionPosition % 7 - 3;
}
void scalfmm_print_everything(scalfmm_handle handle) {
  CapiHandle *c = as_handle(handle);
  if (!check(c, "scalfmm_print_everything")) return;
  std::printf("b200fmm C API handle: kernel %s, height %d, box width %g centre (%g, %g, %g), %zu particles\n",
              c->kernel == chebyshev ? "chebyshev" : "lagrange", c->height, c->width, c->center[0], c->center[1],
              c->center[2], c->x.size());
}

// ---- .fma / .bfma files ----------------------------------------------------------------------------------
// Binary (.bfma): unsigned int {sizeof(real) = 8, values per particle}, long long particle count, double half
// box width, double centre[3], then the particles' values (FFmaGenericLoader::readBinaryHeader, :480-500;
// FFmaGenericWriter::writerBinaryHeader).  ASCII (.fma): the same fields, whitespace separated, one particle
// per line (readAscciHeader, :470-479).  Files whose name contains ".bfma" are binary, as in the reference's
// loader (:247-256).
static bool is_binary(const char *path) { return std::strstr(path, ".bfma") != nullptr; }

b200fmm_status b200fmm_fma_read(const char *path, long long *n, int *nvalues, double *box_width, double *center,
                                double *data, long long cap) {
  if (!path || !n || !nvalues) return B200FMM_ERR_INVALID;
  const bool bin = is_binary(path);
  if (!bin && !std::strstr(path, ".fma")) return B200FMM_ERR_INVALID;
  FILE *f = std::fopen(path, bin ? "rb" : "r");
  if (!f) return B200FMM_ERR_INVALID;
  unsigned int type[2] = {0, 0};
  long long count = 0;
  double hdr[4] = {0, 0, 0, 0};
  bool ok;
  if (bin) {
    ok = std::fread(type, sizeof(unsigned int), 2, f) == 2 && std::fread(&count, sizeof(long long), 1, f) == 1 &&
         std::fread(hdr, sizeof(double), 4, f) == 4;
  } else {
    ok = std::fscanf(f, "%u %u %lld %lf %lf %lf %lf", &type[0], &type[1], &count, &hdr[0], &hdr[1], &hdr[2], &hdr[3]) == 7;
  }
  ok = ok && type[0] == sizeof(double) && type[1] >= 4 && type[1] <= 64 && count >= 0;
  if (!ok) {
    std::fclose(f);
    return B200FMM_ERR_INVALID;
  }
  *n = count;
  *nvalues = (int)type[1];
  if (box_width) *box_width = 2.0 * hdr[0];
  if (center)
    for (int d = 0; d < 3; ++d) center[d] = hdr[1 + d];
  b200fmm_status st = B200FMM_OK;
  if (data) {
    const long long total = count * (long long)type[1];
    if (cap < total) {
      st = B200FMM_ERR_INVALID;
    } else if (bin) {
      if ((long long)std::fread(data, sizeof(double), (size_t)total, f) != total) st = B200FMM_ERR_INVALID;
    } else {
      for (long long k = 0; k < total && st == B200FMM_OK; ++k)
        if (std::fscanf(f, "%lf", data + k) != 1) st = B200FMM_ERR_INVALID;
    }
  }
  std::fclose(f);
  return st;
}

b200fmm_status b200fmm_fma_write(const char *path, long long n, int nvalues, double box_width, const double *center,
                                 const double *data) {
  if (!path || n < 0 || nvalues < 4 || nvalues > 64 || !center || (n > 0 && !data)) return B200FMM_ERR_INVALID;
  const bool bin = is_binary(path);
  if (!bin && !std::strstr(path, ".fma")) return B200FMM_ERR_INVALID;
  FILE *f = std::fopen(path, bin ? "wb" : "w");
  if (!f) return B200FMM_ERR_INVALID;
  const unsigned int type[2] = {(unsigned int)sizeof(double), (unsigned int)nvalues};
  const double half = 0.5 * box_width;
  bool ok;
  if (bin) {
    const double hdr[4] = {half, center[0], center[1], center[2]};
    ok = std::fwrite(type, sizeof(unsigned int), 2, f) == 2 && std::fwrite(&n, sizeof(long long), 1, f) == 1 &&
         std::fwrite(hdr, sizeof(double), 4, f) == 4 &&
         (long long)std::fwrite(data, sizeof(double), (size_t)(n * nvalues), f) == n * nvalues;
  } else {
    // 17 significant digits, so that a round trip through the text form is exact
    ok = std::fprintf(f, "%u   %u\n%lld   %.17g   %.17g  %.17g %.17g\n", type[0], type[1], n, half, center[0],
                      center[1], center[2]) > 0;
    for (long long i = 0; i < n && ok; ++i) {
      for (int v = 0; v < nvalues && ok; ++v) ok = std::fprintf(f, "%.17g    ", data[i * nvalues + v]) > 0;
      ok = ok && std::fputc('\n', f) != EOF;
    }
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? B200FMM_OK : B200FMM_ERR_INVALID;
}

}  // extern "C"
