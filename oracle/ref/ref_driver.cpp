// Reference-side driver: compiled against the ScalFMM sources where they lie (never copied), it
// exposes the reference's own FFmmAlgorithmThread + FChebSymKernel / FChebDenseKernel and its
// FP64 direct sum through a small extern "C" surface so that Python tests and bench.py can run
// the unmodified reference algorithm.  This is test infrastructure only: it is the checker and
// the timed CPU baseline, never part of the product path.
//
// What each entry point runs (paths relative to the reference project root):
//   ref_fmm            Examples/ChebyshevInterpolationFMM.cpp:103-140 (tree insert + execute); kind 0
//                      FChebSymKernel, 1 FChebDenseKernel, 2 FUnifKernel (Lagrange, FFT-based M2L,
//                      Src/Kernels/Uniform/FUnifKernel.hpp)
//   ref_sym_operators  Src/Kernels/Chebyshev/FChebSymM2LHandler.hpp:303-344 (SymmetryHandler)
//   ref_expansions     same run as ref_fmm, then FOctree::forEachCellWithLevel (FOctree.hpp:1713)
//   ref_direct         Examples/DirectComputation.cpp:104-142 (NonMutualParticles loop)
#include <algorithm>
#include <array>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include <omp.h>

#include "Utils/FGlobal.hpp"
#include "Utils/FPoint.hpp"
#include "Kernels/Chebyshev/FChebCell.hpp"
#include "Kernels/Chebyshev/FChebSymKernel.hpp"
#include "Kernels/Chebyshev/FChebDenseKernel.hpp"
#include "Kernels/Uniform/FUnifCell.hpp"
#include "Kernels/Uniform/FUnifKernel.hpp"
#include "Kernels/Interpolation/FInterpMatrixKernel.hpp"
#include "Kernels/P2P/FP2PParticleContainerIndexed.hpp"
#include "Kernels/P2P/FP2PR.hpp"
#include "Components/FSimpleLeaf.hpp"
#include "Containers/FOctree.hpp"
#include "Core/FFmmAlgorithmThread.hpp"
#include "Core/FFmmAlgorithm.hpp"

namespace {

using Clock = std::chrono::steady_clock;
double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

struct Problem {
  int height;
  double box_width;
  double center[3];
  double eps;
  int nthreads;
  int sequential;  // 1: FFmmAlgorithm (sequential driver), 0: FFmmAlgorithmThread
  long long n;
  const double *x, *y, *z, *q;  // q: [nvals][n]
  unsigned ops;
};

struct Outputs {
  double *phi, *fx, *fy, *fz;  // [nvals][n], original particle order
  double *times;               // [3]: kernel construction, insertion, execute
  // optional expansion dump
  long long cap;
  long long *count;
  int *levels;
  long long *mortons;
  double *multipoles, *locals;  // [cap][nvals][nnodes]
};

// The Chebyshev kernels take the compression accuracy; the Lagrange kernel has no compression
// (FUnifKernel.hpp:57-67).
template <class KernelClass, int KIND, class MK>
KernelClass make_kernel(int height, double width, const FPoint<double> &center, const MK *mk, double eps) {
  if constexpr (KIND == 2) {
    (void)eps;
    return KernelClass(height, width, center, mk);
  } else {
    return KernelClass(height, width, center, mk, eps);
  }
}

template <int ORDER, int NVALS, int KIND>
int run_fmm(const Problem &p, Outputs &o) {
  typedef double FReal;
  constexpr int nnodes = ORDER * ORDER * ORDER;
  typedef FP2PParticleContainerIndexed<FReal, 1, 1, NVALS> ContainerClass;
  typedef FSimpleLeaf<FReal, ContainerClass> LeafClass;
  typedef typename std::conditional<KIND == 2, FUnifCell<FReal, ORDER, 1, 1, NVALS>,
                                    FChebCell<FReal, ORDER, 1, 1, NVALS>>::type CellClass;
  typedef FOctree<FReal, CellClass, ContainerClass, LeafClass> OctreeClass;
  typedef FInterpMatrixKernelR<FReal> MatrixKernelClass;
  typedef typename std::conditional<
      KIND == 0, FChebSymKernel<FReal, CellClass, ContainerClass, MatrixKernelClass, ORDER, NVALS>,
      typename std::conditional<KIND == 1,
                                FChebDenseKernel<FReal, CellClass, ContainerClass, MatrixKernelClass, ORDER, NVALS>,
                                FUnifKernel<FReal, CellClass, ContainerClass, MatrixKernelClass, ORDER, NVALS>>::type>::type
      KernelClass;

  omp_set_num_threads(p.nthreads);
  const MatrixKernelClass MatrixKernel;
  const FPoint<FReal> center(p.center[0], p.center[1], p.center[2]);

  auto t0 = Clock::now();
  OctreeClass tree(p.height, std::min(2, p.height - 1), p.box_width, center);
  constexpr int NA = ContainerClass::NbAttributes;
  for (long long i = 0; i < p.n; ++i) {
    std::array<FReal, NA> attr{};
    for (int v = 0; v < NVALS; ++v) attr[v] = p.q[(long long)v * p.n + i];
    tree.insert(FPoint<FReal>(p.x[i], p.y[i], p.z[i]), FSize(i), attr);
  }
  const double t_insert = seconds_since(t0);

  t0 = Clock::now();
  KernelClass kernels = make_kernel<KernelClass, KIND>(p.height, p.box_width, center, &MatrixKernel, p.eps);
  const double t_kernel = seconds_since(t0);

  t0 = Clock::now();
  if (p.sequential) {
    FFmmAlgorithm<OctreeClass, CellClass, ContainerClass, KernelClass, LeafClass> algo(&tree, &kernels);
    algo.execute(p.ops);
  } else {
    FFmmAlgorithmThread<OctreeClass, CellClass, ContainerClass, KernelClass, LeafClass> algo(&tree, &kernels, 10);
    algo.execute(p.ops);
  }
  const double t_exec = seconds_since(t0);
  if (o.times) {
    o.times[0] = t_kernel;
    o.times[1] = t_insert;
    o.times[2] = t_exec;
  }

  if (o.phi) {
    tree.forEachLeaf([&](LeafClass *leaf) {
      const ContainerClass *c = leaf->getTargets();
      const FVector<FSize> &idx = c->getIndexes();
      for (int v = 0; v < NVALS; ++v) {
        const FReal *pot = c->getPotentials(v);
        const FReal *fx = c->getForcesX(v);
        const FReal *fy = c->getForcesY(v);
        const FReal *fz = c->getForcesZ(v);
        for (FSize k = 0; k < c->getNbParticles(); ++k) {
          const long long j = (long long)v * p.n + idx[k];
          o.phi[j] = pot[k];
          o.fx[j] = fx[k];
          o.fy[j] = fy[k];
          o.fz[j] = fz[k];
        }
      }
    });
  }
  if (o.count) {
    long long k = 0;
    tree.forEachCellWithLevel([&](CellClass *cell, const int level) {
      if (k < o.cap) {
        o.levels[k] = level;
        o.mortons[k] = cell->getMortonIndex();
        for (int v = 0; v < NVALS; ++v) {
          std::memcpy(o.multipoles + (k * NVALS + v) * nnodes, cell->getMultipole(v), sizeof(FReal) * nnodes);
          std::memcpy(o.locals + (k * NVALS + v) * nnodes, cell->getLocal(v), sizeof(FReal) * nnodes);
        }
      }
      ++k;
    });
    *o.count = k;
  }
  return 0;
}

template <int ORDER>
int dispatch_nvals(int kind, int nvals, const Problem &p, Outputs &o) {
  if (nvals == 1)
    return kind == 0 ? run_fmm<ORDER, 1, 0>(p, o) : kind == 1 ? run_fmm<ORDER, 1, 1>(p, o) : run_fmm<ORDER, 1, 2>(p, o);
  if (nvals == 16 && kind == 0) return run_fmm<ORDER, 16, 0>(p, o);
  return -2;
}

int dispatch(int kind, int order, int nvals, const Problem &p, Outputs &o) {
  try {
    switch (order) {
      case 3: return dispatch_nvals<3>(kind, nvals, p, o);
      case 4: return dispatch_nvals<4>(kind, nvals, p, o);
      case 5: return dispatch_nvals<5>(kind, nvals, p, o);
      case 6: return dispatch_nvals<6>(kind, nvals, p, o);
      case 7: return dispatch_nvals<7>(kind, nvals, p, o);
      case 8: return dispatch_nvals<8>(kind, nvals, p, o);
      default: return -1;
    }
  } catch (const std::exception &e) {
    std::fprintf(stderr, "ref_fmm: %s\n", e.what());
    return -3;
  }
}

template <int ORDER>
int sym_ops(double eps, int *ranks, unsigned *pindices, unsigned *pvectors, double *uv, long long cap) {
  typedef double FReal;
  constexpr int nnodes = ORDER * ORDER * ORDER;
  typedef FInterpMatrixKernelR<FReal> MatrixKernelClass;
  const MatrixKernelClass MatrixKernel;
  SymmetryHandler<FReal, ORDER, HOMOGENEOUS> handler(&MatrixKernel, eps, FReal(1.), 3);
  long long off = 0;
  for (int t = 0; t < 343; ++t) {
    pindices[t] = handler.pindices[t];
    for (int n = 0; n < nnodes; ++n) pvectors[t * nnodes + n] = handler.pvectors[t][n];
    ranks[t] = handler.getLowRank(0, t);
    const FReal *K = handler.getK(0, t);
    if (K != nullptr && ranks[t] > 0) {
      const long long len = 2LL * ranks[t] * nnodes;
      if (off + len > cap) return -4;
      std::memcpy(uv + off, K, sizeof(FReal) * len);
      off += len;
    }
  }
  return 0;
}

}  // namespace

extern "C" {

int ref_fmm(int kind, int order, int nvals, int height, double box_width, const double *center, double eps,
            int nthreads, int sequential, long long n, const double *x, const double *y, const double *z,
            const double *q, unsigned ops, double *phi, double *fx, double *fy, double *fz, double *times) {
  Problem p{height, box_width, {center[0], center[1], center[2]}, eps, nthreads, sequential, n, x, y, z, q, ops};
  Outputs o{phi, fx, fy, fz, times, 0, nullptr, nullptr, nullptr, nullptr, nullptr};
  return dispatch(kind, order, nvals, p, o);
}

int ref_expansions(int kind, int order, int nvals, int height, double box_width, const double *center, double eps,
                   int nthreads, long long n, const double *x, const double *y, const double *z, const double *q,
                   unsigned ops, long long cap, long long *count, int *levels, long long *mortons,
                   double *multipoles, double *locals) {
  Problem p{height, box_width, {center[0], center[1], center[2]}, eps, nthreads, 0, n, x, y, z, q, ops};
  Outputs o{nullptr, nullptr, nullptr, nullptr, nullptr, cap, count, levels, mortons, multipoles, locals};
  return dispatch(kind, order, nvals, p, o);
}

int ref_sym_operators(int order, double eps, int *ranks, unsigned *pindices, unsigned *pvectors, double *uv,
                      long long cap) {
  try {
    switch (order) {
      case 3: return sym_ops<3>(eps, ranks, pindices, pvectors, uv, cap);
      case 4: return sym_ops<4>(eps, ranks, pindices, pvectors, uv, cap);
      case 5: return sym_ops<5>(eps, ranks, pindices, pvectors, uv, cap);
      case 6: return sym_ops<6>(eps, ranks, pindices, pvectors, uv, cap);
      case 7: return sym_ops<7>(eps, ranks, pindices, pvectors, uv, cap);
      case 8: return sym_ops<8>(eps, ranks, pindices, pvectors, uv, cap);
      default: return -1;
    }
  } catch (const std::exception &e) {
    std::fprintf(stderr, "ref_sym_operators: %s\n", e.what());
    return -3;
  }
}

// FP64 direct sum over all sources for the listed targets (all targets when ntargets < 0).
// Follows Examples/DirectComputation.cpp:112-128 with FP2PR::NonMutualParticles (FP2PR.hpp:45-69).
int ref_direct(long long n, const double *x, const double *y, const double *z, const double *q,
               long long ntargets, const long long *targets, int nthreads, double *phi, double *fx, double *fy,
               double *fz) {
  const long long nt = ntargets < 0 ? n : ntargets;
  omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
  for (long long k = 0; k < nt; ++k) {
    const long long i = ntargets < 0 ? k : targets[k];
    double p = 0, gx = 0, gy = 0, gz = 0;
    for (long long j = 0; j < n; ++j) {
      if (j == i) continue;
      FP2PR::NonMutualParticles<double>(x[i], y[i], z[i], q[i], &gx, &gy, &gz, &p, x[j], y[j], z[j], q[j]);
    }
    phi[k] = p;
    fx[k] = gx;
    fy[k] = gy;
    fz[k] = gz;
  }
  return 0;
}

}  // extern "C"
