// Drop-in check of the FB200Kernel adapter (include/b200fmm_scalfmm.hpp): the reference's own algorithm
// driver runs twice on two copies of the same octree, once with the reference's kernel and once with the
// adapter over the GPU library, and the two results are compared.  Compiled against the ScalFMM sources
// where they lie (never copied) and linked to the GPU library; test infrastructure only.
//
//   kind 0: FChebSymKernel   (Src/Kernels/Chebyshev/FChebSymKernel.hpp); the adapter is given the
//           reference's own compressed operators, exported from its SymmetryHandler
//           (Src/Kernels/Chebyshev/FChebSymM2LHandler.hpp:303-344), so that FP64 results agree to rounding
//   kind 1: FChebDenseKernel (Src/Kernels/Chebyshev/FChebDenseKernel.hpp)
//   driver 0: FFmmAlgorithm (Src/Core/FFmmAlgorithm.hpp); driver 1: FFmmAlgorithmThread with one thread
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include <omp.h>

#include "Utils/FGlobal.hpp"
#include "Utils/FPoint.hpp"
#include "Kernels/Chebyshev/FChebCell.hpp"
#include "Kernels/Chebyshev/FChebSymKernel.hpp"
#include "Kernels/Chebyshev/FChebDenseKernel.hpp"
#include "Kernels/Interpolation/FInterpMatrixKernel.hpp"
#include "Kernels/P2P/FP2PParticleContainerIndexed.hpp"
#include "Components/FSimpleLeaf.hpp"
#include "Containers/FOctree.hpp"
#include "Core/FFmmAlgorithmThread.hpp"
#include "Core/FFmmAlgorithm.hpp"

#include "b200fmm_scalfmm.hpp"

namespace {

struct Sums {
  double num = 0, den = 0;
  void add(double ref, double v) {
    num += (ref - v) * (ref - v);
    den += ref * ref;
  }
  double rel() const { return den > 0 ? std::sqrt(num / den) : std::sqrt(num); }
};

template <int ORDER, int KIND>
int run(int precision, int driver, int height, long long n, const double *x, const double *y, const double *z,
        const double *q, double *errs) {
  typedef double FReal;
  constexpr int nnodes = ORDER * ORDER * ORDER;
  typedef FP2PParticleContainerIndexed<FReal> ContainerClass;
  typedef FSimpleLeaf<FReal, ContainerClass> LeafClass;
  typedef FChebCell<FReal, ORDER> CellClass;
  typedef FOctree<FReal, CellClass, ContainerClass, LeafClass> OctreeClass;
  typedef FInterpMatrixKernelR<FReal> MatrixKernelClass;
  typedef typename std::conditional<KIND == 0,
                                    FChebSymKernel<FReal, CellClass, ContainerClass, MatrixKernelClass, ORDER>,
                                    FChebDenseKernel<FReal, CellClass, ContainerClass, MatrixKernelClass, ORDER>>::type
      RefKernel;
  typedef b200fmm_scalfmm::FB200Kernel<CellClass, ContainerClass, ORDER> GpuKernel;

  omp_set_num_threads(1);
  const MatrixKernelClass MatrixKernel;
  const double width = 1.0;
  const FPoint<FReal> center(0.5, 0.5, 0.5);
  const FReal eps = std::pow(10.0, -ORDER);
  OctreeClass tref(height, std::min(2, height - 1), width, center);
  OctreeClass tgpu(height, std::min(2, height - 1), width, center);
  for (long long i = 0; i < n; ++i) {
    tref.insert(FPoint<FReal>(x[i], y[i], z[i]), FSize(i), q[i]);
    tgpu.insert(FPoint<FReal>(x[i], y[i], z[i]), FSize(i), q[i]);
  }

  RefKernel kref(height, width, center, &MatrixKernel, eps);
  GpuKernel kgpu(height, width, center, KIND == 0 ? B200FMM_CHEB_SYM : B200FMM_CHEB_DENSE, precision, eps);
  // FP64 is given the reference's own compressed operators; MIXED compresses the same kernel evaluations
  // itself (the same pACA + SVD) and runs them in their low-rank form on the tensor cores
  if (KIND == 0 && precision == B200FMM_FP64) {
    SymmetryHandler<FReal, ORDER, HOMOGENEOUS> handler(&MatrixKernel, eps, FReal(1.), 3);
    std::vector<int> ranks(343, 0);
    std::vector<double> uv;
    for (int t = 0; t < 343; ++t) {
      ranks[t] = handler.getLowRank(0, t);
      const FReal *K = handler.getK(0, t);
      if (K != nullptr && ranks[t] > 0) uv.insert(uv.end(), K, K + 2LL * ranks[t] * nnodes);
      else ranks[t] = 0;
    }
    kgpu.setSymOperators(ranks.data(), uv.data(), (long long)uv.size());
  }

  if (driver == 0) {
    FFmmAlgorithm<OctreeClass, CellClass, ContainerClass, RefKernel, LeafClass> aref(&tref, &kref);
    aref.execute();
    FFmmAlgorithm<OctreeClass, CellClass, ContainerClass, GpuKernel, LeafClass> agpu(&tgpu, &kgpu);
    agpu.execute();
  } else {
    FFmmAlgorithmThread<OctreeClass, CellClass, ContainerClass, RefKernel, LeafClass> aref(&tref, &kref);
    aref.execute();
    FFmmAlgorithmThread<OctreeClass, CellClass, ContainerClass, GpuKernel, LeafClass> agpu(&tgpu, &kgpu);
    agpu.execute();
  }

  // particle outputs, by original index
  std::vector<double> out[2][4];
  OctreeClass *trees[2] = {&tref, &tgpu};
  for (int t = 0; t < 2; ++t) {
    for (auto &v : out[t]) v.assign((size_t)n, 0.0);
    trees[t]->forEachLeaf([&](LeafClass *leaf) {
      const ContainerClass *c = leaf->getTargets();
      const FVector<FSize> &idx = c->getIndexes();
      for (FSize k = 0; k < c->getNbParticles(); ++k) {
        out[t][0][(size_t)idx[k]] = c->getPotentials()[k];
        out[t][1][(size_t)idx[k]] = c->getForcesX()[k];
        out[t][2][(size_t)idx[k]] = c->getForcesY()[k];
        out[t][3][(size_t)idx[k]] = c->getForcesZ()[k];
      }
    });
  }
  for (int a = 0; a < 4; ++a) {
    Sums s;
    for (long long i = 0; i < n; ++i) s.add(out[0][a][(size_t)i], out[1][a][(size_t)i]);
    errs[a] = s.rel();
  }
  // cell expansions, every level (both trees iterate their cells in the same order)
  std::vector<const CellClass *> cells[2];
  for (int t = 0; t < 2; ++t) trees[t]->forEachCell([&](CellClass *c) { cells[t].push_back(c); });
  if (cells[0].size() != cells[1].size()) return -5;
  Sums sm, sl;
  for (size_t i = 0; i < cells[0].size(); ++i) {
    if (cells[0][i]->getMortonIndex() != cells[1][i]->getMortonIndex()) return -6;
    for (int k = 0; k < nnodes; ++k) {
      sm.add(cells[0][i]->getMultipole(0)[k], cells[1][i]->getMultipole(0)[k]);
      sl.add(cells[0][i]->getLocal(0)[k], cells[1][i]->getLocal(0)[k]);
    }
  }
  errs[4] = sm.rel();
  errs[5] = sl.rel();
  return 0;
}

std::string g_msg;

}  // namespace

extern "C" {

// errs[6]: rel-L2 of potential, fx, fy, fz over all particles, of the multipoles and of the locals over
// all cells.  Returns 0, or a negative code with adapter_check_message() set.
int adapter_check(int kind, int order, int precision, int driver, int height, long long n, const double *x,
                  const double *y, const double *z, const double *q, double *errs) {
  try {
    if (kind == 0 && order == 4) return run<4, 0>(precision, driver, height, n, x, y, z, q, errs);
    if (kind == 0 && order == 5) return run<5, 0>(precision, driver, height, n, x, y, z, q, errs);
    if (kind == 0 && order == 7) return run<7, 0>(precision, driver, height, n, x, y, z, q, errs);
    if (kind == 1 && order == 4) return run<4, 1>(precision, driver, height, n, x, y, z, q, errs);
    if (kind == 1 && order == 5) return run<5, 1>(precision, driver, height, n, x, y, z, q, errs);
    g_msg = "order/kind not instantiated";
    return -1;
  } catch (const std::exception &e) {
    g_msg = e.what();
    return -3;
  }
}

const char *adapter_check_message(void) { return g_msg.c_str(); }

}  // extern "C"
