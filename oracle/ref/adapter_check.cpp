// Drop-in check of the FB200Kernel adapter (include/b200fmm_scalfmm.hpp): the reference's own algorithm
// driver runs twice on two copies of the same octree, once with the reference's kernel and once with the
// adapter over the GPU library, and the two results are compared.  Compiled against the ScalFMM sources
// where they lie (never copied) and linked to the GPU library; test infrastructure only.
//
//   kind 0: FChebSymKernel   (Src/Kernels/Chebyshev/FChebSymKernel.hpp); the adapter is given the
//           reference's own compressed operators, exported from its SymmetryHandler
//           (Src/Kernels/Chebyshev/FChebSymM2LHandler.hpp:303-344), so that FP64 results agree to rounding
//   kind 1: FChebDenseKernel (Src/Kernels/Chebyshev/FChebDenseKernel.hpp)
//   driver 0: FFmmAlgorithm (Src/Core/FFmmAlgorithm.hpp); driver 1: FFmmAlgorithmThread with one thread;
//   driver 2: FGroupSeqAlgorithm (Src/GroupTree/Core/FGroupSeqAlgorithm.hpp) over the blocked tree FGroupTree
//           with FChebCellPOD cells and FP2PGroupParticleContainer leaves, against FB200GroupKernel
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
#include "Kernels/P2P/FP2PParticleContainer.hpp"
#include "GroupTree/Core/FGroupTree.hpp"
#include "GroupTree/Core/FGroupSeqAlgorithm.hpp"
#include "GroupTree/Core/FP2PGroupParticleContainer.hpp"
#include "GroupTree/Chebyshev/FChebCellPOD.hpp"

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

// The reference's compressed operators, exported from its SymmetryHandler, for the FP64 adapter.
template <int ORDER>
void reference_operators(std::vector<int> &ranks, std::vector<double> &uv, double eps) {
  typedef FInterpMatrixKernelR<double> MatrixKernelClass;
  const MatrixKernelClass MatrixKernel;
  SymmetryHandler<double, ORDER, HOMOGENEOUS> handler(&MatrixKernel, eps, double(1.), 3);
  constexpr int nnodes = ORDER * ORDER * ORDER;
  ranks.assign(343, 0);
  uv.clear();
  for (int t = 0; t < 343; ++t) {
    ranks[t] = handler.getLowRank(0, t);
    const double *K = handler.getK(0, t);
    if (K != nullptr && ranks[t] > 0) uv.insert(uv.end(), K, K + 2LL * ranks[t] * nnodes);
    else ranks[t] = 0;
  }
}

// The blocked tree: two FGroupTree built from the same particles (blocks of `block` cells), the reference's
// FChebSymKernel and the group adapter each driven by FGroupSeqAlgorithm.
template <int ORDER>
int run_group(int precision, int height, int block, long long n, const double *x, const double *y, const double *z,
              const double *q, double *errs) {
  typedef double FReal;
  constexpr int nnodes = ORDER * ORDER * ORDER;
  typedef FInterpMatrixKernelR<FReal> MatrixKernelClass;
  typedef FChebCellPODCore CellSymbClass;
  typedef FChebCellPODPole<FReal, ORDER> CellUpClass;
  typedef FChebCellPODLocal<FReal, ORDER> CellDownClass;
  typedef FChebCellPOD<FReal, ORDER> CellClass;
  typedef FP2PGroupParticleContainer<FReal> ContainerClass;
  typedef FGroupTree<FReal, CellClass, CellSymbClass, CellUpClass, CellDownClass, ContainerClass, 1, 4, FReal>
      TreeClass;
  typedef FChebSymKernel<FReal, CellClass, ContainerClass, MatrixKernelClass, ORDER> RefKernel;
  typedef b200fmm_scalfmm::FB200GroupKernel<CellClass, ContainerClass, ORDER> GpuKernel;
  typedef FGroupSeqAlgorithm<TreeClass, typename TreeClass::CellGroupClass, CellClass, RefKernel,
                             typename TreeClass::ParticleGroupClass, ContainerClass>
      RefAlgo;
  typedef FGroupSeqAlgorithm<TreeClass, typename TreeClass::CellGroupClass, CellClass, GpuKernel,
                             typename TreeClass::ParticleGroupClass, ContainerClass>
      GpuAlgo;

  const MatrixKernelClass MatrixKernel;
  const double width = 1.0;
  const FPoint<FReal> center(0.5, 0.5, 0.5);
  const FReal eps = std::pow(10.0, -ORDER);
  FP2PParticleContainer<FReal> all;
  for (long long i = 0; i < n; ++i) all.push(FPoint<FReal>(x[i], y[i], z[i]), q[i]);
  TreeClass tref(height, width, center, block, &all);
  TreeClass tgpu(height, width, center, block, &all);

  RefKernel kref(height, width, center, &MatrixKernel, eps);
  GpuKernel kgpu(height, width, center, B200FMM_CHEB_SYM, precision, eps);
  if (precision == B200FMM_FP64) {
    std::vector<int> ranks;
    std::vector<double> uv;
    reference_operators<ORDER>(ranks, uv, eps);
    kgpu.setSymOperators(ranks.data(), uv.data(), (long long)uv.size());
  }
  RefAlgo aref(&tref, &kref);
  aref.execute();
  GpuAlgo agpu(&tgpu, &kgpu);
  agpu.execute();

  // particle outputs leaf by leaf (both trees hold the same leaves in the same order)
  std::vector<double> out[2][4];
  TreeClass *trees[2] = {&tref, &tgpu};
  for (int t = 0; t < 2; ++t)
    trees[t]->template forEachLeaf<ContainerClass>([&](ContainerClass *leaf) {
      for (FSize k = 0; k < leaf->getNbParticles(); ++k) {
        out[t][0].push_back(leaf->getPotentials()[k]);
        out[t][1].push_back(leaf->getForcesX()[k]);
        out[t][2].push_back(leaf->getForcesY()[k]);
        out[t][3].push_back(leaf->getForcesZ()[k]);
      }
    });
  if (out[0][0].size() != (size_t)n || out[1][0].size() != (size_t)n) return -7;
  for (int a = 0; a < 4; ++a) {
    Sums s;
    for (long long i = 0; i < n; ++i) s.add(out[0][a][(size_t)i], out[1][a][(size_t)i]);
    errs[a] = s.rel();
  }
  // cell expansions of levels 2..height-1, block by block
  std::vector<std::vector<double>> mul(2), loc(2);
  std::vector<long long> keys[2];
  for (int t = 0; t < 2; ++t)
    trees[t]->forEachCellWithLevel([&](CellClass c, const int level) {
      if (level < 2) return;
      keys[t].push_back(c.getMortonIndex() * 16 + level);
      mul[t].insert(mul[t].end(), c.getMultipole(0), c.getMultipole(0) + nnodes);
      loc[t].insert(loc[t].end(), c.getLocal(0), c.getLocal(0) + nnodes);
    });
  if (keys[0] != keys[1]) return -6;
  Sums sm, sl;
  for (size_t i = 0; i < mul[0].size(); ++i) {
    sm.add(mul[0][i], mul[1][i]);
    sl.add(loc[0][i], loc[1][i]);
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
    if (driver == 2) {  // the blocked tree, blocks of 30 cells (several blocks per level)
      if (kind == 0 && order == 4) return run_group<4>(precision, height, 30, n, x, y, z, q, errs);
      if (kind == 0 && order == 5) return run_group<5>(precision, height, 30, n, x, y, z, q, errs);
      if (kind == 0 && order == 7) return run_group<7>(precision, height, 30, n, x, y, z, q, errs);
      g_msg = "order/kind not instantiated for the blocked tree";
      return -1;
    }
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
