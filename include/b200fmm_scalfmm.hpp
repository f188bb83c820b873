/* FB200Kernel -- ScalFMM kernel adapter over the b200fmm C ABI (header only, C++17).
 *
 * It offers the operator surface of ScalFMM's FAbstractKernels (Src/Components/FAbstractKernels.hpp:23-210):
 * P2M :36, M2M :50, M2L :81-83, NeedFinishedM2LEvent / finishedLevelM2L :93-102, L2L :116, L2P :124,
 * P2P :147-150, P2POuter :171-174, P2PRemote :203-208.  The reference's algorithm drivers are templates
 * on the kernel class, so they call it unchanged: FFmmAlgorithm (Src/Core/FFmmAlgorithm.hpp) and
 * FFmmAlgorithmThread (Src/Core/FFmmAlgorithmThread.hpp) with one OpenMP thread.
 *
 * How the per-cell calls of the reference driver map onto the level-batched GPU operators:
 *   - P2M calls (the bottom pass) record the leaf cells and their particle containers.  At the first
 *     call of another operator the particles are gathered leaf by leaf, the GPU tree is built from them
 *     (b200fmm_set_particles), b200fmm_p2m runs and the leaf multipoles are written into the cells.
 *   - M2M / L2L calls of one level are recorded; when a call of another level or operator arrives the
 *     level runs on the GPU (b200fmm_m2m / b200fmm_l2l) and the parent multipoles / child locals are
 *     written into the recorded cells, matched by Morton index.
 *   - M2L calls are recorded and finishedLevelM2L(level) runs b200fmm_m2l for the level and writes the
 *     locals back (NeedFinishedM2LEvent() is true).
 *   - The first L2P (or P2P / P2POuter / P2PRemote) call of the direct pass runs the operator for every
 *     leaf at once and adds (+=) its potentials and forces into all the containers; later calls of that
 *     operator in the same pass do nothing.
 * The GPU tree is rebuilt from the containers at every bottom pass and is bit-identical to the
 * reference's (same Morton keys, leaves, neighbour and interaction lists), so the neighbour arrays the
 * driver passes are not needed.  Cell expansions are written (=) as the GPU holds them, which equals
 * the reference's += on cells that start from zero (the reference's drivers require reset cells).
 * A driver whose operation mask ends before the direct pass leaves the last M2M / L2L level on the
 * GPU until flush() is called.  One evaluation at a time: the kernel copies made by FFmmAlgorithmThread
 * share one state and one GPU handle, and calls are serialised by a mutex.
 *
 * Errors: a failing b200fmm call throws std::runtime_error with b200fmm_last_error(), as the reference's
 * precompute throws (Src/Kernels/Chebyshev/FChebSymM2LHandler.hpp:156-160); nothing aborts the process.
 *
 * CellClass needs getMortonIndex(), getMultipole(rhs), getLocal(rhs) (FChebCell,
 * Src/Kernels/Chebyshev/FChebCell.hpp:39-55); ContainerClass needs getNbParticles(), getPositions(),
 * getPhysicalValues(rhs), getPotentials(rhs), getForcesX/Y/Z(rhs) (FP2PParticleContainer,
 * Src/Kernels/P2P/FP2PParticleContainer.hpp).
 *
 * FB200GroupKernel is the same adapter for the blocked tree FGroupTree (Src/GroupTree/Core/FGroupTree.hpp),
 * driven by FGroupSeqAlgorithm (Src/GroupTree/Core/FGroupSeqAlgorithm.hpp:58-404).  There the cells and leaves
 * the driver passes are views built on the fly over the blocks' arrays -- FChebCellPOD
 * (Src/GroupTree/Chebyshev/FChebCellPOD.hpp) points at a cell's symbolic data, multipole and local inside
 * FGroupOfCells (Src/GroupTree/Core/FGroupOfCells.hpp:18-120); FP2PGroupParticleContainer points at a leaf's
 * slice of FGroupOfParticles (Src/GroupTree/Core/FGroupOfParticles.hpp:21-200) -- and live only for the call.
 * The group adapter therefore keeps copies of the views (their pointers stay valid, the blocks are the tree's),
 * and reads particles from and writes expansions and results into the block arrays through them.  The
 * driver splits the transfer and direct passes into in-block calls and out-of-block pairs (M2L / P2POuter
 * with one source); the level-batched GPU operators cover both, so the first P2P call of a direct pass runs
 * the whole near field and the P2POuter calls that complete it across blocks add nothing more.  The driver
 * calls no finishedLevelM2L: a level's M2L runs when the driver moves to the next level or operator.
 */
#ifndef B200FMM_SCALFMM_HPP
#define B200FMM_SCALFMM_HPP

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "b200fmm.h"

namespace b200fmm_scalfmm {

inline void check(b200fmm_status st, const char *what) {
  if (st != B200FMM_OK) throw std::runtime_error(std::string("FB200Kernel: ") + what + ": " + b200fmm_last_error());
}

// VIEWS = false: the driver's cells and containers are long-lived objects (FOctree), kept by pointer;
// VIEWS = true: they are views valid only during the call (FGroupTree), kept by value.
template <class CellClass, class ContainerClass, int ORDER, int NVALS = 1, bool VIEWS = false>
class FB200KernelT {
  enum class Op { None, P2M, M2M, M2L, L2L, Direct };
  using CellRef = typename std::conditional<VIEWS, CellClass, CellClass *>::type;
  using ContRef = typename std::conditional<VIEWS, ContainerClass, ContainerClass *>::type;
  static CellRef keep(CellClass *c) {
    if constexpr (VIEWS)
      return *c;
    else
      return c;
  }
  static ContRef keep(ContainerClass *c) {
    if constexpr (VIEWS)
      return *c;
    else
      return c;
  }
  static CellClass &use(CellRef &c) {
    if constexpr (VIEWS)
      return c;
    else
      return *c;
  }
  static ContainerClass &use(ContRef &c) {
    if constexpr (VIEWS)
      return c;
    else
      return *c;
  }

  struct State {
    b200fmm_handle h = nullptr;
    int height = 0;
    std::mutex mu;
    Op pending = Op::None;
    int pending_level = -1;
    bool tree_ready = false, l2p_done = false, p2p_done = false, p2p_outer_done = false;
    std::vector<CellRef> leaf_cells;
    std::vector<ContRef> leaf_tgt;  // the leaves' containers, sources and targets alike
    std::vector<CellRef> cells;     // cells waiting for the write-back of the pending operator
    std::vector<long long> m2l_flushed;
    ~State() {
      if (h) b200fmm_destroy(h);
    }
  };
  std::shared_ptr<State> s_;

  static constexpr int nnodes = ORDER * ORDER * ORDER;

 public:
  /* Mirrors FChebSymKernel(inTreeHeight, inBoxWidth, inBoxCenter, matrixKernel, inEpsilon)
   * (Src/Kernels/Chebyshev/FChebSymKernel.hpp:136-140); the matrix kernel is 1/r.  PointClass has
   * getX/getY/getZ (FPoint).  kernel: b200fmm_kernel, precision: b200fmm_precision. */
  template <class PointClass>
  FB200KernelT(int treeHeight, double boxWidth, const PointClass &boxCenter, int kernel = B200FMM_CHEB_SYM,
               int precision = B200FMM_FP64, double epsilon = -1.0, void *stream = nullptr, int device = -1)
      : s_(std::make_shared<State>()) {
    b200fmm_config cfg{};
    cfg.kernel = kernel;
    cfg.order = ORDER;
    cfg.height = treeHeight;
    cfg.nrhs = NVALS;
    cfg.precision = precision;
    cfg.box_width = boxWidth;
    cfg.center[0] = boxCenter.getX();
    cfg.center[1] = boxCenter.getY();
    cfg.center[2] = boxCenter.getZ();
    cfg.epsilon = epsilon;
    cfg.stream = stream;
    cfg.device = device;
    check(b200fmm_create(&cfg, &s_->h), "create");
    s_->height = treeHeight;
  }
  FB200KernelT(const FB200KernelT &) = default;  // copies share the state (FFmmAlgorithmThread copies kernels)

  b200fmm_handle handle() const { return s_->h; }

  /* Replace the compressed operators (the reference's storage layout, b200fmm_set_sym_operators). */
  void setSymOperators(const int *ranks, const double *uv, long long uv_len) {
    std::lock_guard<std::mutex> g(s_->mu);
    check(b200fmm_set_sym_operators(s_->h, ranks, uv, uv_len), "set_sym_operators");
  }

  static constexpr bool NeedFinishedM2LEvent() { return true; }

  void P2M(CellClass *const pole, const ContainerClass *const particles) {
    std::lock_guard<std::mutex> g(s_->mu);
    State &s = *s_;
    if (s.pending != Op::P2M) {  // a new bottom pass: a new evaluation
      s.leaf_cells.clear();
      s.leaf_tgt.clear();
      s.tree_ready = false;
      s.l2p_done = s.p2p_done = s.p2p_outer_done = false;
      s.m2l_flushed.clear();
      s.pending = Op::P2M;
    }
    s.leaf_cells.push_back(keep(pole));
    s.leaf_tgt.push_back(keep(const_cast<ContainerClass *>(particles)));
  }

  void M2M(CellClass *const pole, const CellClass *const *const /*child*/, const int level) {
    std::lock_guard<std::mutex> g(s_->mu);
    begin(Op::M2M, level);
    s_->cells.push_back(keep(pole));
  }

  void M2L(CellClass *const local, const CellClass * /*distantNeighbors*/[], const int /*neighborPositions*/[],
           const int /*size*/, const int level) {
    std::lock_guard<std::mutex> g(s_->mu);
    begin(Op::M2L, level);
    s_->cells.push_back(keep(local));
  }

  void finishedLevelM2L(const int level) {
    std::lock_guard<std::mutex> g(s_->mu);
    State &s = *s_;
    if (std::find(s.m2l_flushed.begin(), s.m2l_flushed.end(), level) != s.m2l_flushed.end()) return;
    if (s.pending != Op::M2L || s.pending_level != level) begin(Op::M2L, level);  // a level without M2L calls
    flush_pending();
  }

  void L2L(const CellClass *const /*local*/, CellClass **const child, const int level) {
    std::lock_guard<std::mutex> g(s_->mu);
    begin(Op::L2L, level);
    for (int k = 0; k < 8; ++k)
      if (child[k]) s_->cells.push_back(keep(child[k]));
  }

  void L2P(const CellClass *const /*local*/, ContainerClass *const /*particles*/) {
    std::lock_guard<std::mutex> g(s_->mu);
    begin(Op::Direct, -1);
    if (s_->l2p_done) return;
    run_direct([&] { check(b200fmm_l2p(s_->h), "l2p"); });
    s_->l2p_done = true;
  }

  template <class CoordinateClass>
  void P2P(const CoordinateClass & /*leafPosition*/, ContainerClass *const /*targets*/,
           const ContainerClass *const /*sources*/, ContainerClass *const /*directNeighbors*/[],
           const int /*neighborPositions*/[], const int /*size*/) {
    std::lock_guard<std::mutex> g(s_->mu);
    begin(Op::Direct, -1);
    if (s_->p2p_done) return;
    run_direct([&] { check(b200fmm_p2p(s_->h, 0), "p2p"); });
    s_->p2p_done = true;
  }

  /* Neighbours only (the inner-leaf part is left to the caller), as FChebSymKernel::P2POuter. */
  template <class CoordinateClass>
  void P2POuter(const CoordinateClass & /*leafPosition*/, ContainerClass *const /*targets*/,
                ContainerClass *const /*directNeighbors*/[], const int /*neighborPositions*/[], const int /*size*/) {
    std::lock_guard<std::mutex> g(s_->mu);
    begin(Op::Direct, -1);
    // the blocked driver completes its in-block P2P calls with cross-block P2POuter pairs: the whole near field
    // ran at the first P2P call already
    if (VIEWS && s_->p2p_done) return;
    if (s_->p2p_outer_done) return;
    run_direct([&] { check(b200fmm_p2p(s_->h, 1), "p2p (neighbours only)"); });
    s_->p2p_outer_done = true;
  }

  /* Targets <- neighbour sources, non-mutual (FChebSymKernel::P2PRemote); over all leaves of a pass this
   * is the neighbours-only near field. */
  template <class CoordinateClass>
  void P2PRemote(const CoordinateClass &leafPosition, ContainerClass *const targets,
                 const ContainerClass *const /*sources*/, const ContainerClass *const /*directNeighbors*/[],
                 const int positions[], const int size) {
    P2POuter(leafPosition, targets, nullptr, positions, size);
  }

  /* Write back what is still pending on the GPU (a driver that stops before the direct pass). */
  void flush() {
    std::lock_guard<std::mutex> g(s_->mu);
    if (s_->pending == Op::P2M) flush_p2m();
    flush_pending();
    s_->pending = Op::None;
  }

 private:
  void begin(Op op, int level) {
    State &s = *s_;
    if (s.pending == Op::P2M) flush_p2m();
    if (!s.tree_ready) throw std::runtime_error("FB200Kernel: the bottom pass (P2M) of this evaluation did not run");
    if (s.pending != op || s.pending_level != level) {
      flush_pending();
      s.pending = op;
      s.pending_level = level;
    }
  }

  // write-back of the recorded cells of one level from the GPU, matched by Morton index
  void write_cells(int level, bool multipoles) {
    State &s = *s_;
    long long ncells[32];
    long long np = 0;
    check(b200fmm_tree_info(s.h, ncells, &np), "tree_info");
    const long long n = ncells[level];
    std::vector<long long> keys((size_t)n);
    std::vector<double> v((size_t)n * NVALS * nnodes);
    check(b200fmm_get_cells(s.h, level, keys.data(), multipoles ? v.data() : nullptr, multipoles ? nullptr : v.data()),
          "get_cells");
    for (CellRef &cr : s.cells) {
      CellClass *c = &use(cr);
      const long long key = (long long)c->getMortonIndex();
      const auto it = std::lower_bound(keys.begin(), keys.end(), key);
      if (it == keys.end() || *it != key) throw std::runtime_error("FB200Kernel: a cell of the driver's tree is not in the GPU tree");
      const size_t i = (size_t)(it - keys.begin());
      for (int r = 0; r < NVALS; ++r)
        std::memcpy(multipoles ? c->getMultipole(r) : c->getLocal(r), v.data() + (i * NVALS + r) * nnodes,
                    sizeof(double) * nnodes);
    }
    s.cells.clear();
  }

  void flush_pending() {
    State &s = *s_;
    switch (s.pending) {
      case Op::M2M:
        check(b200fmm_m2m(s.h, s.pending_level), "m2m");
        write_cells(s.pending_level, true);
        break;
      case Op::M2L:
        check(b200fmm_m2l(s.h, s.pending_level), "m2l");
        write_cells(s.pending_level, false);
        s.m2l_flushed.push_back(s.pending_level);
        break;
      case Op::L2L:
        check(b200fmm_l2l(s.h, s.pending_level), "l2l");
        write_cells(s.pending_level + 1, false);
        break;
      default:
        s.cells.clear();
        break;
    }
    s.pending = Op::None;
    s.pending_level = -1;
  }

  // the bottom pass is complete: gather the particles leaf by leaf, build the GPU tree, run P2M
  void flush_p2m() {
    State &s = *s_;
    long long n = 0;
    for (ContRef &cr : s.leaf_tgt) n += (long long)use(cr).getNbParticles();
    std::vector<double> x((size_t)n), y((size_t)n), z((size_t)n), q((size_t)n * NVALS);
    long long off = 0;
    for (ContRef &cr : s.leaf_tgt) {
      const ContainerClass *c = &use(cr);
      const long long m = (long long)c->getNbParticles();
      const auto *const *pos = c->getPositions();
      for (long long k = 0; k < m; ++k) {
        x[(size_t)(off + k)] = pos[0][k];
        y[(size_t)(off + k)] = pos[1][k];
        z[(size_t)(off + k)] = pos[2][k];
      }
      for (int r = 0; r < NVALS; ++r) {
        const auto *qv = c->getPhysicalValues(r);
        for (long long k = 0; k < m; ++k) q[(size_t)(r * n + off + k)] = qv[k];
      }
      off += m;
    }
    check(b200fmm_set_particles(s.h, n, x.data(), y.data(), z.data(), q.data(), 0), "set_particles");
    check(b200fmm_p2m(s.h), "p2m");
    s.cells.assign(s.leaf_cells.begin(), s.leaf_cells.end());
    s.tree_ready = true;
    s.pending = Op::None;
    write_cells(s.height - 1, true);
  }

  // run one direct-pass operator for every leaf and add its potentials and forces into the containers
  template <class Fn>
  void run_direct(Fn &&fn) {
    State &s = *s_;
    check(b200fmm_zero_results(s.h), "zero_results");
    fn();
    long long ncells[32];
    long long n = 0;
    check(b200fmm_tree_info(s.h, ncells, &n), "tree_info");
    std::vector<double> phi((size_t)n * NVALS), fx(phi.size()), fy(phi.size()), fz(phi.size());
    check(b200fmm_get_results(s.h, phi.data(), fx.data(), fy.data(), fz.data(), 0), "get_results");
    long long off = 0;
    for (ContRef &cr : s.leaf_tgt) {
      ContainerClass *c = &use(cr);
      const long long m = (long long)c->getNbParticles();
      for (int r = 0; r < NVALS; ++r) {
        auto *p = c->getPotentials(r);
        auto *gx = c->getForcesX(r);
        auto *gy = c->getForcesY(r);
        auto *gz = c->getForcesZ(r);
        const size_t b = (size_t)(r * n + off);
        for (long long k = 0; k < m; ++k) {
          p[k] += phi[b + (size_t)k];
          gx[k] += fx[b + (size_t)k];
          gy[k] += fy[b + (size_t)k];
          gz[k] += fz[b + (size_t)k];
        }
      }
      off += m;
    }
  }
};

// The adapter for the pointer octree FOctree (FFmmAlgorithm, FFmmAlgorithmThread).
template <class CellClass, class ContainerClass, int ORDER, int NVALS = 1>
using FB200Kernel = FB200KernelT<CellClass, ContainerClass, ORDER, NVALS, false>;
// The adapter for the blocked tree FGroupTree (FGroupSeqAlgorithm), whose cells and leaves are views.
template <class CellClass, class ContainerClass, int ORDER, int NVALS = 1>
using FB200GroupKernel = FB200KernelT<CellClass, ContainerClass, ORDER, NVALS, true>;

}  // namespace b200fmm_scalfmm

#endif
