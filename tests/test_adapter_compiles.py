"""The FB200Kernel adapter header (include/b200fmm_scalfmm.hpp) is self-contained C++17: it compiles with
stand-in cell and container types that have the reference's member functions (FChebCell, FP2PParticleContainer)
and every operator of the FAbstractKernels surface is instantiated.  CPU only: nothing is run."""
import shutil
import subprocess

import pytest

from conftest import ROOT

SRC = r"""
#include "b200fmm_scalfmm.hpp"
struct Point { double getX() const { return 0.5; } double getY() const { return 0.5; } double getZ() const { return 0.5; } };
struct Cell {
  double m[2 * 64], l[2 * 64];
  long long getMortonIndex() const { return 0; }
  double *getMultipole(int r) { return m + 64 * r; }
  double *getLocal(int r) { return l + 64 * r; }
  const double *getMultipole(int r) const { return m + 64 * r; }
  const double *getLocal(int r) const { return l + 64 * r; }
};
struct Container {
  double *p[3];
  double v[5];
  long long getNbParticles() const { return 0; }
  const double *const *getPositions() const { return p; }
  const double *getPhysicalValues(int = 0) const { return v; }
  double *getPotentials(int = 0) { return v; }
  double *getForcesX(int = 0) { return v; }
  double *getForcesY(int = 0) { return v; }
  double *getForcesZ(int = 0) { return v; }
};
struct Coord {};
template class b200fmm_scalfmm::FB200KernelT<Cell, Container, 4, 2, false>;
template class b200fmm_scalfmm::FB200KernelT<Cell, Container, 4, 2, true>;
void use(b200fmm_scalfmm::FB200Kernel<Cell, Container, 4, 2> &k, Cell *c, Container *t, Cell **ch,
         const Cell **nb, const int *pos, Container **nbp) {
  static_assert(b200fmm_scalfmm::FB200Kernel<Cell, Container, 4, 2>::NeedFinishedM2LEvent(), "flush event");
  k.P2M(c, t); k.M2M(c, ch, 2); k.M2L(c, nb, pos, 0, 2); k.finishedLevelM2L(2); k.L2L(c, ch, 2);
  k.L2P(c, t); k.P2P(Coord{}, t, t, nbp, pos, 0); k.P2POuter(Coord{}, t, nbp, pos, 0);
  k.P2PRemote(Coord{}, t, t, (const Container *const *)nbp, pos, 0); k.flush();
  b200fmm_scalfmm::FB200Kernel<Cell, Container, 4, 2> copy(k); (void)copy;
  b200fmm_scalfmm::FB200Kernel<Cell, Container, 4, 2> made(4, 1.0, Point{}); (void)made;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_adapter_header_compiles(tmp_path):
    src = tmp_path / "adapter_use.cpp"
    src.write_text(SRC)
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", f"-I{ROOT / 'include'}",
                        str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
