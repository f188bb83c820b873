"""Drop-in check of the FB200Kernel adapter (include/b200fmm_scalfmm.hpp).

The reference's own algorithm drivers (FFmmAlgorithm, FFmmAlgorithmThread with one thread, and FGroupSeqAlgorithm
over the blocked tree FGroupTree with FB200GroupKernel) run on two
copies of one octree: once with the reference's FChebSymKernel / FChebDenseKernel, once with the adapter
over the GPU library.  Potentials and forces of every particle and the multipoles and locals of every
cell are compared (relative L2, FMath::FAccurater).  The check program is built from the reference sources
into oracle/_ref/libadapter_check.so (oracle/Makefile); it is required here, not skipped.

Tolerances: FP64 with the reference's own compressed operators (sym) or the dense operators: 1e-12;
MIXED (FP32 P2P, split-FP16 tensor-core M2L) against the reference's FP64: 2e-6 on the particle outputs.
"""
import ctypes

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

LIB = ROOT / "oracle" / "_ref" / "libadapter_check.so"
FP64, MIXED = 0, 1


def check(kind, order, precision, driver, height, n, seed=3):
    assert LIB.exists(), f"{LIB} was not built (make -C oracle ref)"
    L = ctypes.CDLL(str(LIB))
    dp = ctypes.POINTER(ctypes.c_double)
    L.adapter_check.restype = ctypes.c_int
    L.adapter_check.argtypes = [ctypes.c_int] * 5 + [ctypes.c_longlong] + [dp] * 5
    L.adapter_check_message.restype = ctypes.c_char_p
    rng = np.random.default_rng(seed)
    x, y, z = (np.ascontiguousarray(rng.random(n)) for _ in range(3))
    q = rng.uniform(-1, 1, n)
    errs = np.zeros(6)
    rc = L.adapter_check(kind, order, precision, driver, height, n, *(a.ctypes.data_as(dp) for a in (x, y, z, q, errs)))
    assert rc == 0, f"adapter_check failed ({rc}): {L.adapter_check_message().decode()}"
    return dict(zip(("phi", "fx", "fy", "fz", "multipole", "local"), errs))


@pytest.mark.parametrize("driver", [0, 1])
def test_adapter_sym_fp64_is_a_drop_in(driver):
    e = check(kind=0, order=5, precision=FP64, driver=driver, height=4, n=2000)
    assert max(e.values()) <= 1e-12, e


def test_adapter_dense_fp64_is_a_drop_in():
    e = check(kind=1, order=4, precision=FP64, driver=0, height=4, n=2000)
    assert max(e.values()) <= 1e-12, e


def test_adapter_mixed_close_to_reference():
    e = check(kind=0, order=7, precision=MIXED, driver=0, height=4, n=3000)
    for k in ("phi", "fx", "fy", "fz"):
        assert e[k] <= 2e-6, e
    assert e["multipole"] <= 1e-12, e  # P2M/M2M stay FP64 in MIXED


@pytest.mark.parametrize("order,height,n", [(5, 4, 3000), (4, 5, 4000)])
def test_group_tree_adapter_fp64_is_a_drop_in(order, height, n):
    """The blocked tree (FGroupTree of FChebCellPOD cells and FP2PGroupParticleContainer leaves, blocks of 30
    cells) driven by the reference's FGroupSeqAlgorithm: its in-block calls, its cross-block M2L and P2POuter
    pairs and its cell and leaf views all go through FB200GroupKernel, which reads and writes the block arrays.
    Every particle output and every cell expansion of levels 2..height-1 matches FChebSymKernel on the same
    blocked tree to 1e-12 (FP64, the reference's compressed operators)."""
    e = check(kind=0, order=order, precision=FP64, driver=2, height=height, n=n)
    assert max(e.values()) <= 1e-12, e


def test_group_tree_adapter_mixed_close_to_reference():
    e = check(kind=0, order=7, precision=MIXED, driver=2, height=4, n=3000)
    for k in ("phi", "fx", "fy", "fz"):
        assert e[k] <= 2e-6, e
    assert e["multipole"] <= 1e-12, e
