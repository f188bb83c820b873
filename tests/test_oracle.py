"""Pin the CPU oracle (oracle/fmm_oracle.c + oracle/precompute.py) against the reference's own outputs:
the golden fixtures made by tests/golden/make_golden.py from the compiled reference, the reference's
known-answer data files when they are present, and the reference's structural unit tests
(UTests/utestMorton.cpp, utestNeighborIndexes.cpp)."""
import numpy as np
import pytest

from conftest import REFERENCE_DATA, read_bfma
from oracle import oracle as O
from oracle import precompute as PC

FIELDS = ("phi", "fx", "fy", "fz")


def test_morton_roundtrip():
    # UTests/utestMorton.cpp:15-40: encode/decode round trip, x is the MSB of each bit triple
    rng = np.random.default_rng(0)
    for _ in range(2000):
        c = rng.integers(0, 1 << 20, 3)
        k = O.morton_encode(*map(int, c))
        assert O.morton_decode(k) == tuple(map(int, c))
    assert O.morton_encode(1, 0, 0) == 4 and O.morton_encode(0, 1, 0) == 2 and O.morton_encode(0, 0, 1) == 1
    assert O.morton_encode(3, 0, 0) == 0b100100


def test_morton_keys_face_rule():
    # FCoordinateComputer.hpp:19-21: a particle exactly on the upper face goes to the last cell
    x = np.array([0.0, 1.0, 0.5, 0.999999])
    k = O.morton_keys(x, x, x, 1.0, (0.5, 0.5, 0.5), 4)
    last = O.morton_encode(7, 7, 7)
    assert k[0] == 0 and k[1] == last and k[2] == O.morton_encode(4, 4, 4) and k[3] == last
    with pytest.raises(ValueError):
        O.morton_keys(np.array([1.5]), np.array([0.5]), np.array([0.5]), 1.0, (0.5, 0.5, 0.5), 4)


def test_neighbor_lists_bruteforce():
    # utestNeighborIndexes.cpp: the 26-neighbour and 189-interaction rules against a brute-force scan
    height = 5
    lim = 1 << (height - 1)
    rng = np.random.default_rng(1)
    for _ in range(200):
        ix, iy, iz = map(int, rng.integers(0, lim, 3))
        keys, pos = O.leaf_neighbors(ix, iy, iz, height)
        exp = []
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    if (dx or dy or dz) and 0 <= ix + dx < lim and 0 <= iy + dy < lim and 0 <= iz + dz < lim:
                        exp.append((O.morton_encode(ix + dx, iy + dy, iz + dz), ((dx + 1) * 3 + dy + 1) * 3 + dz + 1))
        assert list(zip(keys.tolist(), pos.tolist())) == exp
        level = height - 1
        ik, ip = O.interaction_list(ix, iy, iz, level)
        got = set(zip(ik.tolist(), ip.tolist()))
        want = set()
        for sx in range(lim):
            for sy in range(lim):
                for sz in range(lim):
                    d = (sx - ix, sy - iy, sz - iz)
                    if max(map(abs, d)) > 1 and max(abs((sx >> 1) - (ix >> 1)), abs((sy >> 1) - (iy >> 1)),
                                                    abs((sz >> 1) - (iz >> 1))) <= 1:
                        want.add((O.morton_encode(sx, sy, sz), ((d[0] + 3) * 7 + d[1] + 3) * 7 + d[2] + 3))
        assert got == want
    # an interior cell has exactly 189 far neighbours
    assert len(O.interaction_list(6, 6, 6, 4)[0]) == 189


@pytest.mark.parametrize("order", [3, 5, 7])
def test_symmetry_tables_match_reference(golden, order):
    g = golden(f"sym_ops_p{order}.npz")
    pind, pvec = O.sym_tables(order)
    assert (pind == g["pindices"]).all()
    assert (pvec[g["far_slots"]] == g["pvectors_far"]).all()


@pytest.mark.parametrize("order", [3, 4, 5, 6, 7])
def test_precompute_matches_reference_operators(golden, order):
    """Own restatement of pACA + QR + SVD: same ranks as the reference, and the same low-rank operator
    U V^T to the compression tolerance eps = 10^-p (pivot ties between mirror-symmetric nodes may be
    broken differently, which changes the factors only within eps)."""
    g = golden(f"sym_ops_p{order}.npz")
    ref = O.unpack_sym(g["ranks"], g["uv"], order)
    mine = PC.sym_operators(order)
    assert sorted(mine) == sorted(ref)
    eps = 10.0 ** (-order)
    for slot in ref:
        U, V = mine[slot]
        RU, RV = ref[slot]
        assert U.shape == RU.shape
        A, B = U @ V.T, RU @ RV.T
        assert np.linalg.norm(A - B) / np.linalg.norm(B) < 10 * eps


FMM_CASES = ["sym_p5_h4_n2000", "sym_p7_h4_n2000", "sym_p4_h5_n3000", "sym_p6_h3_n500", "dense_p4_h4_n2000",
             "dense_p5_h3_n1000", "sym_p5_h4_n1500_rhs16",
             # the reference's FUnifKernel, whose M2L runs through FFTs (served by oracle/ref/fftw): the
             # restatement's dense Lagrange M2L equals it to rounding
             "lagrange_p4_h4_n2000", "lagrange_p6_h3_n1000"]


@pytest.mark.parametrize("name", FMM_CASES)
def test_oracle_fmm_matches_reference(golden, name):
    g = golden(f"fmm_{name}.npz")
    order = int(g["order"])
    kw = {}
    if int(g["kind"]) == O.CHEB_SYM:
        s = golden(f"sym_ops_p{order}.npz")
        kw = dict(sym_ranks=s["ranks"], sym_uv=s["uv"])
    r = O.fmm(int(g["kind"]), order, int(g["height"]), 1.0, (0.5, 0.5, 0.5), g["x"], g["y"], g["z"], g["q"], **kw)
    for f in FIELDS:
        assert O.rel_l2(r[f], g[f]) < 1e-12, f


def test_oracle_expansions_match_reference(golden):
    g = golden("expansions_sym_p4_h4_n1000.npz")
    s = golden("sym_ops_p4.npz")
    r = O.fmm(O.CHEB_SYM, 4, 4, 1.0, (0.5, 0.5, 0.5), g["x"], g["y"], g["z"], g["q"], sym_ranks=s["ranks"],
              sym_uv=s["uv"], dump=True)
    for lvl in (2, 3):
        mine = {int(k): i for i, k in enumerate(r["mortons"]) if r["levels"][i] == lvl}
        theirs = [(int(k), i) for i, k in enumerate(g["mortons"]) if g["levels"][i] == lvl]
        assert len(mine) == len(theirs)
        for key, i in theirs:
            j = mine[key]
            assert O.rel_l2(r["multipoles"][j, 0], g["multipoles"][i]) < 1e-12
            assert O.rel_l2(r["locals"][j, 0], g["locals"][i]) < 1e-12


def test_oracle_direct_matches_reference(golden):
    g = golden("direct_n1500.npz")
    d = O.direct(g["x"], g["y"], g["z"], g["q"])
    for f in FIELDS:
        assert O.rel_l2(d[f], g[f]) < 1e-13


@pytest.mark.skipif(not (REFERENCE_DATA / "UTest" / "DirectDouble.bfma").exists(),
                    reason="reference data files not present")
def test_oracle_known_answer_directdouble():
    """Data/UTest/DirectDouble.bfma holds 5000 particles with their direct-sum potential and forces
    (used by UTests/FUKernelTester.hpp:39-171)."""
    f = read_bfma(REFERENCE_DATA / "UTest" / "DirectDouble.bfma")
    d = f["data"]
    x, y, z, q = (d[:, i] for i in range(4))
    got = O.direct(x, y, z, q)
    for k, col in zip(FIELDS, (4, 5, 6, 7)):
        assert O.rel_l2(got[k], d[:, col]) < 1e-12


@pytest.mark.skipif(not (REFERENCE_DATA / "UTest" / "unitCubeRef20kDouble.bfma").exists(),
                    reason="reference data files not present")
def test_oracle_reproduces_published_accuracy(golden):
    """Data/ResultCompareKernels.txt:28-35: FChebSymKernel order 7, height 5 on unitCubeRef20kDouble.bfma
    gives potential rel-L2 1.13529e-08 and Fx 1.66035e-06 against the stored direct sum."""
    f = read_bfma(REFERENCE_DATA / "UTest" / "unitCubeRef20kDouble.bfma")
    d = f["data"]
    s = golden("sym_ops_p7.npz")
    r = O.fmm(O.CHEB_SYM, 7, 5, f["box_width"], f["center"], d[:, 0], d[:, 1], d[:, 2], d[:, 3],
              sym_ranks=s["ranks"], sym_uv=s["uv"])
    assert abs(O.rel_l2(r["phi"], d[:, 4]) / 1.13529e-08 - 1) < 2e-3
    assert abs(O.rel_l2(r["fx"], d[:, 5]) / 1.66035e-06 - 1) < 2e-3
