"""Parity of the CUDA FMM (through the C ABI) with the reference and with the CPU oracle.

Tolerances (relative L2 over the whole vector, FMath::FAccurater):
  * FP64 path with the reference's own compressed operators: 1e-12 against the reference's outputs;
  * FP64 path with this library's own operator compression: the compression tolerance 10^-p can move the
    factors (pivot ties), so 50 * 10^-p against the reference;
  * integer tree work (keys, permutation, lists): exact;
  * MIXED path: 2e-6 against the FP64 path (FP32 P2P + split-FP16 tensor-core M2L); the bench gates the
    1M-particle headline case at 1e-6 on the potential.
"""
import os

import numpy as np
import pytest

import scalfmm_b200 as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("phi", "fx", "fy", "fz")
CENTER = (0.5, 0.5, 0.5)


def run(g, kernel="cheb_sym", precision="fp64", ops=S.ALL, sym=None, nrhs=1):
    f = S.FMM(kernel, int(g["order"]), int(g["height"]), nrhs=nrhs, precision=precision)
    if sym is not None:
        f.set_sym_operators(sym["ranks"], sym["uv"])
    f.set_particles(g["x"], g["y"], g["z"], g["q"])
    f.execute(ops)
    r = f.results()
    f.close()
    return r


SYM_CASES = ["sym_p5_h4_n2000", "sym_p7_h4_n2000", "sym_p4_h5_n3000", "sym_p6_h3_n500"]


@pytest.mark.parametrize("name", SYM_CASES)
def test_fp64_sym_matches_reference_with_reference_operators(golden, name):
    g = golden(f"fmm_{name}.npz")
    sym = golden(f"sym_ops_p{int(g['order'])}.npz")
    r = run(g, sym=sym)
    for f in FIELDS:
        assert S.rel_l2(r[f], g[f]) < 1e-12, (f, S.rel_l2(r[f], g[f]))


@pytest.mark.parametrize("name", SYM_CASES)
def test_fp64_sym_own_operators_close_to_reference(golden, name):
    g = golden(f"fmm_{name}.npz")
    r = run(g)
    tol = 50 * 10.0 ** (-int(g["order"]))
    for f in FIELDS:
        assert S.rel_l2(r[f], g[f]) < tol, (f, S.rel_l2(r[f], g[f]))


@pytest.mark.parametrize("order", [4, 5, 7])
def test_own_operator_compression_matches_reference(golden, order):
    sym = golden(f"sym_ops_p{order}.npz")
    f = S.FMM("cheb_sym", order, 3)
    ranks, uv = f.get_sym_operators()
    f.close()
    assert (ranks == sym["ranks"]).all()
    mine, ref = O.unpack_sym(ranks, uv, order), O.unpack_sym(sym["ranks"], sym["uv"], order)
    for slot in ref:
        A = mine[slot][0] @ mine[slot][1].T
        B = ref[slot][0] @ ref[slot][1].T
        assert np.linalg.norm(A - B) / np.linalg.norm(B) < 10 * 10.0 ** (-order)


@pytest.mark.parametrize("name", ["dense_p4_h4_n2000", "dense_p5_h3_n1000"])
def test_fp64_dense_matches_reference(golden, name):
    g = golden(f"fmm_{name}.npz")
    r = run(g, kernel="cheb_dense")
    for f in FIELDS:
        assert S.rel_l2(r[f], g[f]) < 1e-12, (f, S.rel_l2(r[f], g[f]))


def test_multi_rhs_matches_reference(golden):
    g = golden("fmm_sym_p5_h4_n1500_rhs16.npz")
    sym = golden("sym_ops_p5.npz")
    r = run(g, sym=sym, nrhs=16)
    for f in FIELDS:
        assert r[f].shape == (16, g["x"].size)
        assert S.rel_l2(r[f], g[f]) < 1e-12, f


def test_expansions_per_level_match_reference(golden):
    g = golden("expansions_sym_p4_h4_n1000.npz")
    sym = golden("sym_ops_p4.npz")
    f = S.FMM("cheb_sym", 4, 4)
    f.set_sym_operators(sym["ranks"], sym["uv"])
    f.set_particles(g["x"], g["y"], g["z"], g["q"])
    f.execute()
    for lvl in (2, 3):
        keys, M, L = f.cells(lvl)
        ref = {int(k): i for i, k in enumerate(g["mortons"]) if g["levels"][i] == lvl}
        assert sorted(ref) == sorted(keys.tolist())
        idx = [ref[int(k)] for k in keys]
        assert S.rel_l2(M[:, 0], g["multipoles"][idx]) < 1e-12
        assert S.rel_l2(L[:, 0], g["locals"][idx]) < 1e-12
    f.close()


def test_tree_is_bit_exact_with_oracle():
    rng = np.random.default_rng(5)
    n, H = 20000, 6
    x, y, z = rng.random((3, n))
    x[:50] = 1.0  # the upper face maps to the last cell
    y[50:100] = 0.0
    q = rng.uniform(-1, 1, n)
    f = S.FMM("cheb_sym", 3, H)
    f.set_particles(x, y, z, q)
    keys = O.morton_keys(x, y, z, 1.0, CENTER, H)
    order = np.lexsort((np.arange(n), keys))  # stable sort by key
    assert (f.permutation() == order).all()
    leaf_keys = np.unique(keys)
    nc, npart = f.tree_info()
    assert npart == n and nc[H - 1] == leaf_keys.size
    for lvl in range(H):
        k, _, _ = f.cells(lvl, expansions=False)
        assert (k == np.unique(leaf_keys >> (3 * (H - 1 - lvl)))).all()
    f.close()


def _tree_case(kind, n, seed):
    from distributions import ellipsoid_surface, plummer

    rng = np.random.default_rng(seed)
    if kind == "uniform":
        x, y, z = rng.random((3, n))
    elif kind == "plummer":
        x, y, z = plummer(n, seed)
    else:
        x, y, z = ellipsoid_surface(n, seed)
    return x, y, z, rng.uniform(-1, 1, n)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kind", ["uniform", "plummer", "ellipsoid"])
def test_tree_lists_are_bit_exact_with_oracle(kind, precision):
    """The 26-neighbour leaf lists and the 189-candidate interaction lists of every level, element by element,
    against the oracle's restatement of FTreeCoordinate::getNeighborsIndexes / getInteractionNeighbors
    (Src/Containers/FTreeCoordinate.hpp:189-264) filtered to the cells that exist, as FOctree does
    (Src/Containers/FOctree.hpp:914-975, 1364-1400)."""
    H = 5
    x, y, z, q = _tree_case(kind, 20000, 11)
    f = S.FMM("cheb_sym", 3, H, precision=precision)
    f.set_particles(x, y, z, q)
    leaf_keys, _, _ = f.cells(H - 1, expansions=False)
    index = {int(k): i for i, k in enumerate(leaf_keys)}
    nbr = f.leaf_neighbors()
    assert nbr.shape == (leaf_keys.size, 27)
    for i, k in enumerate(leaf_keys):
        ok, opos = O.leaf_neighbors(*O.morton_decode(int(k)), H)
        want = np.full(27, -1, np.int32)
        want[13] = i
        for kk, pp in zip(ok.tolist(), opos.tolist()):
            want[pp] = index.get(kk, -1)
        assert (nbr[i] == want).all(), (i, nbr[i], want)
    for lvl in range(2, H):
        keys, _, _ = f.cells(lvl, expansions=False)
        idx = {int(k): i for i, k in enumerate(keys)}
        src, pos = f.interaction_lists(lvl)
        for i, k in enumerate(keys):
            ok, opos = O.interaction_list(*O.morton_decode(int(k)), lvl)
            want = sorted((pp, idx[kk]) for kk, pp in zip(ok.tolist(), opos.tolist()) if kk in idx)
            got = sorted((int(p_), int(s_)) for p_, s_ in zip(pos[i], src[i]) if s_ >= 0)
            assert got == want, (lvl, i)
            assert ((src[i] >= 0) == (pos[i] >= 0)).all()
    f.close()


def test_direct_gpu_matches_reference(golden):
    g = golden("direct_n1500.npz")
    d = S.direct(g["x"], g["y"], g["z"], g["q"])
    for k in FIELDS:
        assert S.rel_l2(d[k], g[k]) < 1e-13
    t = np.array([0, 7, 1499, 300])
    d2 = S.direct(g["x"], g["y"], g["z"], g["q"], targets=t)
    for k in FIELDS:
        assert np.allclose(d2[k], g[k][t], rtol=1e-13, atol=0)


@pytest.mark.parametrize("ops", [S.P2P, S.P2M | S.M2M | S.M2L | S.L2L | S.L2P, S.P2M | S.M2M | S.M2L | S.L2L])
def test_operation_masks_match_oracle(golden, ops):
    g = golden("fmm_sym_p5_h4_n2000.npz")
    sym = golden("sym_ops_p5.npz")
    r = run(g, sym=sym, ops=ops)
    o = O.fmm(O.CHEB_SYM, 5, 4, 1.0, CENTER, g["x"], g["y"], g["z"], g["q"], ops=ops, sym_ranks=sym["ranks"],
              sym_uv=sym["uv"])
    for f in FIELDS:
        if not np.any(o[f]):
            assert not np.any(r[f])
        else:
            assert S.rel_l2(r[f], o[f]) < 1e-12, f


def test_level_batched_operators_equal_execute(golden):
    g = golden("fmm_sym_p4_h5_n3000.npz")
    sym = golden("sym_ops_p4.npz")
    f = S.FMM("cheb_sym", 4, 5)
    f.set_sym_operators(sym["ranks"], sym["uv"])
    f.set_particles(g["x"], g["y"], g["z"], g["q"])
    f.reset_expansions()
    f.p2m()
    for lvl in (3, 2):
        f.m2m(lvl)
    for lvl in (2, 3, 4):
        f.m2l(lvl)
    for lvl in (2, 3):
        f.l2l(lvl)
    f.l2p()
    f.p2p(0)
    r = f.results()
    for k in FIELDS:
        assert S.rel_l2(r[k], g[k]) < 1e-12
    # P2PRemote variant: neighbours only = full P2P minus the leaf's own pairs
    f.reset_expansions()
    f.p2p(1)
    remote = f.results()
    f.reset_expansions()
    f.p2p(0)
    full = f.results()
    o_self = O.fmm(O.CHEB_SYM, 4, 5, 1.0, CENTER, g["x"], g["y"], g["z"], g["q"], ops=O.P2P, sym_ranks=sym["ranks"],
                   sym_uv=sym["uv"])
    assert S.rel_l2(full["phi"], o_self["phi"]) < 1e-12
    assert S.rel_l2(remote["phi"], full["phi"]) > 1e-3  # the self-leaf pairs are missing
    f.close()


@pytest.mark.parametrize("order", [6, 7])
def test_level_batched_mixed_on_compacted_levels(order):
    """MIXED level-batched operators on a clustered tree whose sparse levels run the tensor-core M2L on
    compacted blocks: one M2L launch per level gives the results of execute() (whose single launch covers every
    level) to the mixed level; the FP32 partial sums are only grouped differently."""
    from distributions import plummer

    x, y, z = plummer(30000, seed=71)
    q = np.random.default_rng(72).uniform(-1.0, 1.0, x.size)
    H = 6
    f = S.FMM("cheb_sym", order, H, precision="mixed")
    f.set_particles(x, y, z, q)
    f.execute()
    want = f.results()
    f.reset_expansions()
    f.p2m()
    for lvl in range(H - 2, 1, -1):
        f.m2m(lvl)
    for lvl in range(2, H):
        f.m2l(lvl)
    for lvl in range(2, H - 1):
        f.l2l(lvl)
    f.l2p()
    f.p2p(0)
    got = f.results()
    f.close()
    for k in FIELDS:
        assert S.rel_l2(got[k], want[k]) < 2e-6, (k, S.rel_l2(got[k], want[k]))


def test_async_results_overlap_the_next_tree():
    """get_results_async queues each step's results on a copy stream of their own while the next step uploads
    and builds its tree (trees of different sizes and shapes, one set of host buffers written twice); after
    synchronize() every step's host arrays hold that step's results, as the blocking get_results gives them."""
    import torch
    from distributions import plummer

    rng = np.random.default_rng(81)
    trees = [tuple(rng.random((3, 30000))), plummer(25000, seed=82), tuple(rng.random((3, 40000))),
             tuple(rng.random((3, 30000)))]
    charges = [rng.uniform(-1.0, 1.0, t[0].size) for t in trees]
    f = S.FMM("cheb_sym", 5, 5, precision="mixed")
    shared = [torch.empty(30000, dtype=torch.float64).pin_memory() for _ in range(4)]
    bufs = []
    for i, ((x, y, z), q) in enumerate(zip(trees, charges)):
        f.set_particles(x, y, z, q)
        f.execute()
        # steps 0 and 3 write the same host buffers: the later copy must land last
        b = shared if i in (0, 3) else [torch.empty(x.size, dtype=torch.float64).pin_memory() for _ in range(4)]
        f.results_into_async(*b)
        bufs.append(b)
    f.synchronize()
    f.close()
    for i, ((x, y, z), q, b) in enumerate(zip(trees, charges, bufs)):
        if i == 0:
            continue
        want = _mixed_eval(x, y, z, q, 5, order=5)
        for k, t in zip(FIELDS, b):
            assert S.rel_l2(t.numpy(), want[k]) < 1e-12, (i, k)


@pytest.mark.parametrize("kernel,precision,order,height,dist,count", [
    ("cheb_sym", "mixed", 5, 5, "uniform", 3), ("cheb_sym", "fp64", 5, 6, "plummer", 4),
    ("lagrange", "mixed", 6, 6, "ellipsoid", 2), ("cheb_sym", "mixed", 7, 6, "plummer", 3)])
def test_shards_add_up_to_the_whole_evaluation(kernel, precision, order, height, dist, count):
    """Target shards (set_shard): each shard evaluates the particles of its Morton range of leaves and leaves the
    others at zero, so every particle is evaluated by exactly one shard and the shards' results add up to the
    whole evaluation (FP64 to rounding; MIXED to the mixed level, the M2L's FP32 partial sums being grouped by
    other work ranges).  Uniform, clustered (compacted M2L levels, CTA pairs at order 7) and surface trees."""
    from distributions import ellipsoid_surface, plummer

    rng = np.random.default_rng(91)
    if dist == "uniform":
        x, y, z = rng.random((3, 30000))
    elif dist == "plummer":
        x, y, z = plummer(30000, seed=92)
    else:
        x, y, z = ellipsoid_surface(30000, seed=93)
    q = rng.uniform(-1.0, 1.0, x.size)
    f = S.FMM(kernel, order, height, precision=precision)
    f.set_particles(x, y, z, q)
    f.execute()
    whole = f.results()
    total = {k: np.zeros(x.size) for k in FIELDS}
    owners = np.zeros(x.size, np.int64)
    for r in range(count):
        f.set_shard(r, count)
        f.execute()
        part = f.results()
        owners += part["phi"] != 0.0
        for k in FIELDS:
            total[k] += part[k]
    # the same shard again: the second evaluation is captured into a CUDA graph, the third replays it
    for _ in range(2):
        f.execute()
        rep = f.results()
        for k in FIELDS:
            assert S.rel_l2(rep[k], part[k]) < 1e-12, k
    f.set_shard(0, 1)
    f.execute()
    again = f.results()
    f.close()
    assert np.all(owners == 1)
    tol = 1e-12 if precision == "fp64" else 2e-6
    for k in FIELDS:
        assert S.rel_l2(total[k], whole[k]) < tol, (k, S.rel_l2(total[k], whole[k]))
        assert S.rel_l2(again[k], whole[k]) < tol, k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_more_shards_than_leaves(precision):
    """Shards whose Morton range holds no leaf evaluate nothing (their results are all zero); the others
    still add up to the whole evaluation.  Also a set_shard before any particles, and one with several
    right-hand sides."""
    rng = np.random.default_rng(95)
    n = 40
    # two tight clusters: two occupied leaves at height 3, so most of 16 shards hold no leaf
    c = np.where(np.arange(n) < n // 2, 0.12, 0.82)
    x, y, z = (c + 0.03 * rng.random(n) for _ in range(3))
    q = rng.uniform(-1.0, 1.0, (2, n))
    f = S.FMM("cheb_sym", 4, 3, nrhs=2, precision=precision)
    f.set_shard(1, 2)
    f.set_shard(0, 1)
    f.set_particles(x, y, z, q)
    f.execute()
    whole = f.results()
    count = 16
    total = {k: np.zeros_like(whole[k]) for k in FIELDS}
    empty = 0
    for r in range(count):
        f.set_shard(r, count)
        f.execute()
        part = f.results()
        empty += int(not np.any(part["phi"]))
        for k in FIELDS:
            total[k] += part[k]
    f.close()
    assert empty > 0
    tol = 1e-12 if precision == "fp64" else 2e-6
    for k in FIELDS:
        assert S.rel_l2(total[k], whole[k]) < tol, k


def _sweep_case(rng):
    from distributions import ellipsoid_surface, plummer

    kernel = str(rng.choice(["cheb_sym", "cheb_dense", "lagrange"]))
    order = int(rng.integers(3, 8))
    height = int(rng.integers(3, 8))
    n = int(np.exp(rng.uniform(np.log(2000), np.log(60000))))
    dist = str(rng.choice(["uniform", "plummer", "ellipsoid", "clusters"]))
    if dist == "uniform":
        x, y, z = rng.random((3, n))
    elif dist == "plummer":
        x, y, z = plummer(n, seed=int(rng.integers(1 << 30)))
    elif dist == "ellipsoid":
        x, y, z = ellipsoid_surface(n, seed=int(rng.integers(1 << 30)))
    else:
        c = rng.random((4, 3)) * 0.8 + 0.1
        p = np.clip(c[rng.integers(0, 4, n)] + rng.normal(0.0, 0.02, (n, 3)), 0.0, 1.0 - 1e-12)
        x, y, z = p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy()
    q = rng.uniform(-1.0, 1.0, n)
    if dist != "plummer":
        # at least about two particles per leaf (the Plummer core fills deep leaves on its own)
        height = min(height, max(3, int(np.log(n / 2) / np.log(8)) + 1))
    return kernel, order, height, dist, (x, y, z, q), str(int(rng.integers(0, 2))), int(rng.choice([1, 1, 2, 3]))


@pytest.mark.parametrize("case", range(12))
def test_seeded_configurations_mixed_vs_fp64(case):
    """A seeded sweep over kernels (symmetric and dense Chebyshev, Lagrange), orders 3-7, heights 3-7, uniform /
    clustered / surface / multi-cluster particles, CTA pairs forced on or off and 1-3 target shards: MIXED
    against FP64 within 3e-6 on every output.  Trees whose leaves hold under about two particles on average
    are left out (Plummer excepted): there the far field carries nearly all of the forces, and the Lagrange
    M2L in MIXED reaches 3e-6 at order 6 and 6e-6 at order 7 in every M2L form, tiles and compacted blocks
    alike."""
    rng = np.random.default_rng(1000 + case)
    kernel, order, height, dist, (x, y, z, q), pair, shards = _sweep_case(rng)
    if kernel == "lagrange" and order == 7:
        order = 6
    res = {}
    old = os.environ.get("B200FMM_TC_PAIR")
    os.environ["B200FMM_TC_PAIR"] = pair
    try:
        for prec in ("fp64", "mixed"):
            f = S.FMM(kernel, order, height, precision=prec)
            f.set_particles(x, y, z, q)
            r = {k: np.zeros(x.size) for k in FIELDS}
            for s_ in range(shards):
                f.set_shard(s_, shards)
                f.execute()
                part = f.results()
                for k in FIELDS:
                    r[k] += part[k]
            res[prec] = r
            f.close()
    finally:
        if old is None:
            os.environ.pop("B200FMM_TC_PAIR", None)
        else:
            os.environ["B200FMM_TC_PAIR"] = old
    for k in FIELDS:
        e = S.rel_l2(res["mixed"][k], res["fp64"][k])
        assert e < 3e-6, (kernel, order, height, dist, pair, shards, k, e)


def test_edge_cases():
    # one particle: no interactions at all
    f = S.FMM("cheb_sym", 4, 3)
    f.set_particles([0.3], [0.3], [0.3], [1.0])
    f.execute()
    r = f.results()
    assert r["phi"][0] == 0 and r["fx"][0] == 0
    # two particles in one leaf: exact pair
    f.set_particles([0.1, 0.12], [0.1, 0.1], [0.1, 0.1], [1.0, -2.0])
    f.execute()
    r = f.results()
    assert abs(r["phi"][0] - (-2.0 / 0.02)) < 1e-9 and abs(r["phi"][1] - 1.0 / 0.02) < 1e-9
    # particles outside the box are rejected with a status code
    with pytest.raises(S.B200FmmError):
        f.set_particles([1.5], [0.5], [0.5], [1.0])
    with pytest.raises(S.B200FmmError):
        f.set_particles([np.nan], [0.5], [0.5], [1.0])
    f.close()
    # clustered particles (many empty leaves) against the oracle
    rng = np.random.default_rng(9)
    n = 3000
    pos = np.clip(0.2 + 0.05 * rng.standard_normal((3, n)), 0, 1)
    pos[:, :300] = rng.random((3, 300))
    q = rng.uniform(-1, 1, n)
    sym = O.unpack_sym  # noqa: F841 (operators below come from the library itself)
    f = S.FMM("cheb_sym", 5, 6)
    ranks, uv = f.get_sym_operators()
    f.set_particles(pos[0], pos[1], pos[2], q)
    f.execute()
    r = f.results()
    o = O.fmm(O.CHEB_SYM, 5, 6, 1.0, CENTER, pos[0], pos[1], pos[2], q, sym_ranks=ranks, sym_uv=uv)
    for k in FIELDS:
        assert S.rel_l2(r[k], o[k]) < 1e-12
    f.close()


@pytest.mark.parametrize("kernel", ["cheb_sym", "cheb_dense", "lagrange"])
def test_mixed_close_to_fp64(kernel):
    """MIXED against FP64 with the same operators (CHEB_SYM: the compressed ones, applied in their low-rank
    form on the tensor cores), order 5, height 5."""
    rng = np.random.default_rng(3)
    n = 30000
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1, 1, n)
    out = {}
    for prec in ("fp64", "mixed"):
        f = S.FMM(kernel, 5, 5, precision=prec)
        f.set_particles(x, y, z, q)
        f.execute()
        out[prec] = f.results()
        f.close()
    for k in FIELDS:
        assert S.rel_l2(out["mixed"][k], out["fp64"][k]) < 2e-6, (k, S.rel_l2(out["mixed"][k], out["fp64"][k]))


@pytest.mark.parametrize("order", [5, 6, 7])
def test_first_product_issuers_agree(order):
    """The low-rank M2L's first product issues its MMAs from one thread or from two (one per TMEM
    accumulator, each skipping the other's chunks but passing every stage).  Each accumulator receives the
    same MMAs in the same order either way, so the results are bit-identical; order 6 (three segments of
    3, 3 and 1 K chunks) is where the second thread skips a chunk that the stage ring reuses."""
    from distributions import plummer

    x, y, z = plummer(40000, seed=71)
    q = np.random.default_rng(72).uniform(-1.0, 1.0, x.size)
    out = {}
    for issuers in ("1", "2"):
        old = os.environ.get("B200FMM_TC_YISSUERS")
        os.environ["B200FMM_TC_YISSUERS"] = issuers
        try:
            f = S.FMM("cheb_sym", order, 6, precision="mixed")
            f.set_particles(x, y, z, q)
            f.execute()
            f.execute()
            out[issuers] = f.results()
            f.close()
        finally:
            if old is None:
                os.environ.pop("B200FMM_TC_YISSUERS", None)
            else:
                os.environ["B200FMM_TC_YISSUERS"] = old
    for k in FIELDS:
        assert np.array_equal(out["1"][k], out["2"][k]), (k, S.rel_l2(out["1"][k], out["2"][k]))


def test_mixed_close_to_fp64_clustered_order7():
    """MIXED against FP64 on a clustered (Plummer) tree at order 7, height 6: the sparse levels run the
    low-rank first product compacted."""
    from distributions import plummer

    x, y, z = plummer(60000, seed=61)
    q = np.random.default_rng(62).uniform(-1.0, 1.0, x.size)
    out = {}
    for prec in ("fp64", "mixed"):
        f = S.FMM("cheb_sym", 7, 6, precision=prec)
        f.set_particles(x, y, z, q)
        f.execute()
        out[prec] = f.results()
        f.close()
    for k in FIELDS:
        assert S.rel_l2(out["mixed"][k], out["fp64"][k]) < 2e-6, (k, S.rel_l2(out["mixed"][k], out["fp64"][k]))


@pytest.mark.parametrize("name", ["lagrange_p4_h4_n2000", "lagrange_p6_h3_n1000"])
def test_lagrange_matches_reference(golden, name):
    """The reference's FUnifKernel (Fourier-space M2L) against the dense Lagrange M2L here: FP64 to 1e-12,
    MIXED (tensor-core M2L, FP32 P2P) to 2e-6."""
    g = golden(f"fmm_{name}.npz")
    for prec, tol in (("fp64", 1e-12), ("mixed", 2e-6)):
        r = run(g, kernel="lagrange", precision=prec)
        for k in FIELDS:
            assert S.rel_l2(r[k], g[k]) < tol, (prec, k, S.rel_l2(r[k], g[k]))


def test_lagrange_fp64_matches_oracle():
    rng = np.random.default_rng(4)
    n = 2000
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1, 1, n)
    f = S.FMM("lagrange", 5, 4)
    f.set_particles(x, y, z, q)
    f.execute()
    r = f.results()
    f.close()
    o = O.fmm(O.LAGRANGE, 5, 4, 1.0, CENTER, x, y, z, q)
    for k in FIELDS:
        assert S.rel_l2(r[k], o[k]) < 1e-12, k


@pytest.mark.parametrize("order,height", [(5, 5), (7, 4), (4, 6)])
def test_mixed_m2l_locals_match_fp64_dense(order, height):
    """Isolates the tensor-core M2L: same multipoles (FP64 P2M/M2M in both), locals after M2L compared per
    level against the FP64 dense M2L.  Tolerance 2e-6: split-FP16 operands carry 22 bits and each transfer
    vector's tensor-core FP32 accumulation chain adds ~1e-6 at p = 7 (measured 1.1e-6 at level 2)."""
    rng = np.random.default_rng(order * 10 + height)
    n = 20000
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1, 1, n)
    ops = S.P2M | S.M2M | S.M2L
    loc = {}
    for prec in ("fp64", "mixed"):
        f = S.FMM("cheb_dense", order, height, precision=prec)
        f.set_particles(x, y, z, q)
        f.execute(ops)
        loc[prec] = {lvl: f.cells(lvl)[2] for lvl in range(2, height)}
        f.close()
    for lvl in range(2, height):
        err = S.rel_l2(loc["mixed"][lvl], loc["fp64"][lvl])
        assert err < 2e-6, (lvl, err)


@pytest.mark.parametrize("order,height", [(3, 5), (6, 4), (7, 5)])
def test_cta_pair_m2l_matches_single_cta(order, height, monkeypatch):
    """The tensor-core M2L on CTA pairs (cta_group::2, M = 256, each CTA holding half of every operator
    chunk) against single CTAs (B200FMM_TC_PAIR=0): both within 2e-6 of the FP64 dense M2L, and of each
    other (their work ranges, hence their FP32 partial sums, differ).  Levels 2 and 3 have one tile in z, so
    their pairs run with a missing second tile; 3 work ranges per CTA exercise fragments that start and
    end inside a tile's transfer vectors."""
    rng = np.random.default_rng(order * 100 + height)
    n = 20000
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1, 1, n)
    ops = S.P2M | S.M2M | S.M2L
    monkeypatch.setenv("B200FMM_TC_SPLITS", "3")
    loc = {}
    for mode, prec, pair in (("fp64", "fp64", "1"), ("pair", "mixed", "1"), ("single", "mixed", "0")):
        monkeypatch.setenv("B200FMM_TC_PAIR", pair)
        f = S.FMM("cheb_dense", order, height, precision=prec)
        f.set_particles(x, y, z, q)
        f.execute(ops)
        loc[mode] = {lvl: f.cells(lvl)[2] for lvl in range(2, height)}
        f.close()
    for lvl in range(2, height):
        assert S.rel_l2(loc["pair"][lvl], loc["single"][lvl]) < 2e-6, lvl
        assert S.rel_l2(loc["pair"][lvl], loc["fp64"][lvl]) < 2e-6, lvl
        assert S.rel_l2(loc["single"][lvl], loc["fp64"][lvl]) < 2e-6, lvl


@pytest.mark.parametrize("order,height,pair", [(3, 5, "0"), (5, 5, "0"), (6, 4, "0"), (7, 5, "1"), (7, 4, "0")])
def test_lowrank_m2l_locals_match_fp64_sym(order, height, pair, monkeypatch):
    """Isolates the low-rank tensor-core M2L (CHEB_SYM, MIXED): the same multipoles (FP64 P2M/M2M in both), the
    locals after M2L against the FP64 compressed-operator M2L, level by level, on single CTAs and on CTA
    pairs.  Tolerance 1e-6: the first product Y = V^T M and the second U Y each carry split-FP16 operands
    (22 bits) and short FP32 accumulation segments (measured 5e-7 at order 7)."""
    rng = np.random.default_rng(order * 10 + height + 1)
    n = 20000
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1, 1, n)
    ops = S.P2M | S.M2M | S.M2L
    monkeypatch.setenv("B200FMM_TC_PAIR", pair)
    loc = {}
    for prec in ("fp64", "mixed"):
        f = S.FMM("cheb_sym", order, height, precision=prec)
        f.set_particles(x, y, z, q)
        f.execute(ops)
        loc[prec] = {lvl: f.cells(lvl)[2] for lvl in range(2, height)}
        f.close()
    for lvl in range(2, height):
        err = S.rel_l2(loc["mixed"][lvl], loc["fp64"][lvl])
        assert err < 1e-6, (lvl, err)


def test_cheb_sym_mixed_dense_operators_on_request(monkeypatch):
    """B200FMM_TC_LOWRANK=0 keeps the dense tensor-core M2L for CHEB_SYM: it then matches the FP64 dense
    kernel (the uncompressed operators) within the MIXED tolerance."""
    rng = np.random.default_rng(61)
    n = 20000
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1, 1, n)
    monkeypatch.setenv("B200FMM_TC_LOWRANK", "0")
    f = S.FMM("cheb_sym", 5, 5, precision="mixed")
    f.set_particles(x, y, z, q)
    f.execute()
    got = f.results()
    f.close()
    g = S.FMM("cheb_dense", 5, 5)
    g.set_particles(x, y, z, q)
    g.execute()
    want = g.results()
    g.close()
    for k in FIELDS:
        assert S.rel_l2(got[k], want[k]) < 2e-6, k


def _fp64_and_mixed(kernel, order, height, x, y, z, q, nrhs=1):
    out = {}
    for prec in ("fp64", "mixed"):
        f = S.FMM(kernel, order, height, nrhs=nrhs, precision=prec)
        if prec == "fp64":
            out["ops"] = f.get_sym_operators() if kernel == "cheb_sym" else None
        f.set_particles(x, y, z, q)
        f.execute()
        out[prec] = f.results()
        f.close()
    return out


def test_ellipsoid_surface_lagrange_p6():
    """The uneven-surface workload's shape (points on an ellipsoid surface, Lagrange order 6) on a deep tree
    whose leaves are mostly empty: FP64 against the CPU restatement to 1e-12, MIXED against FP64 to 2e-6."""
    from distributions import ellipsoid_surface

    n, height = 12000, 6
    x, y, z = ellipsoid_surface(n, seed=21)
    q = np.random.default_rng(22).uniform(0.0, 1.0, n)
    out = _fp64_and_mixed("lagrange", 6, height, x, y, z, q)
    o = O.fmm(O.LAGRANGE, 6, height, 1.0, CENTER, x, y, z, q)
    for k in FIELDS:
        assert S.rel_l2(out["fp64"][k], o[k]) < 1e-12, k
        assert S.rel_l2(out["mixed"][k], out["fp64"][k]) < 2e-6, k


def test_plummer_cheb_sym():
    """The batch workload's Plummer-sphere particles (strongly clustered centre): FP64 ChebSym against the
    CPU restatement with the library's own operators to 1e-12, MIXED against FP64 to 2e-6."""
    from distributions import plummer

    n, height = 15000, 6
    x, y, z = plummer(n, seed=23)
    q = np.random.default_rng(24).uniform(-1.0, 1.0, n)
    out = _fp64_and_mixed("cheb_sym", 5, height, x, y, z, q)
    ranks, uv = out["ops"]
    o = O.fmm(O.CHEB_SYM, 5, height, 1.0, CENTER, x, y, z, q, sym_ranks=ranks, sym_uv=uv)
    for k in FIELDS:
        assert S.rel_l2(out["fp64"][k], o[k]) < 1e-12, k
        assert S.rel_l2(out["mixed"][k], out["fp64"][k]) < 2e-6, k


def test_multi_rhs_mixed_matches_single_rhs():
    """Sixteen charge vectors on one tree (the multi-RHS workload's shape, order 7): each RHS of the MIXED
    multi-RHS evaluation is within the MIXED tolerance (2e-6) of a single-RHS FP64 evaluation of that charge
    vector with the same (compressed) operators, and within 2e-6 of a single-RHS MIXED evaluation (the work
    ranges of the tensor-core M2L are split differently with 16 RHS, so the FP32 partial sums group
    differently and the two MIXED errors do not cancel)."""
    rng = np.random.default_rng(25)
    n, height, nrhs = 20000, 5, 16
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1.0, 1.0, (nrhs, n))
    f = S.FMM("cheb_sym", 7, height, nrhs=nrhs, precision="mixed")
    f.set_particles(x, y, z, q.ravel())
    f.execute()
    multi = f.results()
    f.close()
    for r in (0, 7, 15):
        single = {}
        for kernel, prec in (("cheb_sym", "fp64"), ("cheb_sym", "mixed")):
            g = S.FMM(kernel, 7, height, precision=prec)
            g.set_particles(x, y, z, q[r])
            g.execute()
            single[prec] = g.results()
            g.close()
        for k in FIELDS:
            m = np.asarray(multi[k]).reshape(nrhs, n)[r]
            assert S.rel_l2(m, single["fp64"][k]) < 2e-6, (r, k)
            assert S.rel_l2(m, single["mixed"][k]) < 2e-6, (r, k)


@pytest.mark.parametrize("kernel,precision", [("cheb_sym", "fp64"), ("cheb_sym", "mixed"), ("lagrange", "mixed")])
def test_repeated_execute_replays_a_graph(kernel, precision):
    """New charges on one tree (an iterative solver's pattern): the second execute() captures the passes into
    a CUDA graph and later ones replay it.  Each replay must equal a fresh handle's plain evaluation of the
    same charges (1e-12: only the order of FP64 atomic additions may differ), and only the total time is
    reported for a replay."""
    rng = np.random.default_rng(31)
    n, order, height = 6000, 5, 5
    x, y, z = rng.random((3, n))
    qs = [rng.uniform(-1, 1, n) for _ in range(4)]
    f = S.FMM(kernel, order, height, precision=precision)
    f.set_particles(x, y, z, qs[0])
    f.execute()
    assert f.timings()["p2m"] > 0  # plain launches: per-pass times
    for q in qs[1:]:
        f.set_charges(q)
        f.execute()
        got = f.results()
        t = f.timings()
        assert t["p2m"] == 0 and t["total"] > 0
        g = S.FMM(kernel, order, height, precision=precision)
        g.set_particles(x, y, z, q)
        g.execute()
        want = g.results()
        g.close()
        for k in FIELDS:
            assert S.rel_l2(got[k], want[k]) < 1e-12, k
    # a new tree goes back to plain launches
    f.set_particles(y, z, x, qs[0])
    f.execute()
    assert f.timings()["p2m"] > 0
    f.close()


@pytest.mark.parametrize("kernel,precision,tol", [("cheb_sym", "fp64", 1e-12), ("cheb_sym", "mixed", 1e-10),
                                                  ("lagrange", "mixed", 1e-10)])
def test_batch_matches_single_problems(kernel, precision, tol):
    """A batch of problems of uneven size, order and height (the batch workload's shape: Plummer positions,
    orders 4..6, heights for about 30 particles per leaf) run over 3 worker streams equals each problem run
    on its own handle (same arithmetic; only the order of FP64 atomic additions may differ); the batch is
    run twice so that the second call reuses the workers' handles."""
    from distributions import plummer

    rng = np.random.default_rng(41)
    problems = []
    for k in range(9):
        n = int(np.exp(rng.uniform(np.log(1500), np.log(40000))))
        x, y, z = plummer(n, seed=100 + k)
        height = int(min(6, max(3, np.ceil(np.log(max(n / 30, 1)) / np.log(8)) + 1)))
        problems.append(dict(x=x, y=y, z=z, q=rng.uniform(-1, 1, n), order=4 + k % 3, height=height))
    b = S.Batch(kernel, precision, nstreams=3, device=0)
    for _ in range(2):
        outs = b.run(problems)
        assert b.last_time_ms() > 0 and b.last_device_ms() > 0
        for pr, out in zip(problems, outs):
            f = S.FMM(kernel, pr["order"], pr["height"], precision=precision)
            f.set_particles(pr["x"], pr["y"], pr["z"], pr["q"])
            f.execute()
            want = f.results()
            f.close()
            for k in FIELDS:
                assert S.rel_l2(out[k], want[k]) < tol, (pr["order"], pr["height"], k)
    b.close()


def test_autotune_keeps_mixed_accuracy():
    """The split autotuner picks one of its candidates, reports a kernel time, and the evaluation after it
    stays within the MIXED tolerance of FP64 (the split only regroups FP32 partial sums)."""
    rng = np.random.default_rng(51)
    n, height = 30000, 5
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1, 1, n)
    f = S.FMM("cheb_sym", 6, height, precision="mixed")
    f.set_particles(x, y, z, q)
    k, ms = f.autotune()
    assert k in (1, 2, 3, 4) and ms > 0
    f.execute()
    got = f.results()
    f.close()
    g = S.FMM("cheb_sym", 6, height)
    g.set_particles(x, y, z, q)
    g.execute()
    want = g.results()
    g.close()
    for key in FIELDS:
        assert S.rel_l2(got[key], want[key]) < 2e-6, key


def test_mixed_handle_reused_from_dense_to_sparse_tree():
    """The low-rank M2L's first product skips the tiles of a sparse tree that hold no cell; the Y rows of such a
    tile must still read as zero when an earlier, denser tree on the same handle wrote values there.  A handle
    that evaluated a uniform tree and then a clustered one gives the clustered tree's results of a fresh
    handle (to rounding: both run the same operators and work split)."""
    from distributions import plummer

    rng = np.random.default_rng(31)
    n, H = 30000, 5
    xu, yu, zu = rng.random((3, n))
    xp, yp, zp = plummer(n, seed=32)
    q = rng.uniform(-1.0, 1.0, n)
    reused = S.FMM("cheb_sym", 6, H, precision="mixed")
    reused.set_particles(xu, yu, zu, q)
    reused.execute()
    reused.set_particles(xp, yp, zp, q)
    reused.execute()
    got = reused.results()
    reused.close()
    fresh = S.FMM("cheb_sym", 6, H, precision="mixed")
    fresh.set_particles(xp, yp, zp, q)
    fresh.execute()
    want = fresh.results()
    fresh.close()
    for k in FIELDS:
        assert S.rel_l2(got[k], want[k]) < 1e-12, (k, S.rel_l2(got[k], want[k]))


def _mixed_eval(x, y, z, q, H, env=None, order=6, kernel="cheb_sym", precision="mixed"):
    old = {k: os.environ.get(k) for k in (env or {})}
    os.environ.update(env or {})
    try:
        f = S.FMM(kernel, order, H, precision=precision)
        f.set_particles(x, y, z, q)
        f.execute()
        r = f.results()
        f.close()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return r


@pytest.mark.parametrize("order", [5, 6, 7])
def test_compacted_first_product_matches_tile_mode(order):
    """A level less than half full runs the first product over blocks of 128 occupied cells instead of the
    parity grid's tiles; every Y row depends on its own cell only, so the results equal those of the tile mode
    (B200FMM_TC_YCOMPACT=0) on the same clustered tree."""
    from distributions import plummer

    x, y, z = plummer(30000, seed=41)
    q = np.random.default_rng(42).uniform(-1.0, 1.0, x.size)
    got = _mixed_eval(x, y, z, q, 6, order=order)
    want = _mixed_eval(x, y, z, q, 6, {"B200FMM_TC_YCOMPACT": "0"}, order=order)
    for k in FIELDS:
        assert np.array_equal(got[k], want[k]), (k, S.rel_l2(got[k], want[k]))


@pytest.mark.parametrize("kernel,order,pair", [("cheb_sym", 5, "0"), ("cheb_sym", 6, "0"), ("cheb_sym", 6, "1"),
                                               ("cheb_sym", 7, "1"), ("lagrange", 6, "0"), ("lagrange", 5, "1")])
def test_compacted_second_product_matches_tile_mode(kernel, order, pair):
    """A level less than half full runs the second M2L product (U Y, or K M in the dense form) over blocks of
    128 cells of one parity whose A rows are gathered, instead of the parity grid's tiles, on single CTAs and
    on CTA pairs.  The accumulator segments are cut where the block's busy transfer vectors put them, so the
    results agree with the tile mode (B200FMM_TC_TCOMPACT=0) to the mixed-precision level rather than bitwise;
    both agree with FP64, and two fresh handles give identical results (the placement is deterministic)."""
    from distributions import ellipsoid_surface, plummer

    if kernel == "lagrange":
        x, y, z = ellipsoid_surface(40000, seed=44)
    else:
        x, y, z = plummer(30000, seed=43)
    q = np.random.default_rng(45).uniform(-1.0, 1.0, x.size)
    env = {"B200FMM_TC_PAIR": pair}
    got = _mixed_eval(x, y, z, q, 6, env, order=order, kernel=kernel)
    again = _mixed_eval(x, y, z, q, 6, env, order=order, kernel=kernel)
    tiles = _mixed_eval(x, y, z, q, 6, {**env, "B200FMM_TC_TCOMPACT": "0"}, order=order, kernel=kernel)
    ref = _mixed_eval(x, y, z, q, 6, order=order, kernel=kernel, precision="fp64")
    for k in FIELDS:
        assert np.array_equal(got[k], again[k]), k
        assert S.rel_l2(got[k], tiles[k]) < 2e-6, (k, S.rel_l2(got[k], tiles[k]))
        e_c, e_t = S.rel_l2(got[k], ref[k]), S.rel_l2(tiles[k], ref[k])
        assert e_c < 2e-6 and e_c < 1.5 * e_t + 1e-8, (k, e_c, e_t)


def test_mixed_handle_reused_across_sparse_and_dense_trees():
    """One handle evaluates clustered, clustered, uniform and clustered trees in turn: the Y rows a compacted
    level wrote for one tree are cleared before the next, and levels switch between compacted and tile mode;
    each evaluation gives the results of a fresh handle."""
    from distributions import plummer

    rng = np.random.default_rng(51)
    n, H = 30000, 6
    trees = [plummer(n, seed=52), plummer(n, seed=53), tuple(rng.random((3, n))), plummer(n, seed=52)]
    q = rng.uniform(-1.0, 1.0, n)
    reused = S.FMM("cheb_sym", 6, H, precision="mixed")
    for x, y, z in trees:
        reused.set_particles(x, y, z, q)
        reused.execute()
        got = reused.results()
        want = _mixed_eval(x, y, z, q, H)
        for k in FIELDS:
            assert S.rel_l2(got[k], want[k]) < 1e-12, (k, S.rel_l2(got[k], want[k]))
    reused.close()
