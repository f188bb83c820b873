"""The allocation-free near-field entry point (b200fmm_p2p_noalloc).

Some callers cannot allocate device memory while this step runs -- an application that has handed all device
memory to its own pool up front, or a loop that cannot afford cudaMalloc's implicit synchronisation -- so this
entry point keeps its scratch in a fixed device array inside the library.  The tests call it through the C ABI
twice in a row on caller-owned device buffers and compare each result with the regular handle-based
b200fmm_p2p on the same particles and with the FP64 near field of the CPU oracle.  This file is named so that
pytest collects it last.

Tolerances: the two calls in a row agree exactly.  Against the handle's P2P the same FP32 arithmetic runs, but
the handle walks the source leaves in column order (one run per neighbour column) while the allocation-free
entry point, which cannot sort, keeps Morton order (runs of Morton-adjacent leaves): the per-stage partial
sums are grouped differently, so the two agree to the FP32 path's accuracy (compensated sums: 1e-6 relative),
not bit for bit.  Against the oracle's FP64 near field the bar is the same 1e-6 relative.
"""
import ctypes

import numpy as np
import pytest

import scalfmm_b200 as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CENTER = (0.5, 0.5, 0.5)
FIELDS = ("phi", "fx", "fy", "fz")


def leaf_tables(x, y, z, height):
    keys = O.morton_keys(x, y, z, 1.0, CENTER, height)
    order = np.lexsort((np.arange(keys.size), keys))  # stable, like the library's radix sort
    sk = keys[order]
    leaf_keys, first = np.unique(sk, return_index=True)
    leaf_start = np.append(first, sk.size).astype(np.int64)
    index = {int(k): i for i, k in enumerate(leaf_keys)}
    lim = 1 << (height - 1)
    nbr = np.full((leaf_keys.size, 27), -1, np.int32)
    for i, k in enumerate(leaf_keys):
        ix, iy, iz = O.morton_decode(int(k))
        for p in range(27):
            dx, dy, dz = p // 9 - 1, (p // 3) % 3 - 1, p % 3 - 1
            jx, jy, jz = ix + dx, iy + dy, iz + dz
            if 0 <= jx < lim and 0 <= jy < lim and 0 <= jz < lim:
                nbr[i, p] = index.get(O.morton_encode(jx, jy, jz), -1)
    return order, leaf_keys.astype(np.int64), leaf_start, nbr


def self_leaf_near_field(xs, ys, zs, qs, leaf_start):
    """FP64 near field of every leaf on itself (FP2P::GenericInner, Src/Kernels/P2P/FP2P.hpp:174-269), sorted
    order: what variant 0 adds over variant 1."""
    out = [np.zeros(xs.size) for _ in range(4)]
    for a, b in zip(leaf_start[:-1], leaf_start[1:]):
        if b - a < 2:
            continue
        d = np.stack([xs[a:b], ys[a:b], zs[a:b]])
        diff = d[:, :, None] - d[:, None, :]
        r2 = (diff ** 2).sum(0)
        np.fill_diagonal(r2, np.inf)
        inv = 1.0 / np.sqrt(r2)
        out[0][a:b] = inv @ qs[a:b]
        w = -(qs[a:b, None] * qs[None, a:b]) * inv ** 3
        for k in range(3):
            out[1 + k][a:b] = (w * diff[k]).sum(1)
    return out


def call_noalloc(t, n, nleaves, height, variant, out, stream):
    center = (ctypes.c_double * 3)(*CENTER)
    return S.lib().b200fmm_p2p_noalloc(
        n, *[ctypes.c_void_p(t[k].data_ptr()) for k in ("x", "y", "z", "q")], nleaves,
        *[ctypes.c_void_p(t[k].data_ptr()) for k in ("keys", "start", "nbr")], height, 1.0, center, variant,
        *[ctypes.c_void_p(o.data_ptr()) for o in out], ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("variant", [0, 1])
def test_p2p_noalloc_matches_handle_p2p_and_oracle(golden, variant):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(77)
    n, height = 30000, 5
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1.0, 1.0, n)

    # the existing entry point: handle-based P2P in MIXED precision
    f = S.FMM("cheb_sym", 4, height, precision="mixed", device=0)
    f.set_particles(x, y, z, q)
    f.reset_expansions()
    f.p2p(variant)
    ref = f.results()
    f.close()

    order, leaf_keys, leaf_start, nbr = leaf_tables(x, y, z, height)
    # the oracle's FP64 near field (leaf with itself and its 26 neighbours); variant 1 leaves the leaf itself out
    sym = golden("sym_ops_p4.npz")
    o = O.fmm(O.CHEB_SYM, 4, height, 1.0, CENTER, x, y, z, q, ops=O.P2P, sym_ranks=sym["ranks"], sym_uv=sym["uv"])
    want = {k: o[k][order].copy() for k in FIELDS}
    if variant == 1:
        own = self_leaf_near_field(x[order], y[order], z[order], q[order], leaf_start)
        for k, v in zip(FIELDS, own):
            want[k] -= v

    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(x=x[order], y=y[order], z=z[order], q=q[order], keys=leaf_keys, start=leaf_start, nbr=nbr).items()}
    stream = torch.cuda.Stream(dev)
    for call in range(2):  # two calls in a row share the library's scratch array
        out = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(4)]
        torch.cuda.synchronize()
        rc = call_noalloc(t, n, leaf_keys.size, height, variant, out, stream)
        assert rc == 0, S.lib().b200fmm_last_error()
        got = [o_.cpu().numpy() for o_ in out]
        for k, g in zip(FIELDS, got):
            assert S.rel_l2(g, ref[k][order]) < 1e-6, (call, k, S.rel_l2(g, ref[k][order]))
            assert S.rel_l2(g, want[k]) < 1e-6, (call, k, S.rel_l2(g, want[k]))
        if call == 0:
            first = got
        else:
            for a, b in zip(first, got):
                assert np.array_equal(a, b)


@pytest.mark.parametrize("flaw", ["end_past_n", "falling_start", "neighbour_out_of_range", "keys_not_rising"])
def test_p2p_noalloc_rejects_inconsistent_tables(flaw):
    """Bad leaf tables are caught on the device before any kernel indexes through them; the outputs stay
    untouched.  The tables keep their declared sizes, so the check itself reads only inside them."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(3)
    n, height = 4000, 4
    x, y, z = rng.random((3, n))
    q = rng.uniform(-1.0, 1.0, n)
    order, leaf_keys, leaf_start, nbr = leaf_tables(x, y, z, height)
    leaf_start, nbr, leaf_keys = leaf_start.copy(), nbr.copy(), leaf_keys.copy()
    if flaw == "end_past_n":
        leaf_start[-1] = n + 64
    elif flaw == "falling_start":
        leaf_start[3] = leaf_start[5] + 1
    elif flaw == "neighbour_out_of_range":
        nbr[1, 0] = leaf_keys.size
    else:
        leaf_keys[2] = leaf_keys[1]
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(x=x[order], y=y[order], z=z[order], q=q[order], keys=leaf_keys, start=leaf_start, nbr=nbr).items()}
    out = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(4)]
    stream = torch.cuda.Stream(dev)
    torch.cuda.synchronize()
    rc = call_noalloc(t, n, leaf_keys.size, height, 0, out, stream)
    assert rc == 1
    assert b"inconsistent leaf tables" in S.lib().b200fmm_last_error()
    assert all(int(torch.count_nonzero(o)) == 0 for o in out)


def test_p2p_noalloc_rejects_oversized_input():
    n = S.NOALLOC_MAX_PARTICLES + 1
    center = (ctypes.c_double * 3)(*CENTER)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = S.lib().b200fmm_p2p_noalloc(n, dummy, dummy, dummy, dummy, 1, dummy, dummy, dummy, 5, 1.0, center, 0,
                                     dummy, dummy, dummy, dummy, None)
    assert rc == 1
    assert b"262144" in S.lib().b200fmm_last_error()
