"""The allocation-free near-field entry point (b200fmm_p2p_noalloc).

Some callers cannot allocate device memory while this step runs -- a framework capturing the step into a
CUDA graph that forbids allocations during capture, or an application that has handed all device memory
to its own pool -- so this entry point keeps its scratch in a fixed device array inside the library.  The
test calls it through the C ABI twice in a row on caller-owned device buffers and compares each result with
the regular handle-based b200fmm_p2p on the same particles.  This file is named so that pytest collects it
last.

Tolerance: the two calls in a row agree exactly.  Against the handle's P2P the same FP32 arithmetic runs, but
the handle walks the source leaves in column order (one run per neighbour column) while the allocation-free
entry point, which cannot sort, keeps Morton order (runs of Morton-adjacent leaves): the per-stage partial
sums are grouped differently, so the two agree to the FP32 path's accuracy (compensated sums: 1e-6 relative),
not bit for bit.
"""
import ctypes

import numpy as np
import pytest

import scalfmm_b200 as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CENTER = (0.5, 0.5, 0.5)


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


@pytest.mark.parametrize("variant", [0, 1])
def test_p2p_noalloc_matches_handle_p2p(variant):
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
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(x=x[order], y=y[order], z=z[order], q=q[order], keys=leaf_keys, start=leaf_start, nbr=nbr).items()}
    stream = torch.cuda.Stream(dev)
    center = (ctypes.c_double * 3)(*CENTER)
    for call in range(2):  # two calls in a row share the library's scratch array
        out = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(4)]
        torch.cuda.synchronize()
        rc = S.lib().b200fmm_p2p_noalloc(
            n, *[ctypes.c_void_p(t[k].data_ptr()) for k in ("x", "y", "z", "q")], leaf_keys.size,
            *[ctypes.c_void_p(t[k].data_ptr()) for k in ("keys", "start", "nbr")], height, 1.0, center, variant,
            *[ctypes.c_void_p(o.data_ptr()) for o in out], ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, S.lib().b200fmm_last_error()
        got = [o.cpu().numpy() for o in out]
        for k, g in zip(("phi", "fx", "fy", "fz"), got):
            want = ref[k][order]
            assert S.rel_l2(g, want) < 1e-6, (call, k, S.rel_l2(g, want))
        if call == 0:
            first = got
        else:
            for a, b in zip(first, got):
                assert np.array_equal(a, b)


def test_p2p_noalloc_rejects_oversized_input():
    n = S.NOALLOC_MAX_PARTICLES + 1
    center = (ctypes.c_double * 3)(*CENTER)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = S.lib().b200fmm_p2p_noalloc(n, dummy, dummy, dummy, dummy, 1, dummy, dummy, dummy, 5, 1.0, center, 0,
                                     dummy, dummy, dummy, dummy, None)
    assert rc == 1
    assert b"262144" in S.lib().b200fmm_last_error()
