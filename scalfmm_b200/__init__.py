"""scalfmm_b200: B200 (sm_100a) implementation of the ScalFMM interpolation-FMM hot path.

The product is the C-ABI shared library ``libb200fmm.so`` (declared in include/b200fmm.h).  This module
is a thin ctypes binding used by the tests and the benchmark; it mirrors the reference's flow
(Examples/ChebyshevInterpolationFMM.cpp: build tree -> build kernel -> algo.execute()) and its operator
surface (FAbstractKernels P2M/M2M/M2L/L2L/L2P/P2P, level-batched).  There is no CPU fallback: loading
fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libb200fmm.so"

CHEB_SYM, CHEB_DENSE, LAGRANGE = 0, 1, 2
FP64, MIXED = 0, 1
P2P, P2M, M2M, M2L, L2L, L2P = 1, 2, 4, 8, 16, 32
ALL = 63
KERNELS = {"cheb_sym": CHEB_SYM, "cheb_dense": CHEB_DENSE, "lagrange": LAGRANGE}
PRECISIONS = {"fp64": FP64, "mixed": MIXED}

# every entry point declared in include/b200fmm.h
EXPORTS = (
    "b200fmm_create", "b200fmm_destroy", "b200fmm_last_error", "b200fmm_version", "b200fmm_set_sym_operators",
    "b200fmm_get_sym_operators", "b200fmm_set_particles", "b200fmm_set_charges", "b200fmm_execute",
    "b200fmm_reset_expansions", "b200fmm_zero_results", "b200fmm_p2m", "b200fmm_m2m", "b200fmm_m2l", "b200fmm_l2l", "b200fmm_l2p",
    "b200fmm_p2p", "b200fmm_get_results", "b200fmm_get_results_async", "b200fmm_join_results", "b200fmm_synchronize", "b200fmm_set_shard", "b200fmm_tree_info", "b200fmm_get_cells",
    "b200fmm_get_permutation", "b200fmm_last_timings", "b200fmm_last_kernel_times", "b200fmm_tree_stats",
    "b200fmm_last_launch_count", "b200fmm_autotune", "b200fmm_p2p_noalloc", "b200fmm_batch_create", "b200fmm_batch_execute",
    "b200fmm_batch_last_time", "b200fmm_batch_last_device_time", "b200fmm_batch_destroy", "b200fmm_direct", "b200fmm_m2l_flops",
    "b200fmm_get_leaf_neighbors", "b200fmm_get_interaction_lists", "b200fmm_fma_read", "b200fmm_fma_write",
    "b200fmm_get_leaf_ranges", "b200fmm_get_tuning",
)
NOALLOC_MAX_PARTICLES = 262144

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_longlong)


class B200FmmError(RuntimeError):
    pass


class Problem(ctypes.Structure):
    """b200fmm_problem: one problem of a batch (host arrays)."""
    _fields_ = [("n", ctypes.c_longlong), ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p),
                ("q", ctypes.c_void_p), ("phi", ctypes.c_void_p), ("fx", ctypes.c_void_p), ("fy", ctypes.c_void_p),
                ("fz", ctypes.c_void_p), ("order", ctypes.c_int), ("height", ctypes.c_int),
                ("box_width", ctypes.c_double), ("center", ctypes.c_double * 3)]


class Config(ctypes.Structure):
    _fields_ = [
        ("kernel", ctypes.c_int),
        ("order", ctypes.c_int),
        ("height", ctypes.c_int),
        ("nrhs", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("box_width", ctypes.c_double),
        ("center", ctypes.c_double * 3),
        ("epsilon", ctypes.c_double),
        ("stream", ctypes.c_void_p),
        ("device", ctypes.c_int),
    ]


_lib = None


def build(verbose: bool = False) -> None:
    """Compile libb200fmm.so for sm_100a (nvcc; works without a GPU)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", str(HERE / "csrc"), "-j8"], check=True,
                   stdout=None if verbose else subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise B200FmmError(f"{LIB_PATH} is missing: build it with `make -C scalfmm_b200/csrc`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name in EXPORTS:
            getattr(L, name).restype = ctypes.c_int
        L.b200fmm_last_error.restype = ctypes.c_char_p
        L.b200fmm_version.restype = ctypes.c_char_p
        L.b200fmm_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]
        L.b200fmm_destroy.argtypes = [ctypes.c_void_p]
        L.b200fmm_set_sym_operators.argtypes = [ctypes.c_void_p, _ip, _dp, ctypes.c_longlong]
        L.b200fmm_get_sym_operators.argtypes = [ctypes.c_void_p, _ip, _dp, ctypes.c_longlong, _lp]
        L.b200fmm_set_particles.argtypes = [ctypes.c_void_p, ctypes.c_longlong] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
        L.b200fmm_set_charges.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.b200fmm_execute.argtypes = [ctypes.c_void_p, ctypes.c_uint]
        for n in ("b200fmm_reset_expansions", "b200fmm_zero_results", "b200fmm_p2m", "b200fmm_l2p",
                  "b200fmm_synchronize", "b200fmm_join_results"):
            getattr(L, n).argtypes = [ctypes.c_void_p]
        for n in ("b200fmm_m2m", "b200fmm_m2l", "b200fmm_l2l", "b200fmm_p2p"):
            getattr(L, n).argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.b200fmm_get_results.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
        L.b200fmm_get_results_async.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4
        L.b200fmm_set_shard.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.b200fmm_tree_info.argtypes = [ctypes.c_void_p, _lp, _lp]
        L.b200fmm_get_cells.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _dp, _dp]
        L.b200fmm_get_permutation.argtypes = [ctypes.c_void_p, _lp]
        L.b200fmm_get_leaf_neighbors.argtypes = [ctypes.c_void_p, _ip]
        L.b200fmm_get_leaf_ranges.argtypes = [ctypes.c_void_p, _lp]
        L.b200fmm_get_tuning.argtypes = [ctypes.c_void_p, _ip]
        L.b200fmm_fma_read.argtypes = [ctypes.c_char_p, _lp, _ip, _dp, _dp, _dp, ctypes.c_longlong]
        L.b200fmm_fma_write.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.b200fmm_get_interaction_lists.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _ip]
        L.b200fmm_last_timings.argtypes = [ctypes.c_void_p, _dp]
        L.b200fmm_last_launch_count.argtypes = [ctypes.c_void_p, _lp]
        L.b200fmm_last_kernel_times.argtypes = [ctypes.c_void_p, _dp]
        L.b200fmm_tree_stats.argtypes = [ctypes.c_void_p, _lp, _lp]
        L.b200fmm_p2p_noalloc.argtypes = ([ctypes.c_longlong] + [ctypes.c_void_p] * 4 + [ctypes.c_longlong]
                                          + [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int]
                                          + [ctypes.c_void_p] * 5)
        L.b200fmm_autotune.argtypes = [ctypes.c_void_p, _ip, _dp]
        L.b200fmm_m2l_flops.argtypes = [ctypes.c_void_p, _dp]
        L.b200fmm_batch_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_void_p)]
        L.b200fmm_batch_execute.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.b200fmm_batch_last_time.argtypes = [ctypes.c_void_p, _dp]
        L.b200fmm_batch_last_device_time.argtypes = [ctypes.c_void_p, _dp]
        L.b200fmm_batch_destroy.argtypes = [ctypes.c_void_p]
        L.b200fmm_direct.argtypes = [ctypes.c_longlong, _dp, _dp, _dp, _dp, ctypes.c_longlong, _lp, _dp, _dp, _dp, _dp]
        _lib = L
    return _lib


def _check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().b200fmm_last_error().decode(errors="replace")
        raise B200FmmError(f"{what} failed (status {rc}): {msg}")


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class FMM:
    """One FMM configuration on one GPU (a b200fmm handle).

    kernel: 'cheb_sym' (FChebSymKernel), 'cheb_dense' (FChebDenseKernel) or 'lagrange' (FUnifKernel);
    precision: 'fp64' or 'mixed'.
    """

    def __init__(self, kernel="cheb_sym", order=7, height=6, nrhs=1, precision="fp64", box_width=1.0,
                 center=(0.5, 0.5, 0.5), epsilon=0.0, device=-1, stream=None):
        self.order, self.height, self.nrhs = order, height, nrhs
        self.nn = order ** 3
        cfg = Config(KERNELS[kernel] if isinstance(kernel, str) else kernel, order, height, nrhs,
                     PRECISIONS[precision] if isinstance(precision, str) else precision, box_width,
                     (ctypes.c_double * 3)(*center), epsilon, stream, device)
        h = ctypes.c_void_p()
        _check(lib().b200fmm_create(ctypes.byref(cfg), ctypes.byref(h)), "b200fmm_create")
        self._h = h
        self.n = 0

    # -- lifecycle --------------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().b200fmm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- operators --------------------------------------------------------------------------------------
    def set_sym_operators(self, ranks, uv):
        ranks = np.ascontiguousarray(ranks, dtype=np.int32)
        uv = _f64(uv)
        _check(lib().b200fmm_set_sym_operators(self._h, _ptr(ranks, _ip), _ptr(uv), uv.size), "set_sym_operators")

    def get_sym_operators(self):
        n = ctypes.c_longlong()
        ranks = np.zeros(343, np.int32)
        _check(lib().b200fmm_get_sym_operators(self._h, _ptr(ranks, _ip), None, 0, ctypes.byref(n)), "get_sym_operators")
        uv = np.zeros(n.value)
        _check(lib().b200fmm_get_sym_operators(self._h, _ptr(ranks, _ip), _ptr(uv), uv.size, ctypes.byref(n)),
               "get_sym_operators")
        return ranks, uv

    # -- particles --------------------------------------------------------------------------------------
    def set_particles(self, x, y, z, q):
        """Host numpy arrays, or CUDA tensors (anything with data_ptr()) for device-resident inputs."""
        if hasattr(x, "data_ptr"):
            n = x.numel()
            args = [ctypes.c_void_p(t.data_ptr()) for t in (x, y, z, q)]
            _check(lib().b200fmm_set_particles(self._h, n, *args, 1 if x.is_cuda else 0), "set_particles")
        else:
            x, y, z, q = _f64(x), _f64(y), _f64(z), _f64(q)
            n = x.size
            self._keep = (x, y, z, q)
            _check(lib().b200fmm_set_particles(self._h, n, *[ctypes.c_void_p(a.ctypes.data) for a in (x, y, z, q)], 0),
                   "set_particles")
        self.n = n

    def set_charges(self, q):
        if hasattr(q, "data_ptr"):
            _check(lib().b200fmm_set_charges(self._h, ctypes.c_void_p(q.data_ptr()), 1), "set_charges")
        else:
            q = _f64(q)
            _check(lib().b200fmm_set_charges(self._h, ctypes.c_void_p(q.ctypes.data), 0), "set_charges")

    # -- algorithm --------------------------------------------------------------------------------------
    def execute(self, ops=ALL):
        _check(lib().b200fmm_execute(self._h, ops), "execute")

    def reset_expansions(self):
        _check(lib().b200fmm_reset_expansions(self._h), "reset_expansions")

    def autotune(self):
        """Pick the tensor-core M2L work split for the current tree (MIXED); returns (splits, kernel ms)."""
        k, ms = ctypes.c_int(), ctypes.c_double()
        _check(lib().b200fmm_autotune(self._h, ctypes.byref(k), ctypes.byref(ms)), "autotune")
        return k.value, ms.value

    def zero_results(self):
        _check(lib().b200fmm_zero_results(self._h), "zero_results")

    def p2m(self):
        _check(lib().b200fmm_p2m(self._h), "p2m")

    def m2m(self, level):
        _check(lib().b200fmm_m2m(self._h, level), "m2m")

    def m2l(self, level):
        _check(lib().b200fmm_m2l(self._h, level), "m2l")

    def l2l(self, level):
        _check(lib().b200fmm_l2l(self._h, level), "l2l")

    def l2p(self):
        _check(lib().b200fmm_l2p(self._h), "l2p")

    def p2p(self, variant=0):
        _check(lib().b200fmm_p2p(self._h, variant), "p2p")

    def synchronize(self):
        _check(lib().b200fmm_synchronize(self._h), "synchronize")

    # -- outputs ----------------------------------------------------------------------------------------
    def results(self):
        R, n = self.nrhs, self.n
        out = [np.zeros(R * n) for _ in range(4)]
        _check(lib().b200fmm_get_results(self._h, *[ctypes.c_void_p(o.ctypes.data) for o in out], 0), "get_results")
        shape = (R, n) if R > 1 else (n,)
        return dict(zip(("phi", "fx", "fy", "fz"), (o.reshape(shape) for o in out)))

    def results_into(self, phi, fx, fy, fz):
        """Write the results into four tensors (CUDA tensors, or pinned host tensors)."""
        _check(lib().b200fmm_get_results(self._h, *[ctypes.c_void_p(t.data_ptr()) for t in (phi, fx, fy, fz)],
                                         1 if phi.is_cuda else 0), "get_results")

    def results_into_async(self, phi, fx, fy, fz):
        """Queue the results' copy into four pinned host tensors without waiting; they hold the results once
        synchronize() has returned."""
        if any(t.is_cuda for t in (phi, fx, fy, fz)):
            raise ValueError("results_into_async writes host tensors")
        _check(lib().b200fmm_get_results_async(self._h, *[ctypes.c_void_p(t.data_ptr()) for t in (phi, fx, fy, fz)]),
               "get_results_async")

    def set_shard(self, rank, count):
        """Evaluate only shard `rank` of `count` (a Morton range of leaves with about N / count particles) from
        the next execute() on; the other particles' results stay zero, so the shards' results add up to the
        whole evaluation.  count = 1 evaluates every particle."""
        _check(lib().b200fmm_set_shard(self._h, int(rank), int(count)), "set_shard")

    def join_results(self):
        """Make the handle's stream wait on the device for the queued result copies."""
        _check(lib().b200fmm_join_results(self._h), "join_results")

    def tree_info(self):
        nc = np.zeros(self.height, np.int64)
        npart = ctypes.c_longlong()
        _check(lib().b200fmm_tree_info(self._h, _ptr(nc, _lp), ctypes.byref(npart)), "tree_info")
        return nc, npart.value

    def cells(self, level, expansions=True):
        nc, _ = self.tree_info()
        n = int(nc[level])
        keys = np.zeros(n, np.int64)
        M = np.zeros(n * self.nrhs * self.nn) if expansions else None
        L = np.zeros(n * self.nrhs * self.nn) if expansions else None
        _check(lib().b200fmm_get_cells(self._h, level, _ptr(keys, _lp), _ptr(M) if expansions else None,
                                       _ptr(L) if expansions else None), "get_cells")
        if not expansions:
            return keys, None, None
        return keys, M.reshape(n, self.nrhs, self.nn), L.reshape(n, self.nrhs, self.nn)

    def permutation(self):
        perm = np.zeros(self.n, np.int64)
        _check(lib().b200fmm_get_permutation(self._h, _ptr(perm, _lp)), "get_permutation")
        return perm

    def leaf_neighbors(self):
        """[nleaves, 27] leaf index at each neighbour position ((dx+1)*3+(dy+1))*3+(dz+1), -1 if empty."""
        nc, _ = self.tree_info()
        nbr = np.zeros(int(nc[self.height - 1]) * 27, np.int32)
        _check(lib().b200fmm_get_leaf_neighbors(self._h, _ptr(nbr, _ip)), "get_leaf_neighbors")
        return nbr.reshape(-1, 27)

    def interaction_lists(self, level):
        """([ncells, 189] source cell, [ncells, 189] position ((dx+3)*7+(dy+3))*7+(dz+3)), -1 if absent."""
        nc, _ = self.tree_info()
        n = int(nc[level])
        src = np.zeros(n * 189, np.int32)
        pos = np.zeros(n * 189, np.int32)
        _check(lib().b200fmm_get_interaction_lists(self._h, level, _ptr(src, _ip), _ptr(pos, _ip)),
               "get_interaction_lists")
        return src.reshape(n, 189), pos.reshape(n, 189)

    def tuning(self):
        """(M2L work ranges per CTA, largest leaf the near field takes whole, targets per piece of a larger leaf)."""
        v = np.zeros(3, np.int32)
        _check(lib().b200fmm_get_tuning(self._h, _ptr(v, _ip)), "get_tuning")
        return tuple(int(a) for a in v)

    def timings(self):
        ms = np.zeros(8)
        _check(lib().b200fmm_last_timings(self._h, _ptr(ms)), "last_timings")
        return dict(zip(("tree", "p2m", "m2m", "m2l", "l2l", "l2p", "p2p", "total"), ms.tolist()))

    def kernel_times(self):
        ms = np.zeros(4)
        _check(lib().b200fmm_last_kernel_times(self._h, _ptr(ms)), "last_kernel_times")
        return dict(zip(("m2l", "p2p", "p2m", "l2p"), ms.tolist()))

    def tree_stats(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().b200fmm_tree_stats(self._h, ctypes.byref(a), ctypes.byref(b)), "tree_stats")
        return a.value, b.value

    def launch_count(self):
        c = ctypes.c_longlong()
        _check(lib().b200fmm_last_launch_count(self._h, ctypes.byref(c)), "last_launch_count")
        return c.value

    def m2l_flops(self):
        """Algorithmic FLOPs of one M2L pass of the current tree, for the operator form this handle runs."""
        v = ctypes.c_double()
        _check(lib().b200fmm_m2l_flops(self._h, ctypes.byref(v)), "m2l_flops")
        return v.value


class Batch:
    """Many independent problems of uneven size, spread over worker streams (b200fmm_batch_*).

    run(problems) takes a list of dicts with x, y, z, q (numpy), order, height and optionally box_width and
    center, and returns one dict of phi, fx, fy, fz per problem."""

    def __init__(self, kernel="cheb_sym", precision="mixed", nstreams=4, device=-1):
        h = ctypes.c_void_p()
        _check(lib().b200fmm_batch_create(KERNELS[kernel], PRECISIONS[precision], nstreams, device, ctypes.byref(h)),
               "batch_create")
        self._h = h

    def run(self, problems):
        keep, arr = [], (Problem * len(problems))()
        outs = []
        for k, pr in enumerate(problems):
            x, y, z, q = (_f64(pr[a]) for a in ("x", "y", "z", "q"))
            out = {f: np.zeros(x.size) for f in ("phi", "fx", "fy", "fz")}
            keep += [x, y, z, q]
            outs.append(out)
            c = pr.get("center", (0.5, 0.5, 0.5))
            arr[k] = Problem(x.size, x.ctypes.data, y.ctypes.data, z.ctypes.data, q.ctypes.data,
                             out["phi"].ctypes.data, out["fx"].ctypes.data, out["fy"].ctypes.data,
                             out["fz"].ctypes.data, int(pr["order"]), int(pr["height"]),
                             float(pr.get("box_width", 1.0)), (ctypes.c_double * 3)(*c))
        _check(lib().b200fmm_batch_execute(self._h, len(problems), arr), "batch_execute")
        return outs

    def last_time_ms(self):
        ms = ctypes.c_double()
        _check(lib().b200fmm_batch_last_time(self._h, ctypes.byref(ms)), "batch_last_time")
        return ms.value

    def last_device_ms(self):
        """Device time of the last run: start event to the last worker stream's end event."""
        ms = ctypes.c_double()
        _check(lib().b200fmm_batch_last_device_time(self._h, ctypes.byref(ms)), "batch_last_device_time")
        return ms.value

    def close(self):
        if self._h:
            lib().b200fmm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def direct(x, y, z, q, targets=None):
    """FP64 direct sum on the GPU for the listed targets (all when None)."""
    x, y, z, q = _f64(x), _f64(y), _f64(z), _f64(q)
    t = None if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
    nt = x.size if t is None else t.size
    out = [np.zeros(nt) for _ in range(4)]
    _check(lib().b200fmm_direct(x.size, _ptr(x), _ptr(y), _ptr(z), _ptr(q), -1 if t is None else nt,
                                None if t is None else _ptr(t, _lp), *[_ptr(o) for o in out]), "direct")
    return dict(zip(("phi", "fx", "fy", "fz"), out))


def read_fma(path):
    """A .fma (text) or .bfma (binary) particle file (FFmaGenericLoader): dict(box_width, center, data[n, nvalues])."""
    n, nv = ctypes.c_longlong(), ctypes.c_int()
    w = ctypes.c_double()
    c = np.zeros(3)
    p = str(path).encode()
    _check(lib().b200fmm_fma_read(p, ctypes.byref(n), ctypes.byref(nv), ctypes.byref(w), _ptr(c), None, 0),
           "fma_read")
    data = np.zeros(n.value * nv.value)
    _check(lib().b200fmm_fma_read(p, ctypes.byref(n), ctypes.byref(nv), ctypes.byref(w), _ptr(c), _ptr(data),
                                  data.size), "fma_read")
    return dict(box_width=w.value, center=tuple(c), data=data.reshape(n.value, nv.value))


def write_fma(path, data, box_width=1.0, center=(0.5, 0.5, 0.5)):
    """Write particles (an [n, nvalues] array: x, y, z, q[, phi, fx, fy, fz]) as .fma or .bfma."""
    data = np.ascontiguousarray(data, dtype=np.float64)
    c = _f64(center)
    _check(lib().b200fmm_fma_write(str(path).encode(), data.shape[0], data.shape[1], box_width, _ptr(c), _ptr(data)),
           "fma_write")


def shard_indices(x, y, z, height, rank, count, box_width=1.0, center=(0.5, 0.5, 0.5)):
    """Original indices of the particles that shard `rank` of `count` evaluates (FMM.set_shard): the particles
    sorted by leaf Morton key (stable), cut at the first leaf boundary at or after N * r / count for r = rank and
    rank + 1.  Host-side, the same rule as the library's device code, so that a caller knows which results a
    shard produces."""
    x, y, z = (np.asarray(a, dtype=np.float64) for a in (x, y, z))
    n = x.size
    side = 1 << (height - 1)
    leaf_w = box_width / side
    cells = []
    for a, c in ((x, center[0]), (y, center[1]), (z, center[2])):
        r = a - (c - box_width / 2)
        cells.append(np.minimum((r / leaf_w).astype(np.int64), side - 1))
    key = np.zeros(n, np.int64)
    for b in range(height - 1):  # z in the lowest bit of each triple, then y, then x
        key |= ((cells[2] >> b) & 1) << (3 * b)
        key |= ((cells[1] >> b) & 1) << (3 * b + 1)
        key |= ((cells[0] >> b) & 1) << (3 * b + 2)
    order = np.argsort(key, kind="stable")
    sk = key[order]
    starts = np.concatenate(([0], np.flatnonzero(sk[1:] != sk[:-1]) + 1, [n]))

    def boundary(r):
        if r <= 0:
            return 0
        if r >= count:
            return n
        return int(starts[np.searchsorted(starts, n * r // count, side="left")])

    return order[boundary(rank):boundary(rank + 1)]


def rel_l2(a, b):
    """Relative L2 norm sqrt(sum (b-a)^2 / sum b^2) (FMath::FAccurater, Src/Utils/FMath.hpp:590-592)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = float((b * b).sum())
    return float(np.sqrt(((a - b) ** 2).sum() / den)) if den > 0 else float(np.sqrt(((a - b) ** 2).sum()))
