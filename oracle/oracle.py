"""ctypes bindings for the CPU checkers -- TEST INFRASTRUCTURE ONLY.

* ``liboracle.so``: the C restatement of the reference's FMM hot path (fmm_oracle.c).
* ``_ref/libscalfmm_ref.so``: the reference's own FFmmAlgorithmThread + Chebyshev kernels compiled
  from its sources (ref/ref_driver.cpp); optional -- absent when it was never built.

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libscalfmm_ref.so"

CHEB_SYM, CHEB_DENSE, LAGRANGE = 0, 1, 2
P2P, P2M, M2M, M2L, L2L, L2P = 1, 2, 4, 8, 16, 32
ALL_OPS = P2P | P2M | M2M | M2L | L2L | L2P

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_up = ctypes.POINTER(ctypes.c_uint)
_lp = ctypes.POINTER(ctypes.c_longlong)


def _p(a, t=_dp):
    return a.ctypes.data_as(t) if a is not None else None


class _Config(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("order", ctypes.c_int),
        ("height", ctypes.c_int),
        ("nrhs", ctypes.c_int),
        ("nthreads", ctypes.c_int),
        ("box_width", ctypes.c_double),
        ("center", ctypes.c_double * 3),
        ("sym_ranks", _ip),
        ("sym_uv", _dp),
    ]


class _Dump(ctypes.Structure):
    _fields_ = [
        ("cap", ctypes.c_longlong),
        ("count", ctypes.c_longlong),
        ("levels", _ip),
        ("mortons", _lp),
        ("multipoles", _dp),
        ("locals", _dp),
    ]


_lib = None
_ref = None


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build_oracle()
        _lib = ctypes.CDLL(str(ORACLE_SO))
        _lib.orc_fmm.argtypes = [ctypes.POINTER(_Config), ctypes.c_longlong, _dp, _dp, _dp, _dp, ctypes.c_uint,
                                 _dp, _dp, _dp, _dp, ctypes.POINTER(_Dump)]
        _lib.orc_direct.argtypes = [ctypes.c_longlong, _dp, _dp, _dp, _dp, ctypes.c_longlong, _lp, ctypes.c_int,
                                    _dp, _dp, _dp, _dp]
        _lib.orc_morton_keys.argtypes = [ctypes.c_longlong, _dp, _dp, _dp, ctypes.c_double, _dp, ctypes.c_int, _lp]
        _lib.orc_morton_encode.restype = ctypes.c_longlong
        _lib.orc_morton_encode.argtypes = [ctypes.c_int] * 3
        _lib.orc_morton_decode.argtypes = [ctypes.c_longlong, _ip, _ip, _ip]
        _lib.orc_sym_tables.argtypes = [ctypes.c_int, _up, _up]
        _lib.orc_leaf_neighbors.argtypes = [ctypes.c_int] * 4 + [_lp, _ip]
        _lib.orc_interaction_list.argtypes = [ctypes.c_int] * 4 + [_lp, _ip]
    return _lib


def ref_available() -> bool:
    return REF_SO.exists()


def ref():
    global _ref
    if _ref is None:
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        _ref = ctypes.CDLL(str(REF_SO))
        _ref.ref_fmm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp,
                                 ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_longlong, _dp, _dp, _dp, _dp,
                                 ctypes.c_uint, _dp, _dp, _dp, _dp, _dp]
        _ref.ref_expansions.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                        _dp, ctypes.c_double, ctypes.c_int, ctypes.c_longlong, _dp, _dp, _dp, _dp,
                                        ctypes.c_uint, ctypes.c_longlong, _lp, _ip, _lp, _dp, _dp]
        _ref.ref_sym_operators.argtypes = [ctypes.c_int, ctypes.c_double, _ip, _up, _up, _dp, ctypes.c_longlong]
        _ref.ref_direct.argtypes = [ctypes.c_longlong, _dp, _dp, _dp, _dp, ctypes.c_longlong, _lp, ctypes.c_int,
                                    _dp, _dp, _dp, _dp]
    return _ref


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ------------------------------------------------------------------------------------------------
# restatement (liboracle.so)
# ------------------------------------------------------------------------------------------------

def fmm(kind, order, height, box_width, center, x, y, z, q, ops=ALL_OPS, sym_ranks=None, sym_uv=None,
        nthreads=0, dump=False):
    """Full FMM on the CPU restatement.  q has shape (n,) or (nrhs, n).  Returns dict of arrays."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    q = _f64(q)
    nrhs = 1 if q.ndim == 1 else q.shape[0]
    n = x.size
    cfg = _Config(kind, order, height, nrhs, nthreads or os.cpu_count(), box_width,
                  (ctypes.c_double * 3)(*center), None, None)
    if kind == CHEB_SYM:
        sym_ranks = np.ascontiguousarray(sym_ranks, dtype=np.int32)
        sym_uv = _f64(sym_uv)
        cfg.sym_ranks = _p(sym_ranks, _ip)
        cfg.sym_uv = _p(sym_uv)
    out = {k: np.zeros(nrhs * n) for k in ("phi", "fx", "fy", "fz")}
    d = None
    if dump:
        nn = order ** 3
        cap = n * height + 16
        bufs = dict(levels=np.zeros(cap, np.int32), mortons=np.zeros(cap, np.int64),
                    multipoles=np.zeros(cap * nrhs * nn), locals=np.zeros(cap * nrhs * nn))
        d = _Dump(cap, 0, _p(bufs["levels"], _ip), _p(bufs["mortons"], _lp), _p(bufs["multipoles"]),
                  _p(bufs["locals"]))
    rc = lib().orc_fmm(ctypes.byref(cfg), n, _p(x), _p(y), _p(z), _p(q), ops, _p(out["phi"]), _p(out["fx"]),
                       _p(out["fy"]), _p(out["fz"]), ctypes.byref(d) if d is not None else None)
    if rc != 0:
        raise RuntimeError(f"orc_fmm failed: {rc}")
    res = {k: v.reshape(nrhs, n) if nrhs > 1 else v for k, v in out.items()}
    if dump:
        c = d.count
        nn = order ** 3
        res["levels"] = bufs["levels"][:c].copy()
        res["mortons"] = bufs["mortons"][:c].copy()
        res["multipoles"] = bufs["multipoles"][: c * nrhs * nn].reshape(c, nrhs, nn).copy()
        res["locals"] = bufs["locals"][: c * nrhs * nn].reshape(c, nrhs, nn).copy()
    return res


def direct(x, y, z, q, targets=None, nthreads=0):
    x, y, z, q = _f64(x), _f64(y), _f64(z), _f64(q)
    n = x.size
    t = None if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
    nt = n if t is None else t.size
    out = [np.zeros(nt) for _ in range(4)]
    lib().orc_direct(n, _p(x), _p(y), _p(z), _p(q), -1 if t is None else nt, _p(t, _lp),
                     nthreads or os.cpu_count(), *[_p(o) for o in out])
    return dict(zip(("phi", "fx", "fy", "fz"), out))


def morton_keys(x, y, z, box_width, center, height):
    x, y, z = _f64(x), _f64(y), _f64(z)
    keys = np.zeros(x.size, np.int64)
    c = _f64(center)
    rc = lib().orc_morton_keys(x.size, _p(x), _p(y), _p(z), box_width, _p(c), height, _p(keys, _lp))
    if rc != 0:
        raise ValueError("particle outside the box")
    return keys


def morton_encode(ix, iy, iz):
    return lib().orc_morton_encode(ix, iy, iz)


def morton_decode(key):
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib().orc_morton_decode(key, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


def sym_tables(order):
    nn = order ** 3
    pind = np.zeros(343, np.uint32)
    pvec = np.zeros(343 * nn, np.uint32)
    lib().orc_sym_tables(order, _p(pind, _up), _p(pvec, _up))
    return pind, pvec.reshape(343, nn)


def leaf_neighbors(ix, iy, iz, height):
    keys = np.zeros(26, np.int64)
    pos = np.zeros(26, np.int32)
    k = lib().orc_leaf_neighbors(ix, iy, iz, height, _p(keys, _lp), _p(pos, _ip))
    return keys[:k], pos[:k]


def interaction_list(ix, iy, iz, level):
    keys = np.zeros(216, np.int64)
    pos = np.zeros(216, np.int32)
    k = lib().orc_interaction_list(ix, iy, iz, level, _p(keys, _lp), _p(pos, _ip))
    return keys[:k], pos[:k]


# ------------------------------------------------------------------------------------------------
# the reference itself (oracle/_ref/libscalfmm_ref.so)
# ------------------------------------------------------------------------------------------------

def ref_fmm(kind, order, height, box_width, center, x, y, z, q, eps=None, ops=ALL_OPS, nthreads=0,
            sequential=False):
    x, y, z, q = _f64(x), _f64(y), _f64(z), _f64(q)
    nrhs = 1 if q.ndim == 1 else q.shape[0]
    n = x.size
    eps = 10.0 ** (-order) if eps is None else eps
    out = [np.zeros(nrhs * n) for _ in range(4)]
    times = np.zeros(3)
    c = _f64(center)
    rc = ref().ref_fmm(kind, order, nrhs, height, box_width, _p(c), eps, nthreads or os.cpu_count(),
                       int(sequential), n, _p(x), _p(y), _p(z), _p(q), ops, *[_p(o) for o in out], _p(times))
    if rc != 0:
        raise RuntimeError(f"ref_fmm failed: {rc}")
    res = {k: (v.reshape(nrhs, n) if nrhs > 1 else v) for k, v in zip(("phi", "fx", "fy", "fz"), out)}
    res["times"] = dict(kernel=times[0], insert=times[1], execute=times[2])
    return res


def ref_expansions(kind, order, height, box_width, center, x, y, z, q, eps=None, ops=ALL_OPS, nthreads=0):
    x, y, z, q = _f64(x), _f64(y), _f64(z), _f64(q)
    nrhs = 1 if q.ndim == 1 else q.shape[0]
    n = x.size
    nn = order ** 3
    eps = 10.0 ** (-order) if eps is None else eps
    cap = n * height + 16
    count = ctypes.c_longlong(0)
    levels = np.zeros(cap, np.int32)
    mortons = np.zeros(cap, np.int64)
    mul = np.zeros(cap * nrhs * nn)
    loc = np.zeros(cap * nrhs * nn)
    c = _f64(center)
    rc = ref().ref_expansions(kind, order, nrhs, height, box_width, _p(c), eps, nthreads or os.cpu_count(), n,
                              _p(x), _p(y), _p(z), _p(q), ops, cap, ctypes.byref(count), _p(levels, _ip),
                              _p(mortons, _lp), _p(mul), _p(loc))
    if rc != 0:
        raise RuntimeError(f"ref_expansions failed: {rc}")
    k = count.value
    return dict(levels=levels[:k], mortons=mortons[:k], multipoles=mul[: k * nrhs * nn].reshape(k, nrhs, nn),
                locals=loc[: k * nrhs * nn].reshape(k, nrhs, nn))


def ref_sym_operators(order, eps=None):
    nn = order ** 3
    eps = 10.0 ** (-order) if eps is None else eps
    ranks = np.zeros(343, np.int32)
    pind = np.zeros(343, np.uint32)
    pvec = np.zeros(343 * nn, np.uint32)
    cap = 16 * 2 * nn * nn
    uv = np.zeros(cap)
    rc = ref().ref_sym_operators(order, eps, _p(ranks, _ip), _p(pind, _up), _p(pvec, _up), _p(uv), cap)
    if rc != 0:
        raise RuntimeError(f"ref_sym_operators failed: {rc}")
    used = int(2 * ranks.sum() * nn)
    return ranks, uv[:used].copy(), pind, pvec.reshape(343, nn)


def ref_direct(x, y, z, q, targets=None, nthreads=0):
    x, y, z, q = _f64(x), _f64(y), _f64(z), _f64(q)
    n = x.size
    t = None if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
    nt = n if t is None else t.size
    out = [np.zeros(nt) for _ in range(4)]
    ref().ref_direct(n, _p(x), _p(y), _p(z), _p(q), -1 if t is None else nt, _p(t, _lp),
                     nthreads or os.cpu_count(), *[_p(o) for o in out])
    return dict(zip(("phi", "fx", "fy", "fz"), out))


def unpack_sym(ranks, uv, order):
    """{slot: (U, V)} from the reference storage layout."""
    nn = order ** 3
    ops = {}
    off = 0
    for t in range(343):
        r = int(ranks[t])
        if r > 0:
            U = uv[off: off + r * nn].reshape(r, nn).T
            V = uv[off + r * nn: off + 2 * r * nn].reshape(r, nn).T
            ops[t] = (U, V)
            off += 2 * r * nn
    return ops


def rel_l2(a, b):
    """FMath::FAccurater relative L2 norm (Src/Utils/FMath.hpp:590-592): sqrt(sum (b-a)^2 / sum b^2)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = float((b * b).sum())
    return float(np.sqrt(((a - b) ** 2).sum() / den)) if den > 0 else float(np.sqrt(((a - b) ** 2).sum()))
