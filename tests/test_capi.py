"""The ScalFMM C user API shim (include/b200fmm_capi.h) and the .fma / .bfma particle files.

CPU tests (no GPU): the shim's host-side bookkeeping -- insertion order, physical values, positions, forces and
potentials with their _npart variants, the utility functions -- and the particle file reader / writer, pinned
against the reference's own fixture Data/UTest/DirectDouble.bfma where the reference tree is present.

GPU tests: a C program (tests/capi/capi_check.c) compiled against the shim's header drives the Chebyshev FMM
like a C caller of the reference; its output matches the reference's FFmmAlgorithmThread + FChebSymKernel<7>
(what the reference's C API runs for `chebyshev`) within 50 * 10^-7, the bar of this library's own FP64
operator compression against the reference's.  A ctypes test checks the reference's accumulate (+=) semantics
and the handling of moved particles.
"""
import ctypes
import shutil
import subprocess

import numpy as np
import pytest

import scalfmm_b200 as S
from conftest import REFERENCE_DATA, ROOT, read_bfma

CENTER = (0.5, 0.5, 0.5)
BOTH = 2


def capi():
    L = S.lib()
    L.scalfmm_init.restype = ctypes.c_void_p
    L.scalfmm_init.argtypes = [ctypes.c_int, ctypes.c_int]
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    for name, args in {
        "scalfmm_tree_insert_particles": [vp, ctypes.c_int, dp, dp, dp, ctypes.c_int],
        "scalfmm_tree_insert_particles_xyz": [vp, ctypes.c_int, dp, ctypes.c_int],
        "scalfmm_set_physical_values": [vp, ctypes.c_int, dp, ctypes.c_int],
        "scalfmm_get_physical_values": [vp, ctypes.c_int, dp, ctypes.c_int],
        "scalfmm_set_physical_values_npart": [vp, ctypes.c_int, ip, dp, ctypes.c_int],
        "scalfmm_get_physical_values_npart": [vp, ctypes.c_int, ip, dp, ctypes.c_int],
        "scalfmm_get_positions_xyz": [vp, ctypes.c_int, dp, ctypes.c_int],
        "scalfmm_get_positions_npart": [vp, ctypes.c_int, ip, dp, dp, dp, ctypes.c_int],
        "scalfmm_set_positions_xyz_npart": [vp, ctypes.c_int, ip, dp, ctypes.c_int],
        "scalfmm_add_to_positions": [vp, ctypes.c_int, dp, dp, dp, ctypes.c_int],
        "scalfmm_set_positions": [vp, ctypes.c_int, dp, dp, dp, ctypes.c_int],
        "scalfmm_get_potentials": [vp, ctypes.c_int, dp, ctypes.c_int],
        "scalfmm_set_potentials": [vp, ctypes.c_int, dp, ctypes.c_int],
        "scalfmm_get_forces": [vp, ctypes.c_int, dp, dp, dp, ctypes.c_int],
        "scalfmm_set_forces_xyz": [vp, ctypes.c_int, dp, ctypes.c_int],
        "scalfmm_get_forces_npart": [vp, ctypes.c_int, ip, dp, dp, dp, ctypes.c_int],
        "scalfmm_update_tree": [vp],
        "scalfmm_execute_fmm": [vp],
        "scalfmm_execute_fmm_far_field": [vp],
        "scalfmm_get_nb_timers": [vp],
        "scalfmm_get_timers": [vp, dp],
        "scalfmm_dealloc_handle": [vp, vp],
        "scalfmm_utils_parentChildPosition": [ctypes.c_int, ip],
        "scalfmm_utils_interactionPosition": [ctypes.c_int, ip],
        "scalfmm_algorithm_config": [vp, ctypes.c_int],
        "scalfmm_apply_on_leaf": [vp, vp],
        "b200fmm_capi_status": [vp],
        "b200fmm_capi_set_precision": [vp, ctypes.c_int],
    }.items():
        getattr(L, name).argtypes = args
    return L


def P(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def test_capi_header_symbols_are_exported():
    import re

    text = (ROOT / "include" / "b200fmm_capi.h").read_text()
    names = set(re.findall(r"B200FMM_API\s+[\w\s\*]*?\b((?:scalfmm|b200fmm)_\w+)\s*\(", text))
    assert len(names) >= 49
    L = S.lib()
    for name in names:
        assert hasattr(L, name), name


def test_capi_host_bookkeeping_without_a_gpu():
    """Insertion order, physical values, positions, potentials and forces, _npart variants: all host state,
    exercised before any tree is built (no device involved)."""
    L = capi()
    assert L.scalfmm_init(0, 1) is None  # user_defined_kernel is not part of this library
    h = L.scalfmm_init(1, 1)  # chebyshev, multi_thread
    assert h
    rng = np.random.default_rng(2)
    xyz = rng.random((50, 3))
    L.scalfmm_tree_insert_particles_xyz(h, 30, P(np.ascontiguousarray(xyz[:30])), BOTH)
    x2, y2, z2 = (np.ascontiguousarray(xyz[30:, k]) for k in range(3))
    L.scalfmm_tree_insert_particles(h, 20, P(x2), P(y2), P(z2), BOTH)  # appended after the first 30
    got = np.zeros((50, 3))
    L.scalfmm_get_positions_xyz(h, 50, P(got), BOTH)
    assert np.array_equal(got, xyz)
    q = rng.uniform(-1, 1, 50)
    L.scalfmm_set_physical_values(h, 50, P(q), BOTH)
    idx = np.array([3, 41, 7], np.int32)
    L.scalfmm_set_physical_values_npart(h, 3, P(idx, ctypes.c_int), P(np.array([9.0, 8.0, 7.0])), BOTH)
    q[idx] = [9.0, 8.0, 7.0]
    back = np.zeros(50)
    L.scalfmm_get_physical_values(h, 50, P(back), BOTH)
    assert np.array_equal(back, q)
    sub = np.zeros(3)
    L.scalfmm_get_physical_values_npart(h, 3, P(idx, ctypes.c_int), P(sub), BOTH)
    assert np.array_equal(sub, [9.0, 8.0, 7.0])
    # potentials and forces start at zero; set_ overwrites them
    phi = np.zeros(50)
    L.scalfmm_get_potentials(h, 50, P(phi), BOTH)
    assert not phi.any()
    L.scalfmm_set_potentials(h, 50, P(np.arange(50.0)), BOTH)
    L.scalfmm_get_potentials(h, 50, P(phi), BOTH)
    assert np.array_equal(phi, np.arange(50.0))
    f = np.arange(150.0).reshape(50, 3)
    L.scalfmm_set_forces_xyz(h, 50, P(f), BOTH)
    fx, fy, fz = np.zeros(3), np.zeros(3), np.zeros(3)
    L.scalfmm_get_forces_npart(h, 3, P(idx, ctypes.c_int), P(fx), P(fy), P(fz), BOTH)
    assert np.array_equal(np.stack([fx, fy, fz], 1), f[idx])
    # moving particles
    d = np.full(50, 0.001)
    L.scalfmm_add_to_positions(h, 50, P(d), P(d), P(d), BOTH)
    L.scalfmm_set_positions_xyz_npart(h, 1, P(np.array([5], np.int32), ctypes.c_int), P(np.array([0.1, 0.2, 0.3])),
                                      BOTH)
    px, py, pz = np.zeros(2), np.zeros(2), np.zeros(2)
    L.scalfmm_get_positions_npart(h, 2, P(np.array([5, 6], np.int32), ctypes.c_int), P(px), P(py), P(pz), BOTH)
    assert np.allclose([px[0], py[0], pz[0]], [0.1, 0.2, 0.3])
    assert np.allclose([px[1], py[1], pz[1]], xyz[6] + 0.001)
    # a count that differs from the inserted particles is refused, the state stays
    L.scalfmm_get_potentials(h, 49, P(phi), BOTH)
    assert L.b200fmm_capi_status(h) == 1
    # algorithms outside sequential / multi_thread are refused
    L.scalfmm_algorithm_config(h, 2)
    assert L.b200fmm_capi_status(h) == 6
    assert L.scalfmm_get_nb_timers(h) == 9
    L.scalfmm_dealloc_handle(h, None)


def test_capi_utilities_follow_the_reference_encodings():
    L = capi()
    out = np.zeros(3, np.int32)
    for c in range(8):
        L.scalfmm_utils_parentChildPosition(c, P(out, ctypes.c_int))
        assert list(out) == [1 if (c >> 2) & 1 else -1, 1 if (c >> 1) & 1 else -1, 1 if c & 1 else -1]
    for t in (0, 171, 342, 100):
        L.scalfmm_utils_interactionPosition(t, P(out, ctypes.c_int))
        assert list(out) == [t // 49 - 3, (t // 7) % 7 - 3, t % 7 - 3]


@pytest.mark.parametrize("suffix", [".bfma", ".fma"])
def test_fma_round_trip(tmp_path, suffix):
    rng = np.random.default_rng(4)
    data = np.column_stack([rng.random((100, 3)), rng.uniform(-1, 1, (100, 5))])
    path = tmp_path / f"p{suffix}"
    S.write_fma(path, data, box_width=2.5, center=(0.1, -0.2, 0.3))
    f = S.read_fma(path)
    assert f["box_width"] == 2.5 and f["center"] == (0.1, -0.2, 0.3)
    assert np.array_equal(f["data"], data)  # the text form carries 17 significant digits


def test_fma_rejects_unknown_names_and_sizes(tmp_path):
    with pytest.raises(S.B200FmmError):
        S.write_fma(tmp_path / "p.txt", np.zeros((2, 4)))
    with pytest.raises(S.B200FmmError):
        S.write_fma(tmp_path / "p.bfma", np.zeros((2, 3)))  # at least x, y, z, q
    (tmp_path / "bad.bfma").write_bytes(b"\x04\x00\x00\x00\x04\x00\x00\x00")  # 4-byte reals, truncated
    with pytest.raises(S.B200FmmError):
        S.read_fma(tmp_path / "bad.bfma")


@pytest.mark.skipif(not (REFERENCE_DATA / "UTest" / "DirectDouble.bfma").exists(), reason="reference data absent")
def test_fma_reads_the_reference_fixture():
    """The reference's own binary fixture (5000 particles, x y z q phi fx fy fz) reads identically through the
    library's reader and the test suite's independent one."""
    path = REFERENCE_DATA / "UTest" / "DirectDouble.bfma"
    mine = S.read_fma(path)
    ref = read_bfma(path)
    assert mine["box_width"] == ref["box_width"] and mine["center"] == ref["center"]
    assert np.array_equal(mine["data"], ref["data"])


# ---- GPU ------------------------------------------------------------------------------------------------
def build_capi_check(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    exe = tmp_path / "capi_check"
    subprocess.run([cc, "-std=c99", "-O1", "-I", str(ROOT / "include"), str(ROOT / "tests" / "capi" / "capi_check.c"),
                    "-L", str(ROOT / "scalfmm_b200"), "-lb200fmm", f"-Wl,-rpath,{ROOT / 'scalfmm_b200'}", "-o",
                    str(exe)], check=True)
    return exe


@pytest.mark.gpu
@pytest.mark.parametrize("suffix", [".bfma", ".fma"])
def test_c_program_matches_reference_chebyshev(golden, tmp_path, suffix):
    g = golden("fmm_sym_p7_h4_n2000.npz")
    exe = build_capi_check(tmp_path)
    src = tmp_path / f"in{suffix}"
    S.write_fma(src, np.column_stack([g["x"], g["y"], g["z"], g["q"]]), 1.0, CENTER)
    out = tmp_path / f"out{suffix}"
    r = subprocess.run([str(exe), str(src), str(out), str(int(g["height"]))], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    res = S.read_fma(out)["data"]
    tol = 50 * 10.0 ** -7  # own operator compression against the reference's, FP64
    for k, col in (("phi", 4), ("fx", 5), ("fy", 6), ("fz", 7)):
        assert S.rel_l2(res[:, col], g[k]) < tol, (k, S.rel_l2(res[:, col], g[k]))


@pytest.mark.gpu
def test_capi_accumulates_and_follows_moved_particles(golden):
    L = capi()
    g = golden("fmm_sym_p7_h4_n2000.npz")
    n = g["x"].size
    h = L.scalfmm_init(1, 0)
    cells = (ctypes.c_void_p * 5)()
    leaves = (ctypes.c_void_p * 5)()
    L.scalfmm_build_tree.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                     type(cells), type(leaves)]
    L.scalfmm_build_tree(h, int(g["height"]), 1.0, P(np.array(CENTER)), cells, leaves)
    x, y, z, q = (np.ascontiguousarray(g[k]) for k in ("x", "y", "z", "q"))
    L.scalfmm_tree_insert_particles(h, n, P(x), P(y), P(z), BOTH)
    L.scalfmm_set_physical_values(h, n, P(q), BOTH)
    L.scalfmm_execute_fmm(h)
    phi1 = np.zeros(n)
    L.scalfmm_get_potentials(h, n, P(phi1), BOTH)
    assert S.rel_l2(phi1, g["phi"]) < 5e-6
    L.scalfmm_execute_fmm(h)  # the containers accumulate
    phi2 = np.zeros(n)
    L.scalfmm_get_potentials(h, n, P(phi2), BOTH)
    assert S.rel_l2(phi2, 2 * phi1) < 1e-14
    # far field alone, from zeroed potentials
    L.scalfmm_set_potentials(h, n, P(np.zeros(n)), BOTH)
    L.scalfmm_execute_fmm_far_field(h)
    far = np.zeros(n)
    L.scalfmm_get_potentials(h, n, P(far), BOTH)
    assert 0 < np.abs(far).sum() and S.rel_l2(far, phi1) > 1e-3
    # move every particle, update, recompute from zero: the result follows the new positions
    xs = np.ascontiguousarray(x[::-1])
    ys = np.ascontiguousarray(y[::-1])
    zs = np.ascontiguousarray(z[::-1])
    L.scalfmm_set_positions(h, n, P(xs), P(ys), P(zs), BOTH)
    L.scalfmm_update_tree(h)
    L.scalfmm_set_potentials(h, n, P(np.zeros(n)), BOTH)
    L.scalfmm_execute_fmm(h)
    moved = np.zeros(n)
    L.scalfmm_get_potentials(h, n, P(moved), BOTH)
    f = S.FMM("cheb_sym", 7, int(g["height"]), precision="fp64")
    f.set_particles(xs, ys, zs, q)
    f.execute()
    assert S.rel_l2(moved, f.results()["phi"]) < 1e-14
    f.close()
    # apply_on_leaf visits every particle once, leaf by leaf in Morton order
    seen = []
    CB = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong),
                          ctypes.c_longlong, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_void_p,
                          ctypes.c_void_p)
    keys = []

    def on_leaf(level, nb, idx, key, llc, cell, leaf, user):
        seen.extend(idx[i] for i in range(nb))
        keys.append(key)

    cb = CB(on_leaf)
    L.scalfmm_apply_on_leaf(h, ctypes.cast(cb, ctypes.c_void_p))
    assert sorted(seen) == list(range(n)) and keys == sorted(keys)
    t = np.zeros(9)
    L.scalfmm_get_timers(h, P(t))
    assert t[2] > 0  # M2L
    assert L.b200fmm_capi_status(h) == 0
    L.scalfmm_dealloc_handle(h, None)
