"""Generate the golden fixtures in this directory by running the reference itself.

The reference (ScalFMM, polatory fork) is compiled from its sources by ``make -C oracle ref`` into
oracle/_ref/libscalfmm_ref.so; this script calls it through oracle/oracle.py and writes small .npz
files that pin both the CPU restatement (oracle/fmm_oracle.c) and the CUDA product.  Inputs are seeded
synthetic particles (uniform in the unit cube, charges uniform in [-1, 1]) and are stored with the
outputs, so the fixtures are self-contained.

Run from the repository root:  OPENBLAS_NUM_THREADS=1 python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent
CENTER = (0.5, 0.5, 0.5)


def particles(n, seed, nrhs=1):
    rng = np.random.default_rng(seed)
    pos = rng.random((3, n))
    q = rng.uniform(-1.0, 1.0, (nrhs, n)) if nrhs > 1 else rng.uniform(-1.0, 1.0, n)
    return pos, q


def sym_ops():
    for order in (3, 4, 5, 6, 7):
        ranks, uv, pind, pvec = O.ref_sym_operators(order)
        far = np.array([t for t in range(343) if max(abs(t // 49 - 3), abs((t // 7) % 7 - 3), abs(t % 7 - 3)) > 1])
        np.savez_compressed(OUT / f"sym_ops_p{order}.npz", order=order, eps=10.0 ** (-order), ranks=ranks, uv=uv,
                            pindices=pind, pvectors_far=pvec[far], far_slots=far)


def fmm_cases():
    cases = [
        # name, kind, order, height, n, seed, nrhs
        ("sym_p5_h4_n2000", O.CHEB_SYM, 5, 4, 2000, 11, 1),
        ("sym_p7_h4_n2000", O.CHEB_SYM, 7, 4, 2000, 12, 1),
        ("sym_p4_h5_n3000", O.CHEB_SYM, 4, 5, 3000, 13, 1),
        ("sym_p6_h3_n500", O.CHEB_SYM, 6, 3, 500, 14, 1),
        ("dense_p4_h4_n2000", O.CHEB_DENSE, 4, 4, 2000, 15, 1),
        ("dense_p5_h3_n1000", O.CHEB_DENSE, 5, 3, 1000, 16, 1),
        ("sym_p5_h4_n1500_rhs16", O.CHEB_SYM, 5, 4, 1500, 17, 16),
        # the reference's FUnifKernel: its M2L runs in Fourier space (FFTW calls served by oracle/ref/fftw)
        ("lagrange_p4_h4_n2000", O.LAGRANGE, 4, 4, 2000, 18, 1),
        ("lagrange_p6_h3_n1000", O.LAGRANGE, 6, 3, 1000, 19, 1),
    ]
    only = set(sys.argv[1:])  # optional case names: regenerate just those
    for name, kind, order, height, n, seed, nrhs in cases:
        if only and name not in only:
            continue
        pos, q = particles(n, seed, nrhs)
        r = O.ref_fmm(kind, order, height, 1.0, CENTER, pos[0], pos[1], pos[2], q)
        np.savez_compressed(OUT / f"fmm_{name}.npz", kind=kind, order=order, height=height, x=pos[0], y=pos[1],
                            z=pos[2], q=q, phi=r["phi"], fx=r["fx"], fy=r["fy"], fz=r["fz"])


def expansion_case():
    order, height, n = 4, 4, 1000
    pos, q = particles(n, 21)
    e = O.ref_expansions(O.CHEB_SYM, order, height, 1.0, CENTER, pos[0], pos[1], pos[2], q)
    keep = e["levels"] >= 2
    np.savez_compressed(OUT / "expansions_sym_p4_h4_n1000.npz", order=order, height=height, x=pos[0], y=pos[1],
                        z=pos[2], q=q, levels=e["levels"][keep], mortons=e["mortons"][keep],
                        multipoles=e["multipoles"][keep, 0], locals=e["locals"][keep, 0])


def direct_case():
    pos, q = particles(1500, 31)
    d = O.ref_direct(pos[0], pos[1], pos[2], q)
    np.savez_compressed(OUT / "direct_n1500.npz", x=pos[0], y=pos[1], z=pos[2], q=q, **d)


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("oracle/_ref/libscalfmm_ref.so is missing: run `make -C oracle ref` where the reference exists")
    if len(sys.argv) > 1:
        fmm_cases()
    else:
        sym_ops()
        fmm_cases()
        expansion_case()
        direct_case()
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)
