import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

GOLDEN = ROOT / "tests" / "golden"
# the reference source tree (read as data where it exists): SCALFMM_REFERENCE, by default /root/reference
REFERENCE = Path(os.environ.get("SCALFMM_REFERENCE", "/root/reference"))
REFERENCE_DATA = REFERENCE / "Data"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built product library")


def load_golden(name):
    with np.load(GOLDEN / name) as f:
        return {k: f[k] for k in f.files}


@pytest.fixture(scope="session")
def golden():
    return load_golden


def read_bfma(path):
    """Binary FMA file (Src/Files/FFmaGenericLoader.hpp:189-477): int typeFReal, int nbElts, int64 N,
    double half-width, double cx, cy, cz, then N x nbElts doubles."""
    raw = Path(path).read_bytes()
    hdr_i = np.frombuffer(raw[:8], dtype=np.int32)
    n = int(np.frombuffer(raw[8:16], dtype=np.int64)[0])
    hdr = np.frombuffer(raw[16:48], dtype=np.float64)
    data = np.frombuffer(raw[48:], dtype=np.float64).reshape(n, int(hdr_i[1]))
    return dict(box_width=2 * hdr[0], center=tuple(hdr[1:4]), data=data)
