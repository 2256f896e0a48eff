"""Test configuration: the `gpu` marker, repository paths and shared helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


def golden_path(name: str) -> str:
    return os.path.join(GOLDEN, f"{name}.npz")


def load_golden(name: str):
    path = golden_path(name)
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name}.npz not generated")
    z = np.load(path)
    from cases import Proj

    p = Proj(**{k[5:]: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files if k.startswith("geom_")})
    inp = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    ref = {k[4:]: z[k] for k in z.files if k.startswith("ref_")}
    return p, inp, ref
