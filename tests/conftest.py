import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import Port
    return Port()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("oracle/_ref not built (needs the reference tree at build time)")
    return Ref()


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "sgm_golden.json")) as f:
        manifest = json.load(f)
    arrays = dict(np.load(os.path.join(GOLDEN, "sgm_golden.npz")))
    cases = {}
    for name, meta in manifest["cases"].items():
        c = dict(meta)
        for k, v in arrays.items():
            case, field = k.split("/", 1)
            if case == name:
                c[field] = v
        cases[name] = c
    return cases


@pytest.fixture(scope="session")
def cuda():
    """The GPU tests run the product library; without a GPU they fail (no silent skip / fallback)."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    from open_source_einstar_b200 import _native
    _native.lib()
    return torch.device("cuda:0")


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and a.tobytes() == b.tobytes()


def mismatch_report(a: np.ndarray, b: np.ndarray, n=5) -> str:
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return f"shape {a.shape} vs {b.shape}"
    av = a.view(np.uint32) if a.dtype == np.float32 else a
    bv = b.view(np.uint32) if b.dtype == np.float32 else b
    idx = np.argwhere(av != bv)
    lines = [f"{len(idx)} mismatches"]
    for i in idx[:n]:
        lines.append(f"  at {tuple(i)}: {a[tuple(i)]!r} vs {b[tuple(i)]!r}")
    return "\n".join(lines)
