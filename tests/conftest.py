"""Shared test setup.

Markers: `gpu` -- needs a CUDA device (B200); everything else runs on CPU.
The CPU oracle (oracle/) is test infrastructure: tests use it only as the
checker of the CUDA path.
"""
import glob
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu on a B200)")


def load_golden(prefix: str) -> list[dict]:
    out = []
    for p in sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.json"))):
        with open(p) as f:
            out.append(json.load(f))
    return out


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    O.lib()
    return O


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
