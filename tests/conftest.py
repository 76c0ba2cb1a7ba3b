"""pytest configuration: the `gpu` marker and shared helpers for the parity tests."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path")


def have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    return oracle.load()


def rel_linf(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """max |a-b| / max |b| per primitive variable (last axis)."""
    a = a.reshape(-1, a.shape[-1])
    b = b.reshape(-1, b.shape[-1])
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return np.abs(a - b).max(axis=0) / scale


def rel_l1(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = a.reshape(-1, a.shape[-1])
    b = b.reshape(-1, b.shape[-1])
    return np.abs(a - b).sum(axis=0) / np.maximum(np.abs(b).sum(axis=0), 1e-300)


def cons(prim: np.ndarray, gamma: float = 1.4) -> np.ndarray:
    r, u, v, p = (prim[..., k] for k in range(4))
    return np.stack([r, r * u, r * v, p / (gamma - 1) + 0.5 * r * (u * u + v * v)], axis=-1)
