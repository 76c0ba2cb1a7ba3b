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


def var_scale(b: np.ndarray, gamma: float = 1.4) -> np.ndarray:
    """Per-variable scale of a primitive state (rho, u, v, p): max|rho|, max|p|, and for both
    velocity components the flow's velocity scale max(|u|, |v|, a) (a component that is
    identically zero, like v in a 1-D problem, is measured against that scale)."""
    b = b.reshape(-1, b.shape[-1])
    a = np.sqrt(gamma * np.abs(b[:, 3]) / np.abs(b[:, 0]))
    vs = max(np.abs(b[:, 1]).max(), np.abs(b[:, 2]).max(), a.max())
    return np.array([np.abs(b[:, 0]).max(), vs, vs, np.abs(b[:, 3]).max()])


def rel_linf(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """max |a-b| / scale per primitive variable (last axis); scale from var_scale(b)."""
    s = var_scale(b)
    a = a.reshape(-1, a.shape[-1])
    b = b.reshape(-1, b.shape[-1])
    return np.abs(a - b).max(axis=0) / s


def rel_l1(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """sum |a-b| / (n * scale) per primitive variable; scale from var_scale(b)."""
    s = var_scale(b)
    a = a.reshape(-1, a.shape[-1])
    b = b.reshape(-1, b.shape[-1])
    return np.abs(a - b).sum(axis=0) / (a.shape[0] * s)


def rel_l1_cons(a: np.ndarray, b: np.ndarray, gamma: float = 1.4) -> np.ndarray:
    """The conventional relative L1 error per conserved variable (rho, rho u, rho v, rho E):
    sum |U(a) - U(b)| / sum |U(b)| over the cells. Both momentum components are measured
    against the momentum magnitude sum |rho V| of b, so that a component that is identically
    zero (v in a 1-D problem) has a finite denominator."""
    Ua = cons(a, gamma).reshape(-1, 4)
    Ub = cons(b, gamma).reshape(-1, 4)
    den = np.abs(Ub).sum(axis=0)
    mom = np.hypot(Ub[:, 1], Ub[:, 2]).sum()
    den[1] = den[2] = max(mom, 1e-300)
    return np.abs(Ua - Ub).sum(axis=0) / den


def cons(prim: np.ndarray, gamma: float = 1.4) -> np.ndarray:
    r, u, v, p = (prim[..., k] for k in range(4))
    return np.stack([r, r * u, r * v, p / (gamma - 1) + 0.5 * r * (u * u + v * v)], axis=-1)
