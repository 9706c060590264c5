"""Shared helpers of the GPU parity tests."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


def dev(a):
    return torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def host(t):
    return t.detach().cpu().numpy()


def zeros(*shape):
    return torch.zeros(*shape, dtype=torch.float64, device="cuda")
