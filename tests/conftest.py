"""Pytest configuration: registers the ``gpu`` marker and puts the repo root on sys.path."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU and the built CUDA library")


import numpy as np  # noqa: E402
import pytest  # noqa: E402


@pytest.fixture(scope="session")
def xt():
    """The native library on cuda:0 (GPU tests only; fails loudly without it)."""
    import exatensor_b200 as X
    X.device_init(0)
    return X


class Dev:
    """Device buffers from numpy arrays via torch (plumbing only)."""

    @staticmethod
    def put(a: np.ndarray):
        import torch
        b = np.ascontiguousarray(a).view(np.uint8).ravel()
        return torch.from_numpy(b.copy()).cuda()

    @staticmethod
    def empty(nbytes: int, fill=None):
        import torch
        t = torch.empty(max(16, nbytes), dtype=torch.uint8, device="cuda")
        if fill is not None:
            t.fill_(fill)
        return t

    @staticmethod
    def get(t, dtype, count=None) -> np.ndarray:
        import torch
        torch.cuda.synchronize()
        a = t.cpu().numpy().view(dtype)
        return a[:count] if count is not None else a

    @staticmethod
    def stream():
        import torch
        return torch.cuda.current_stream().cuda_stream


@pytest.fixture(scope="session")
def dev():
    return Dev
