"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rockfit-dem_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    sys.path.insert(0, PKG)
    import build as _b   # rockfit-dem_b200/build.py
    _b.build()
    from oracle import build as ob
    ob.build_oracle()


_ensure_built()


@pytest.fixture(scope="session")
def rfdem():
    import rfdem as m
    return m


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.load()
    return o


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not has_cuda():
        pytest.fail("GPU test run without a CUDA device")
    import torch
    return torch


def to_dev(torch, a):
    """numpy -> CUDA tensor of the same dtype (uint64 via int64 storage)."""
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64).copy()).cuda()
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).cuda()
    return torch.from_numpy(np.ascontiguousarray(a).copy()).cuda()


def to_host(t, dtype):
    a = t.cpu().numpy()
    return a.view(dtype) if a.dtype != dtype else a
