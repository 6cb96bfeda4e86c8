import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def params():
    import luthe_b200 as L
    return L.default_params()


@pytest.fixture(scope="session")
def keys(params):
    import luthe_b200 as L
    return L.keygen(params, 20261203)


@pytest.fixture(scope="session")
def oracle_bsk(params, keys):
    import oracle
    return oracle.OracleBsk(keys["bsk"], params.lwe_dim, params.poly_size)


def to_dev(a):
    """numpy uint array -> torch CUDA tensor holding the same bytes."""
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        a = a.view(np.int64)
    elif a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a.copy()).cuda()


def from_dev(t, dtype):
    return t.cpu().numpy().view(dtype)


@pytest.fixture(scope="session")
def engine(params, keys):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import luthe_b200 as L
    e = L.Engine(params)
    e.upload_keys(keys)
    yield e
    e.close()
