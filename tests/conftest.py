import gzip
import os
import shutil
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    return Reference()


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name))
    return load


@pytest.fixture(scope="session")
def inp_file(tmp_path_factory):
    d = tmp_path_factory.mktemp("inp")

    def get(name):
        out = d / name
        if not out.exists():
            with gzip.open(os.path.join(GOLDEN, name + ".gz"), "rb") as fi, open(out, "wb") as fo:
                shutil.copyfileobj(fi, fo)
        return str(out)
    return get


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx_factory():
    if not has_gpu():
        pytest.skip("no GPU")
    import openfea_b200 as ob
    return ob.Context
