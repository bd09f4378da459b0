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


@pytest.fixture(scope="session")
def ca_sample(oracle, inp_file):
    """The reference's CA sample (sample_model/CA): mesh_o.inp (E = 2.1e5,
    nu = 0.3) and its change file (384 deleted C3D4).  The modified model is
    the same mesh with E = 0 on the deleted elements."""
    import scipy.sparse as sp
    import openfea_b200 as ob
    from openfea_b200 import meshgen as mg
    from oracle import ca_oracle
    E0, nu = 2.1e5, 0.3
    d = ob.inp_read(inp_file("mesh_o.inp"))
    m0 = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, E0, nu)
    fm = oracle.free_index(m0.nd, m0.fix)
    n = 3 * int((fm >= 0).sum())
    cp, ri, val = oracle.assemble(m0, fm)
    K0 = sp.csc_matrix((val, ri, cp), shape=(n, n))
    f = ob.build_single_load(m0.nd, fm, d["load_set"], d["load_dof"], d["load_value"])
    ci = ob.ca_info_read(inp_file("CA_info.txt"))
    dK = ca_oracle.delta_k(oracle, ci, m0.fix, fm, n, E0, nu)
    # the changed elements among the mesh's elements (same node sets)
    key = {tuple(sorted(t[t > 0])): e for e, t in enumerate(d["topo"])}
    idx = np.array([key[tuple(sorted(t[t >= 0] + 1))] for t in ci["topo"]])
    Em = np.full(m0.ne, E0)
    Em[idx] = 0.0
    m1 = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], Em, E0, nu)
    return dict(d=d, m0=m0, m1=m1, fm=fm, n=n, K0=K0, f=f, ci=ci, dK=dK, deleted=idx, E0=E0, nu=nu)
