"""CA reanalysis on the CPU: the change-file reader (ofea_ca_info_read) and
the oracle's restatement of src/ca_analysis.cpp, pinned to the reference's
shipped CA output sample_model/CA/cadcae_ca.vtk."""
import numpy as np
import pytest
import scipy.sparse as sp

import openfea_b200 as ob
from oracle import ca_oracle


def test_ca_info_reader(ca_sample):
    ci = ca_sample["ci"]
    assert ci["xyz"].shape == (625, 3) and ci["kind"].shape == (384,)
    assert set(ci["kind"].tolist()) == {0} and set(ci["etype"].tolist()) == {0}
    assert np.all(ci["topo"][:, 4:] == -1) and ci["topo"][:, :4].min() >= 0 and ci["topo"].max() < 625
    nm = ci["node_map"]
    assert (nm >= 0).sum() == 525 and sorted(nm[nm >= 0].tolist()) == list(range(525))
    # deletion only: the modified coordinates are the original ones
    assert np.array_equal(ci["xyz"], ca_sample["d"]["xyz"])


def test_ca_info_reader_rejects_malformed(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("*nodes_all, 2\n0, 0, 0\n1, 0, 0\n*eles_change, 1, type=C3D4\n0, 0, 1, 5, 1\n*End Assembly\n"
                 "*idref2new, 2\n0\n1\n*End File\n")
    with pytest.raises(ob.OfeaError) as e:
        ob.ca_info_read(str(p))  # node 5 is out of range
    assert e.value.code == -10  # OFEA_ERR_IO
    with pytest.raises(ob.OfeaError):
        ob.ca_info_read(str(tmp_path / "missing.txt"))


def test_delta_k_equals_modified_minus_original(oracle, ca_sample):
    """ΔK of the change list (element by element, as the reference) equals
    K(mesh with E = 0 on the deleted elements) - K0: the form the device path
    uses."""
    s = ca_sample
    cp, ri, val = oracle.assemble(s["m1"], s["fm"])
    K1 = sp.csc_matrix((val, ri, cp), shape=(s["n"], s["n"]))
    diff = abs(K1 - (s["K0"] + s["dK"])).max()
    assert diff <= 1e-14 * abs(s["K0"]).max()


def test_oracle_reproduces_shipped_ca_output(ca_sample, golden):
    """The shipped output was made with the basis degenerate (the driver's
    Pardiso solve leaves no SuperLU factor to re-solve with), i.e. the
    Galerkin solution on span(u_0): n_basis = 1 here, to print precision."""
    s = ca_sample
    u0 = sp.linalg.spsolve(s["K0"].tocsc(), s["f"])
    u = ca_oracle.ca_reanalysis(s["K0"], s["dK"], s["f"], u0, 1)
    un = ca_oracle.to_modified_nodes(u, s["fm"], s["ci"]["node_map"])
    ug = golden("cadcae_ca_u.npz")["u"]
    assert un.shape == ug.shape == (525, 3)
    assert np.linalg.norm(un - ug) / np.linalg.norm(ug) < 1e-5  # 6 printed digits


def test_oracle_larger_basis_approaches_the_modified_solution(ca_sample):
    """With the factor present the basis grows (r_i = -K0^-1 ΔK r_(i-1)) and
    the CA solution approaches the exact solution of the modified model (on
    the DOFs it still connects)."""
    s = ca_sample
    K = (s["K0"] + s["dK"]).tocsr()
    live = np.flatnonzero(np.abs(K.diagonal()) > 0)
    Kl = K[live][:, live]
    uex = np.zeros(s["n"])
    uex[live] = sp.linalg.spsolve(Kl.tocsc(), s["f"][live])
    u0 = sp.linalg.spsolve(s["K0"].tocsc(), s["f"])
    errs = []
    for nb in (1, 2, 4, 6):
        u = ca_oracle.ca_reanalysis(s["K0"], s["dK"], s["f"], u0, nb)
        errs.append(np.linalg.norm(u[live] - uex[live]) / np.linalg.norm(uex[live]))
    assert errs[-1] < errs[0] and errs[2] < errs[1] < errs[0], errs
