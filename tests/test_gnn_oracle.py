"""The CPU restatement of the learned stage (oracle/gnn_oracle.py): its
backward pass against central finite differences, and the stage's algebra.  It is then the
reference the GPU gradients are checked against (tests/test_gpu_learned.py)."""
import numpy as np

from oracle.gnn_oracle import TOTAL, GNNOracle, he_weights, random_level


def test_gnn_oracle_gradient_matches_finite_differences():
    nbr, E, feat = random_level((3, 2, 2), seed=1)
    net = GNNOracle(nbr, E, feat)
    rng = np.random.default_rng(2)
    w = he_weights(2, out_gain=1.0, c0=(0.8, -0.3, 0.1))
    x = rng.normal(0, 1, (2, net.na, 6))
    loss, g = net.grad(w, x)
    assert np.isfinite(loss)
    idx = rng.choice(TOTAL, 80, replace=False)
    scale = np.abs(g).max()
    h = 1e-5
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (net.loss(wp, x) - net.loss(wm, x)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * scale, (i, fd, g[i])


def test_gnn_oracle_energy_minimum_is_galerkin_solution():
    """The loss is minimised by y = Ehat^-1 x (gradient zero there)."""
    nbr, E, feat = random_level((2, 2, 2), seed=3)
    net = GNNOracle(nbr, E, feat)
    na = net.na
    M = np.zeros((6 * na, 6 * na))
    for I in range(na):
        for s in range(27):
            J = nbr[I, s]
            if J >= 0:
                M[6 * I:6 * I + 6, 6 * J:6 * J + 6] = E[I, s]
    x = np.random.default_rng(4).normal(size=(1, na, 6))
    y = np.linalg.solve(M, x.reshape(-1)).reshape(1, na, 6)
    grad_y = (net.apply_E(y) - x) / (6 * na)
    assert np.abs(grad_y).max() < 1e-12


def test_gnn_oracle_stage_is_linear_and_symmetric():
    """y = s * M(s * x) with M a polynomial in B Ehat times B: symmetric for any
    scalings s the network sets."""
    nbr, E, feat = random_level((2, 2, 2), seed=5)
    net = GNNOracle(nbr, E, feat)
    w = he_weights(6, out_gain=1.0, c0=(1.5, -0.4, 0.05))
    na = net.na
    basis = np.eye(6 * na).reshape(6 * na, na, 6)
    S = net.stage(w, basis).reshape(6 * na, 6 * na)
    assert np.abs(S - S.T).max() < 1e-10 * np.abs(S).max()
    assert np.abs(net.scales(w) - 1.0).max() > 1e-2  # the scalings are not trivial here
