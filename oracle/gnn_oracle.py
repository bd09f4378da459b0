"""CPU restatement of the learned coarse-correction network (numpy, float64).

TEST INFRASTRUCTURE ONLY: the checker of the GPU forward/backward kernels in
openfea_b200/csrc/learned.cu.  Same weight layout, same energy loss:

  x_I (6) + feature f_I  ->  h0 = relu(W0 [x, f] + b0)
  4 x: a_I = [h_I, sum_J h_J, sum_J dx h_J, sum_J dy h_J, sum_J dz h_J],  h = relu(W a + b)
  y = Wd h + bd
  L = sum_b sum_I (1/2 y_I . (Ehat y)_I - y_I . x_I) / (6 na)

with J over the 26 neighbour slots s != 13 of I (offsets dx = s//9-1,
dy = (s//3)%3-1, dz = s%3-1) and (Ehat y)_I = sum over all 27 slots of
Ehat[I, s] y_J.  The backward pass here is checked against central finite
differences (tests/test_gnn_oracle.py) before it is used to check the GPU.
"""
from __future__ import annotations

import numpy as np

F, IN, OUT, L = 64, 7, 6, 4
A = 5 * F


def layout():
    off, o = {}, 0
    off["W0"] = (o, (F, IN)); o += F * IN
    off["b0"] = (o, (F,)); o += F
    for l in range(L):
        off[f"W{l + 1}"] = (o, (F, A)); o += F * A
        off[f"b{l + 1}"] = (o, (F,)); o += F
    off["Wd"] = (o, (OUT, F)); o += OUT * F
    off["bd"] = (o, (OUT,)); o += OUT
    return off, o


OFF, TOTAL = layout()
SLOTS = np.arange(27)
DX, DY, DZ = SLOTS // 9 - 1, (SLOTS // 3) % 3 - 1, SLOTS % 3 - 1


def unpack(w):
    return {k: w[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in OFF.items()}


class GNNOracle:
    def __init__(self, nbr, Ehat, feat):
        self.nbr = np.asarray(nbr).reshape(-1, 27)
        self.na = self.nbr.shape[0]
        self.E = np.asarray(Ehat, dtype=np.float64).reshape(self.na, 27, 6, 6)
        self.feat = np.asarray(feat, dtype=np.float64).reshape(self.na)

    def agg(self, H):
        B = H.shape[0]
        out = np.zeros((B, self.na, A))
        out[:, :, :F] = H
        for s in range(27):
            if s == 13:
                continue
            J = self.nbr[:, s]
            ok = J >= 0
            hj = np.zeros_like(H)
            hj[:, ok] = H[:, J[ok]]
            out[:, :, F:2 * F] += hj
            out[:, :, 2 * F:3 * F] += DX[s] * hj
            out[:, :, 3 * F:4 * F] += DY[s] * hj
            out[:, :, 4 * F:5 * F] += DZ[s] * hj
        return out

    def agg_bwd(self, dA):
        dH = dA[:, :, :F].copy()
        for s in range(27):
            if s == 13:
                continue
            J = self.nbr[:, s]
            ok = np.nonzero(J >= 0)[0]
            # a_I gathered h_J: dh_J += dA_I (sum part) + offset * dA_I (dir parts)
            contrib = (dA[:, ok, F:2 * F] + DX[s] * dA[:, ok, 2 * F:3 * F] + DY[s] * dA[:, ok, 3 * F:4 * F]
                       + DZ[s] * dA[:, ok, 4 * F:5 * F])
            np.add.at(dH, (slice(None), J[ok]), contrib)
        return dH

    def apply_E(self, Y):
        out = np.zeros_like(Y)
        for s in range(27):
            J = self.nbr[:, s]
            ok = J >= 0
            yj = np.zeros_like(Y)
            yj[:, ok] = Y[:, J[ok]]
            out += np.einsum("ikl,bil->bik", self.E[:, s], yj)
        return out

    def forward(self, w, x):
        p = unpack(np.asarray(w, dtype=np.float64))
        B = x.shape[0]
        X = np.concatenate([x, np.broadcast_to(self.feat[None, :, None], (B, self.na, 1))], axis=2)
        cache = {"X": X}
        Z = X @ p["W0"].T + p["b0"]
        cache["Z0"] = Z
        H = np.maximum(Z, 0)
        for l in range(L):
            Aa = self.agg(H)
            cache[f"A{l}"] = Aa
            Z = Aa @ p[f"W{l + 1}"].T + p[f"b{l + 1}"]
            cache[f"Z{l + 1}"] = Z
            H = np.maximum(Z, 0)
        cache["H"] = H
        Y = H @ p["Wd"].T + p["bd"]
        return Y, cache, p

    def loss(self, w, x):
        Y, _, _ = self.forward(w, x)
        EY = self.apply_E(Y)
        return float(np.sum(0.5 * Y * EY - Y * x) / (6 * self.na))

    def grad(self, w, x):
        Y, c, p = self.forward(w, x)
        EY = self.apply_E(Y)
        loss = float(np.sum(0.5 * Y * EY - Y * x) / (6 * self.na))
        dY = (EY - x) / (6 * self.na)
        g = {}
        g["Wd"] = np.einsum("bio,bif->of", dY, c["H"])
        g["bd"] = dY.sum(axis=(0, 1))
        dH = dY @ p["Wd"]
        dZ = dH * (c[f"Z{L}"] > 0)
        for l in reversed(range(L)):
            Aa = c[f"A{l}"]
            g[f"W{l + 1}"] = np.einsum("bio,bia->oa", dZ, Aa)
            g[f"b{l + 1}"] = dZ.sum(axis=(0, 1))
            dA = dZ @ p[f"W{l + 1}"]
            dH = self.agg_bwd(dA)
            Zp = c[f"Z{l}"] if l > 0 else c["Z0"]
            dZ = dH * (Zp > 0)
        g["W0"] = np.einsum("bio,bik->ok", dZ, c["X"])
        g["b0"] = dZ.sum(axis=(0, 1))
        flat = np.zeros(TOTAL)
        for k, (o, s) in OFF.items():
            flat[o:o + int(np.prod(s))] = g[k].ravel()
        return loss, flat


def he_weights(seed=0, out_gain=0.1):
    """Weights drawn like the library's initialiser: N(0, 2/fan_in), the
    output layer scaled by out_gain, biases small."""
    rng = np.random.default_rng(seed)
    w = np.zeros(TOTAL)
    for k, (o, s) in OFF.items():
        n = int(np.prod(s))
        if k.startswith("W"):
            gain = out_gain if k == "Wd" else np.sqrt(2.0)
            w[o:o + n] = rng.normal(0, gain / np.sqrt(s[1]), n)
        else:
            w[o:o + n] = rng.normal(0, 0.05, n)
    return w


def random_level(nc=(3, 2, 2), seed=0):
    """A small cell grid with its neighbour table, an SPD-like Jacobi-scaled
    block operator and a feature, for checking the oracle on its own."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = nc
    na = nx * ny * nz
    nbr = -np.ones((na, 27), dtype=np.int64)
    E = np.zeros((na, 27, 6, 6))
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                I = (i * ny + j) * nz + k
                for s in range(27):
                    x, y, z = i + DX[s], j + DY[s], k + DZ[s]
                    if 0 <= x < nx and 0 <= y < ny and 0 <= z < nz:
                        nbr[I, s] = (x * ny + y) * nz + z
    for I in range(na):
        for s in range(27):
            J = nbr[I, s]
            if J < 0 or J < I:
                continue
            blk = rng.normal(0, 0.05, (6, 6))
            if s == 13:
                blk = np.eye(6) + 0.5 * (blk + blk.T)
                E[I, s] = blk
            else:
                E[I, s] = blk
                E[J, 26 - s] = blk.T
    feat = rng.normal(0, 0.3, na)
    return nbr, E, feat
