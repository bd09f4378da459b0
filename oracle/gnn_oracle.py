"""CPU restatement of the learned coarse-correction stage (numpy, float64).

TEST INFRASTRUCTURE ONLY: the checker of the GPU forward/backward kernels in
openfea_b200/csrc/learned.cu.  Same weight layout, same stage, same loss.

Level data: na aggregates, the 27-slot neighbour table nbr, the Jacobi-scaled
Galerkin blocks Ehat[I, s] (6 x 6, unit diagonal) and per-aggregate features
feat[I] (NFEAT values).  B = the inverse of Ehat's diagonal blocks.

Network (static per matrix, input the features):
  h0 = relu(W0 feat + b0)                                           (64 wide)
  4 x: a_I = [h_I, (sum_J h_J, sum_J dx h_J, sum_J dy h_J, sum_J dz h_J) / deg_I],
       h = relu(W a + b)                                            (320 -> 64)
  Y = Wd h + bd,  s = exp(Y / 2)                                    (6 per aggregate)
with J over the existing ones (nbr >= 0) of the 26 neighbour slots s != 13 of
I, deg_I their count (offsets dx = s//9-1, dy = (s//3)%3-1, dz = s%3-1).

Stage (linear and symmetric in the scaled coarse residual x):
  y = s * M (s * x),   M = sum_k c_k (B Ehat)^(k-1) B   (k = 1..TERMS)
a polynomial in B Ehat with trainable global coefficients c (in the weight
vector) between per-aggregate, per-mode scalings s set by the network.

The dense products may be evaluated on bfloat16-rounded operands (bf16=True),
as the GPU's tensor-core layers do.

Loss over a batch of inputs x_b (the energy; its minimiser is Ehat^-1 x):
  L = sum_b (1/2 y_b . Ehat y_b - y_b . x_b) / (6 na)
The backward pass here is checked against central finite differences
(tests/test_gnn_oracle.py) before it is used to check the GPU.
"""
from __future__ import annotations

import numpy as np

F, NFEAT, TERMS, L = 64, 8, 3, 4
OUT = 6
A = 5 * F


def layout():
    off, o = {}, 0
    off["W0"] = (o, (F, NFEAT)); o += F * NFEAT
    off["b0"] = (o, (F,)); o += F
    for l in range(L):
        off[f"W{l + 1}"] = (o, (F, A)); o += F * A
        off[f"b{l + 1}"] = (o, (F,)); o += F
    off["Wd"] = (o, (OUT, F)); o += OUT * F
    off["bd"] = (o, (OUT,)); o += OUT
    off["c0"] = (o, (TERMS,)); o += TERMS
    return off, o


OFF, TOTAL = layout()
SLOTS = np.arange(27)
DX, DY, DZ = SLOTS // 9 - 1, (SLOTS // 3) % 3 - 1, SLOTS % 3 - 1


def bf16(x):
    """Round to bfloat16 (nearest even) through float32, as the GPU's
    tensor-core layers round their FP32 operands; returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    return {k: w[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in OFF.items()}


class GNNOracle:
    """bf16=True rounds both operands of every dense-layer product to
    bfloat16 (the GPU runs those products on the tensor cores with BF16
    operands and FP32 accumulation); everything else stays FP64."""

    def __init__(self, nbr, Ehat, feat, bf16=False):
        self.r = globals()["bf16"] if bf16 else (lambda v: v)
        self.nbr = np.asarray(nbr).reshape(-1, 27)
        self.na = self.nbr.shape[0]
        self.E = np.asarray(Ehat, dtype=np.float64).reshape(self.na, 27, 6, 6)
        self.feat = np.asarray(feat, dtype=np.float64).reshape(self.na, NFEAT)
        self.Binv = np.linalg.inv(self.E[:, 13])
        deg = (self.nbr[:, np.arange(27) != 13] >= 0).sum(axis=1)
        self.deg = deg
        self.invdeg = np.where(deg > 0, 1.0 / np.maximum(deg, 1), 0.0)

    # ---- graph operators
    def agg(self, H):
        out = np.zeros((self.na, A))
        out[:, :F] = H
        for s in range(27):
            if s == 13:
                continue
            J = self.nbr[:, s]
            ok = J >= 0
            hj = np.zeros_like(H)
            hj[ok] = H[J[ok]]
            out[:, F:2 * F] += hj
            out[:, 2 * F:3 * F] += DX[s] * hj
            out[:, 3 * F:4 * F] += DY[s] * hj
            out[:, 4 * F:5 * F] += DZ[s] * hj
        out[:, F:] *= self.invdeg[:, None]
        return out

    def agg_bwd(self, dA):
        dH = dA[:, :F].copy()
        dA = dA.copy()
        dA[:, F:] *= self.invdeg[:, None]
        for s in range(27):
            if s == 13:
                continue
            J = self.nbr[:, s]
            ok = np.nonzero(J >= 0)[0]
            contrib = (dA[ok, F:2 * F] + DX[s] * dA[ok, 2 * F:3 * F] + DY[s] * dA[ok, 3 * F:4 * F]
                       + DZ[s] * dA[ok, 4 * F:5 * F])
            np.add.at(dH, J[ok], contrib)
        return dH

    def apply_E(self, Y):
        """Ehat applied to a batch of coarse vectors (B, na, 6)."""
        out = np.zeros_like(Y)
        for s in range(27):
            J = self.nbr[:, s]
            ok = J >= 0
            yj = np.zeros_like(Y)
            yj[:, ok] = Y[:, J[ok]]
            out += np.einsum("ikl,bil->bik", self.E[:, s], yj)
        return out

    def apply_B(self, x):
        return np.einsum("ikl,bil->bik", self.Binv, x)

    def basis(self, u):
        """v_k = (B Ehat)^(k-1) B u, k = 1..TERMS, for a batch u (B, na, 6)."""
        v = [self.apply_B(u)]
        for k in range(1, TERMS):
            v.append(self.apply_B(self.apply_E(v[-1])))
        return v

    def apply_M(self, u, c):
        return sum(ck * vk for ck, vk in zip(c, self.basis(u)))

    # ---- network
    def forward(self, w):
        p = unpack(np.asarray(w, dtype=np.float64))
        cache = {}
        r = self.r
        Z = r(self.feat) @ r(p["W0"]).T + p["b0"]
        cache["Z0"] = Z
        H = np.maximum(Z, 0)
        for l in range(L):
            Aa = self.agg(H)
            cache[f"A{l}"] = Aa
            Z = r(Aa) @ r(p[f"W{l + 1}"]).T + p[f"b{l + 1}"]
            cache[f"Z{l + 1}"] = Z
            H = np.maximum(Z, 0)
        cache["H"] = H
        Y = r(H) @ r(p["Wd"]).T + p["bd"]
        return Y, cache, p

    def scales(self, w):
        Y, _, _ = self.forward(w)
        return np.exp(0.5 * Y)

    def stage(self, w, x):
        Y, _, p = self.forward(w)
        sc = np.exp(0.5 * Y)[None]
        return sc * self.apply_M(sc * x, p["c0"])

    def loss(self, w, x):
        y = self.stage(w, x)
        return float(np.sum(0.5 * y * self.apply_E(y) - y * x) / (6 * self.na))

    def grad(self, w, x):
        Y, c, p = self.forward(w)
        sc = np.exp(0.5 * Y)[None]
        V = self.basis(sc * x)
        wv = sum(ck * vk for ck, vk in zip(p["c0"], V))
        y = sc * wv
        ey = self.apply_E(y)
        loss = float(np.sum(0.5 * y * ey - y * x) / (6 * self.na))
        d = (ey - x) / (6 * self.na)
        # y = s * M (s * x):  dL/ds = d * M(s x) + x * M(s d)  (M symmetric)
        ds = np.sum(d * wv + x * self.apply_M(sc * d, p["c0"]), axis=0)
        g = {"c0": np.array([np.sum(sc * d * vk) for vk in V])}
        r = self.r
        dY = 0.5 * ds * sc[0]
        g["Wd"] = r(dY).T @ r(c["H"])
        g["bd"] = dY.sum(axis=0)
        dH = r(dY) @ r(p["Wd"])
        dZ = dH * (c[f"Z{L}"] > 0)
        for l in reversed(range(L)):
            Aa = c[f"A{l}"]
            g[f"W{l + 1}"] = r(dZ).T @ r(Aa)
            g[f"b{l + 1}"] = dZ.sum(axis=0)
            dA = r(dZ) @ r(p[f"W{l + 1}"])
            dH = self.agg_bwd(dA)
            Zp = c[f"Z{l}"] if l > 0 else c["Z0"]
            dZ = dH * (Zp > 0)
        g["W0"] = r(dZ).T @ r(self.feat)
        g["b0"] = dZ.sum(axis=0)
        flat = np.zeros(TOTAL)
        for k, (o, s) in OFF.items():
            flat[o:o + int(np.prod(s))] = g[k].ravel()
        return loss, flat


def he_weights(seed=0, out_gain=0.1, c0=(1.0, 0.0, 0.0)):
    """Weights drawn like the library's initialiser: N(0, 2/fan_in), the
    output layer scaled by out_gain, biases small, c0 given."""
    rng = np.random.default_rng(seed)
    w = np.zeros(TOTAL)
    for k, (o, s) in OFF.items():
        n = int(np.prod(s))
        if k == "c0":
            w[o:o + n] = c0
        elif k.startswith("W"):
            gain = out_gain if k == "Wd" else np.sqrt(2.0)
            w[o:o + n] = rng.normal(0, gain / np.sqrt(s[1]), n)
        else:
            w[o:o + n] = rng.normal(0, 0.05, n)
    return w


def random_level(nc=(3, 2, 2), seed=0):
    """A small cell grid with its neighbour table, an SPD-like Jacobi-scaled
    block operator and features, for checking the oracle on its own."""
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
                E[I, s] = np.eye(6) + 0.1 * (blk + blk.T)
            else:
                E[I, s] = blk
                E[J, 26 - s] = blk.T
    feat = rng.normal(0, 0.3, (na, NFEAT))
    return nbr, E, feat
