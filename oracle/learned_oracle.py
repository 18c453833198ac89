"""CPU oracle of the learned preconditioner (test infrastructure only).

FP64 numpy restatement of what andosim_b200/csrc/learned.cu computes: the
features of a block-scaled Newton system A^ = L^-1 A L^-T, the message-passing
network, the SPD block-sparse approximate inverse S it parameterises, the
training loss on solver-dumped probe vectors, and the loss gradient with
respect to the weights (hand-written backward, checked here against finite
differences). The preconditioner has no counterpart in the reference, whose
only preconditioner is block Jacobi (pcg_solver.cpp:77-114); this file is the
checker for the CUDA kernels, never called by the product path.

Layout of the flat parameter vector (dense matrices row-major [out][in]):
W_in (64x8), b_in, then per layer U (64x64), E (64x10), c (64), W (64x128),
b (64), then dv (64), dv0, De (2x138), de (2).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

FN, FE, H, NL = 8, 10, 64, 3
DE_IN = 2 * H + FE
W_IN = 0
B_IN = W_IN + H * FN
LAYER0 = B_IN + H
L_U = 0
L_E = L_U + H * H
L_C = L_E + H * FE
L_W = L_C + H
L_B = L_W + H * 2 * H
L_SIZE = L_B + H
DV = LAYER0 + NL * L_SIZE
DV0 = DV + H
DE = DV0 + 1
DE0 = DE + 2 * DE_IN
NPARAM = DE0 + 2
DELTA_MIN = 1e-4


def bf16_round(w: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), as __float2bfloat16_rn."""
    b = np.asarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


@dataclass
class System:
    """A scaled system on the static pattern (+ merged contact blocks)."""
    rowptr: np.ndarray      # V+1
    cols: np.ndarray        # nnzb
    valh: np.ndarray        # (nnzb, 3, 3)
    Lf: np.ndarray          # (V, 6) packed lower-triangular L
    mass: np.ndarray        # V
    fixed: np.ndarray       # V (0/1)
    dt2inv: float
    xrow: Optional[np.ndarray] = None   # merged contact blocks outside the pattern
    xcol: Optional[np.ndarray] = None
    xvalh: Optional[np.ndarray] = None  # (nx, 3, 3)

    @property
    def V(self) -> int:
        return len(self.rowptr) - 1

    def rows(self) -> np.ndarray:
        return np.repeat(np.arange(self.V), np.diff(self.rowptr))

    def slot_T(self) -> np.ndarray:
        r = self.rows()
        key = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(r, self.cols))}
        return np.array([key[(int(b), int(a))] for a, b in zip(r, self.cols)], dtype=np.int64)

    def dense_A(self) -> np.ndarray:
        V = self.V
        A = np.zeros((3 * V, 3 * V))
        for k, (i, j) in enumerate(zip(self.rows(), self.cols)):
            A[3 * i:3 * i + 3, 3 * j:3 * j + 3] += self.valh[k]
        if self.xrow is not None:
            for k, (i, j) in enumerate(zip(self.xrow, self.xcol)):
                A[3 * i:3 * i + 3, 3 * j:3 * j + 3] += self.xvalh[k]
        return A


def features(s: System):
    V = s.V
    rows, cols = s.rows(), s.cols
    A = s.valh.astype(np.float64)
    nf = np.sqrt((A * A).sum(axis=(1, 2)))
    Ef = np.concatenate([A.reshape(-1, 9), nf[:, None]], axis=1)
    off = cols != rows
    stat = np.zeros(V); np.add.at(stat, rows[off], nf[off])
    mx = np.zeros(V); np.maximum.at(mx, rows[off], nf[off])
    deg = np.zeros(V); np.add.at(deg, rows[off], 1.0)
    cont = np.zeros(V); ncont = np.zeros(V)
    if s.xrow is not None and len(s.xrow):
        xn = np.sqrt((s.xvalh.astype(np.float64) ** 2).sum(axis=(1, 2)))
        np.add.at(cont, s.xrow, xn); np.add.at(ncont, s.xrow, 1.0)
    tr = (s.Lf.astype(np.float64) ** 2).sum(axis=1)
    mref = 3.0 * s.mass * s.dt2inv
    fx = s.fixed.astype(bool)
    ok = (~fx) & (mref > 0) & (tr > 0)
    stiff = np.zeros(V)
    stiff[ok] = np.log10(tr[ok] / mref[ok]) * 0.25
    X = np.stack([np.ones(V), np.log1p(ncont), stat, cont, stiff, deg * 0.125, fx.astype(np.float64), mx], axis=1)
    return X, Ef


def _softplus(z):
    return np.where(z > 20.0, z, np.log1p(np.exp(np.minimum(z, 20.0))))


def _sigmoid(z):
    return 1.0 / (1.0 + np.exp(-z))


class Net:
    """Forward, loss and backward of the preconditioner network on one system."""

    def __init__(self, w: np.ndarray, s: System):
        self.w = np.asarray(w, dtype=np.float64)
        self.s = s
        self.rows = s.rows()
        self.cols = np.asarray(s.cols)
        self.off = self.cols != self.rows
        self.up = self.cols > self.rows
        self.sT = s.slot_T()
        self.deg = np.zeros(s.V)
        np.add.at(self.deg, self.rows[self.off], 1.0)

    def layer(self, l):
        L = LAYER0 + l * L_SIZE
        w = self.w
        return (w[L + L_U:L + L_E].reshape(H, H), w[L + L_E:L + L_C].reshape(H, FE), w[L + L_C:L + L_W],
                w[L + L_W:L + L_B].reshape(H, 2 * H), w[L + L_B:L + L_SIZE])

    def forward(self):
        s, w = self.s, self.w
        X, Ef = features(s)
        self.X, self.Ef = X, Ef
        Win, bin_ = w[W_IN:B_IN].reshape(H, FN), w[B_IN:LAYER0]
        self.q0 = X @ Win.T + bin_
        h = np.maximum(self.q0, 0.0)
        self.hs, self.us, self.ms, self.qs, self.ts = [h], [], [], [], []
        ro, co = self.rows[self.off], self.cols[self.off]
        inv = np.where(self.deg > 0, 1.0 / np.maximum(self.deg, 1.0), 0.0)
        for l in range(NL):
            U, E, c, W, b = self.layer(l)
            u = h @ U.T
            t = u[co] + Ef[self.off] @ E.T + c
            m = np.zeros((s.V, H)); np.add.at(m, ro, np.maximum(t, 0.0))
            m *= inv[:, None]
            q = np.concatenate([h, m], axis=1) @ W.T + b
            self.us.append(u); self.ms.append(m); self.qs.append(q); self.ts.append(t)
            h = h + np.maximum(q, 0.0)
            self.hs.append(h)
        dv, dv0 = w[DV:DV0], w[DV0]
        De, de = w[DE:DE0].reshape(2, DE_IN), w[DE0:DE0 + 2]
        self.zv = h @ dv + dv0
        ku = np.nonzero(self.up)[0]
        inp = np.concatenate([h[self.rows[ku]], h[self.cols[ku]], Ef[ku]], axis=1)
        self.ku, self.dec_in = ku, inp
        ab = np.zeros((len(self.cols), 2))
        ab[ku] = inp @ De.T + de
        self.ab = ab
        self.S = self.build_S()
        return self.S

    def coef(self, k):
        """(a, b) of the undirected edge of slot k."""
        kk = k if self.cols[k] > self.rows[k] else self.sT[k]
        return self.ab[kk]

    def build_S(self):
        s = self.s
        A = s.valh.astype(np.float64)
        S = np.zeros_like(A)
        delta = _softplus(self.zv) + DELTA_MIN
        D = delta[:, None, None] * np.eye(3)[None]
        for k in range(len(self.cols)):
            i, j = self.rows[k], self.cols[k]
            if i == j:
                continue
            a, b = self.coef(k)
            S[k] = a * b * A[k]
            if j > i:
                D[i] += a * a * np.eye(3)
            else:
                D[i] += b * b * (A[k] @ A[k].T)
        for k in range(len(self.cols)):
            if self.rows[k] == self.cols[k]:
                S[k] = D[self.rows[k]]
        return S

    def S_dense(self):
        V = self.s.V
        M = np.zeros((3 * V, 3 * V))
        for k, (i, j) in enumerate(zip(self.rows, self.cols)):
            M[3 * i:3 * i + 3, 3 * j:3 * j + 3] = self.S[k]
        return M

    def loss(self, probes: np.ndarray, pnorm: np.ndarray):
        A = self.s.dense_A()
        Sd = self.S_dense()
        self.A_dense, self.S_dense_ = A, Sd
        P = len(pnorm)
        self.Y = probes @ Sd.T
        self.Wv = self.Y @ A.T
        T = (self.Y * self.Wv).sum(axis=1) - 2.0 * (probes * self.Y).sum(axis=1)
        self.probes, self.pnorm = probes, pnorm
        return float(np.mean(1.0 + T / pnorm))

    def backward(self) -> np.ndarray:
        s, w = self.s, self.w
        V, P = s.V, len(self.pnorm)
        g = np.zeros(NPARAM)
        GY = 2.0 * (self.Wv - self.probes) / (self.pnorm[:, None] * P)     # (P, 3V)
        R = self.probes
        gy = GY.reshape(P, V, 3)
        r = R.reshape(P, V, 3)
        A = s.valh.astype(np.float64)
        gbi = (gy * r).sum(axis=(0, 2))
        dzv = gbi * _sigmoid(self.zv)
        dab = np.zeros_like(self.ab)
        for k in self.ku:
            i, j = self.rows[k], self.cols[k]
            Ak = A[k]
            dc = sum(gy[p, i] @ Ak @ r[p, j] + r[p, i] @ Ak @ gy[p, j] for p in range(P))
            gbb = sum(gy[p, j] @ (Ak.T @ Ak) @ r[p, j] for p in range(P))
            a, b = self.ab[k]
            dab[k] = (dc * b + 2 * a * gbi[i], dc * a + 2 * b * gbb)
        h = self.hs[-1]
        dv = w[DV:DV0]
        De = w[DE:DE0].reshape(2, DE_IN)
        g[DV:DV0] = dzv @ h
        g[DV0] = dzv.sum()
        d = dab[self.ku]
        g[DE:DE0] = (d.T @ self.dec_in).ravel()
        g[DE0:DE0 + 2] = d.sum(axis=0)
        dh = dzv[:, None] * dv[None, :]
        np.add.at(dh, self.rows[self.ku], d @ De[:, :H])
        np.add.at(dh, self.cols[self.ku], d @ De[:, H:2 * H])
        ro, co = self.rows[self.off], self.cols[self.off]
        Eoff = self.Ef[self.off]
        inv = np.where(self.deg > 0, 1.0 / np.maximum(self.deg, 1.0), 0.0)
        for l in range(NL - 1, -1, -1):
            U, E, c, W, b = self.layer(l)
            L = LAYER0 + l * L_SIZE
            hp, m, q, t = self.hs[l], self.ms[l], self.qs[l], self.ts[l]
            dq = dh * (q > 0)
            g[L + L_W:L + L_B] = (dq.T @ np.concatenate([hp, m], axis=1)).ravel()
            g[L + L_B:L + L_SIZE] = dq.sum(axis=0)
            dhm = dq @ W
            dm = dhm[:, H:]
            gt = (dm[ro] * inv[ro][:, None]) * (t > 0)
            du = np.zeros((V, H)); np.add.at(du, co, gt)
            g[L + L_E:L + L_C] = (gt.T @ Eoff).ravel()
            g[L + L_C:L + L_W] = gt.sum(axis=0)
            g[L + L_U:L + L_E] = (du.T @ hp).ravel()
            dh = dh + dhm[:, :H] + du @ U
        dq0 = dh * (self.q0 > 0)
        g[W_IN:B_IN] = (dq0.T @ self.X).ravel()
        g[B_IN:LAYER0] = dq0.sum(axis=0)
        return g


def init_weights(seed: int = 0) -> np.ndarray:
    """Initial weights near the Neumann form S = 0.25 (2 I - A^) (any seed)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NPARAM, dtype=np.float32)
    w[W_IN:B_IN] = rng.uniform(-1, 1, H * FN) * np.sqrt(6.0 / FN)
    for l in range(NL):
        L = LAYER0 + l * L_SIZE
        w[L + L_U:L + L_E] = rng.uniform(-1, 1, H * H) * np.sqrt(6.0 / H)
        w[L + L_E:L + L_C] = rng.uniform(-1, 1, H * FE) * np.sqrt(6.0 / FE)
        w[L + L_W:L + L_B] = rng.uniform(-1, 1, H * 2 * H) * 0.5 * np.sqrt(6.0 / (2 * H))
    w[DV:DV0] = rng.uniform(-1, 1, H) * 0.01
    w[DE:DE0] = rng.uniform(-1, 1, 2 * DE_IN) * 0.01
    w[DV0] = -1.2587
    w[DE0], w[DE0 + 1] = 0.5, -0.5
    return w
