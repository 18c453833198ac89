"""CPU checks of the learned-preconditioner oracle (oracle/learned_oracle.py):
its hand-written backward against central finite differences in FP64, and the
positive definiteness of S by construction."""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import scenes
from oracle import learned_oracle as lo


def small_system(seed=0, n=5):
    """A scaled system with the static pattern of a two-sheet grid, identity
    diagonal blocks, symmetric random couplings and a few contact blocks."""
    rng = np.random.default_rng(seed)
    tris = np.concatenate([scenes.grid_triangles(n, n), scenes.grid_triangles(n, n, offset=n * n)])
    V = 2 * n * n
    adj = [set([i]) for i in range(V)]
    for t in tris:
        for a in t:
            for b in t:
                adj[a].add(int(b))
    rowptr = np.zeros(V + 1, dtype=np.int64)
    cols = []
    for i in range(V):
        c = sorted(adj[i]); cols.extend(c); rowptr[i + 1] = len(cols)
    cols = np.array(cols)
    rows = np.repeat(np.arange(V), np.diff(rowptr))
    valh = np.zeros((len(cols), 3, 3))
    key = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(rows, cols))}
    for k, (i, j) in enumerate(zip(rows, cols)):
        if i == j:
            valh[k] = np.eye(3)
        elif i < j:
            B = -0.12 * np.eye(3) + 0.03 * rng.standard_normal((3, 3))
            valh[k] = B
            valh[key[(int(j), int(i))]] = B.T
    xrow = np.array([0, 3 * n + 1, n * n + 2, n * n + 5]); xcol = np.array([n * n + 2, n * n + 5, 0, 3 * n + 1])
    xv = np.zeros((4, 3, 3))
    for a in range(2):
        B = 0.05 * rng.standard_normal((3, 3))
        xv[a] = B
        xv[a + 2] = B.T
    Lf = rng.uniform(0.5, 3.0, (V, 6))
    fixed = np.zeros(V); fixed[n - 1] = 1
    return lo.System(rowptr, cols, valh, Lf, rng.uniform(1e-5, 2e-5, V), fixed, 3600.0, xrow, xcol, xv)


def probes_for(s, P=3, seed=1):
    rng = np.random.default_rng(seed)
    A = s.dense_A()
    R = rng.standard_normal((P, 3 * s.V))
    norms = np.array([r @ np.linalg.solve(A, r) for r in R])
    return R, norms


def test_dense_system_is_spd():
    s = small_system()
    assert np.linalg.eigvalsh(s.dense_A()).min() > 0


@pytest.mark.parametrize("seed", [0, 3])
def test_S_is_symmetric_positive_definite(seed):
    s = small_system(seed)
    w = lo.init_weights(seed)
    w[lo.DE0:lo.DE0 + 2] = [2.0, -1.5]          # large edge terms: still SPD by construction
    net = lo.Net(w, s)
    net.forward()
    S = net.S_dense()
    assert np.abs(S - S.T).max() < 1e-12
    assert np.linalg.eigvalsh(S).min() > 0


def test_backward_matches_finite_differences():
    s = small_system(2)
    R, norms = probes_for(s)
    w = lo.init_weights(5).astype(np.float64)
    rng = np.random.default_rng(0)
    w += 0.05 * rng.standard_normal(w.shape)    # leave the symmetric start point

    def loss(wv):
        net = lo.Net(wv, s)
        net.forward()
        return net.loss(R, norms)

    net = lo.Net(w, s)
    net.forward()
    net.loss(R, norms)
    g = net.backward()
    groups = [(lo.W_IN, lo.B_IN), (lo.B_IN, lo.LAYER0)]
    for l in range(lo.NL):
        L = lo.LAYER0 + l * lo.L_SIZE
        groups += [(L + lo.L_U, L + lo.L_E), (L + lo.L_E, L + lo.L_C), (L + lo.L_C, L + lo.L_W), (L + lo.L_W, L + lo.L_B),
                   (L + lo.L_B, L + lo.L_SIZE)]
    groups += [(lo.DV, lo.DV0), (lo.DV0, lo.DE), (lo.DE, lo.DE0), (lo.DE0, lo.NPARAM)]
    checked = 0
    for a, b in groups:
        for idx in rng.choice(np.arange(a, b), size=min(4, b - a), replace=False):
            h = 1e-6
            wp, wm = w.copy(), w.copy()
            wp[idx] += h; wm[idx] -= h
            fd = (loss(wp) - loss(wm)) / (2 * h)
            assert abs(fd - g[idx]) <= 1e-6 + 1e-4 * abs(fd), (idx, fd, g[idx])
            checked += 1
    assert checked > 60


def test_bf16_rounding_matches_definition():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-30], dtype=np.float32)
    r = lo.bf16_round(x)
    # BF16 keeps 8 significant bits: every rounded value has its low 16 bits clear
    assert ((r.view(np.uint32) & 0xFFFF) == 0).all()
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)
