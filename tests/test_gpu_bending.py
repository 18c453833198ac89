"""Quadratic bending on the GPU (CORRECTED semantics, bending_stiffness > 0)
against the FP64 oracle.

The reference declares Material::bending_stiffness (types.h:56) and never
reads it; the oracle's term (tests/test_oracle_bending.py pins it by central
differences, affine invariance and the discrete-shell fold energy) is the
parity target. With bending the BSR pattern gains the pair of vertices
opposite each interior edge, the constant elastic blocks gain the bending
Hessian and the elastic gradient gains its force.
"""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import scenes
from test_gpu_corrected import corrected_parity, free_run
from test_gpu_learned import run_frames
from test_gpu_parity import extent, max_rel_error

pytestmark = pytest.mark.gpu

KB = 1e-3


def bent(sc, kb=KB):
    sc.material = dict(sc.material, bending_stiffness=kb)
    return sc


def test_bending_system_matches_oracle(oracle, abi):
    sc = bent(scenes.c1(n=16))
    rng = np.random.default_rng(7)
    x = sc.vertices + rng.normal(scale=2e-3, size=sc.vertices.shape)
    v = rng.normal(scale=0.2, size=x.shape)
    corrected_parity(oracle, abi, sc, x, v)
    # the pattern: self blocks, the face pairs and the two opposite vertices of every interior edge
    n = 16
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    S.upload(sc.vertices, np.zeros_like(sc.vertices), sc.vertices, None)
    V, nnzb = S.system_size()
    S.close()
    E = 3 * (n - 1) ** 2 + 2 * (n - 1)
    interior = E - 4 * (n - 1)
    assert nnzb == V + 2 * E + 2 * interior


def test_bending_system_near_rest(oracle, abi):
    """Close to the flat rest sheet the bending force is small against the
    coordinates (the sum over a stencil cancels); it still matches."""
    sc = bent(scenes.c1(n=12))
    x = sc.vertices.copy()
    x[:, 2] += 1e-5 * np.sin(7.0 * x[:, 0]) * np.cos(5.0 * x[:, 1])
    corrected_parity(oracle, abi, sc, x, np.zeros_like(x))


def test_bending_free_run_matches_fp64(oracle, core):
    """The hanging cloth (two corners pinned) with bending stiffness: 8 frames
    of the GPU step stay within 1e-4 of the extent of the FP64 oracle run,
    while bending moves the cloth by far more than that."""
    to, tg, sg = free_run(oracle, core, bent(scenes.c1(n=20)), 8, pcg_tol=1e-5)
    ext = extent(scenes.c1(n=20))
    assert max_rel_error(to, tg, ext) <= 1e-4
    assert all(s["line_search_fail"] == 0 for s in sg)
    t0, _, _ = free_run(oracle, core, scenes.c1(n=20), 8, pcg_tol=1e-5)
    assert np.abs(to[-1] - t0[-1]).max() / ext > 1e-3


def test_bending_learned_step_matches_block_jacobi(abi):
    """The learned preconditioner over the pattern with the bending pairs (the
    network sees them as graph edges): same steps as block Jacobi."""
    sc = bent(scenes.c1(n=16))
    w = abi.precond_init_weights(1)
    ext = float(np.ptp(sc.vertices, axis=0).max())
    sj, xj = run_frames(abi, sc, "block_jacobi", None, 3, dict(pcg_tol=1e-4))
    sl, xl = run_frames(abi, sc, "learned", w, 3, dict(pcg_tol=1e-4))
    assert all(s["pcg_iters"] > 0 for s in sl)
    assert np.abs(xl - xj).max() <= 1e-4 * ext
