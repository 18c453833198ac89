"""Learned preconditioner on the GPU against its CPU oracle
(oracle/learned_oracle.py): the SPD approximate inverse S, the training loss
and its gradient, then what training buys over block Jacobi and how the
solver falls back to it."""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import scenes
from oracle import learned_oracle as lo

pytestmark = pytest.mark.gpu


def contact_scene(n=16):
    """Two curtains 0.5 mm apart: inside the 1 mm barrier distance from the start."""
    sc = scenes.c4(n=n)
    sc.vertices[n * n:, 1] = 0.0005
    return sc


def kinematic_mask(sc):
    """CORRECTED has no kinematic vertices (pins are springs of the solve)."""
    return np.zeros(sc.num_vertices)


def evaluated(abi, sc):
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    p = abi.make_params(sc.params, semantics="corrected")
    S.apply_gravity(sc.gravity, p.dt)
    S.eval_system(p, sc.pins_at(0), sc.walls)
    d = S.last_scaled_system()
    s = lo.System(d["rowptr"], d["cols"], d["valh"].astype(np.float64), d["Lf"], S.masses, kinematic_mask(sc), 1.0 / p.dt ** 2,
                  d["xrow"], d["xcol"], d["xvalh"].astype(np.float64))
    return S, s


def perturbed_weights(abi, seed=3):
    w = abi.precond_init_weights(seed)
    return (w + 0.05 * np.random.default_rng(seed).standard_normal(w.shape)).astype(np.float32)


def test_S_matches_oracle_and_is_spd(abi):
    S, s = evaluated(abi, contact_scene(12))
    assert s.xrow is not None and len(s.xrow) > 0          # contact blocks outside the mesh pattern
    w = perturbed_weights(abi)
    S.set_precond_weights(w)
    Sg = S.precond_eval()
    net = lo.Net(lo.bf16_round(w), s)
    So = net.forward()
    assert np.abs(Sg - So).max() <= 1e-5 * np.abs(So).max()
    net.S = Sg.astype(np.float64)
    M = net.S_dense()
    assert np.abs(M - M.T).max() <= 1e-6 * np.abs(M).max()
    assert np.linalg.eigvalsh(M).min() > 0
    S.close()


def test_loss_and_gradient_match_oracle(abi):
    S, s = evaluated(abi, contact_scene(16))
    w = perturbed_weights(abi, 5)
    T = abi.Trainer(w)
    T.add_system(S, max_probes=4, tol=1e-6)
    probes, norms = T.probes(0, S.V)
    assert probes.shape[0] >= 2 and (norms > 0).all()
    Lg, gg = T.loss(0, grad=True)
    net = lo.Net(lo.bf16_round(w), s)
    net.forward()
    Lo = net.loss(probes.astype(np.float64), norms)
    go = net.backward()
    assert abs(Lg - Lo) <= 1e-5 * abs(Lo)
    assert np.linalg.norm(gg - go) <= 1e-4 * np.linalg.norm(go)
    for a, b in [(lo.W_IN, lo.LAYER0), (lo.LAYER0, lo.LAYER0 + lo.L_SIZE), (lo.DV, lo.NPARAM)]:
        assert np.linalg.norm(gg[a:b] - go[a:b]) <= 1e-4 * np.linalg.norm(go[a:b])
    # deterministic: the same loss and gradient again
    L2, g2 = T.loss(0, grad=True)
    assert L2 == Lg and (g2 == gg).all()
    T.close()
    S.close()


def run_frames(abi, sc, precond, weights, frames, params=None):
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    if weights is not None:
        S.set_precond_weights(weights)
    p = abi.make_params(dict(sc.params, **(params or {})), semantics="corrected", precond=precond)
    stats = []
    for f in range(frames):
        S.apply_gravity(sc.gravity, p.dt)
        stats.append(S.step(p, sc.pins_at(f), sc.walls))
    x, _ = S.download()
    S.close()
    return stats, x


def test_training_cuts_pcg_iterations_on_held_out_frames(abi):
    from andosim_b200 import learned

    n = 32
    w0 = abi.precond_init_weights(0)
    T = abi.Trainer(w0)
    assert learned.c4_training_set(T, seeds=[0, 1], n=n, frames=range(0, 40, 2)) >= 30
    before = learned.mean_loss(T)
    learned.train(T, steps=800, lr=2e-3)
    after = learned.mean_loss(T)
    wt = T.weights()
    T.close()
    assert after < before
    held_out = scenes.c4(seed=2, n=n)
    sj, _ = run_frames(abi, held_out, "block_jacobi", None, 40)
    sl, _ = run_frames(abi, held_out, "learned", wt, 40)
    it_j = sum(s["pcg_iters"] for s in sj) / sum(s["newton_iters"] for s in sj)
    it_l = sum(s["pcg_iters"] for s in sl) / sum(s["newton_iters"] for s in sl)
    assert sum(s["precond_fallbacks"] for s in sl) == 0
    assert it_l <= 0.8 * it_j, (it_l, it_j)


def test_learned_step_matches_block_jacobi_step(abi):
    # pcg_tol 1e-4: both solves converge above the FP32 floor of this system
    # (at 1e-6 block Jacobi itself stops short and the learned solve hands over)
    sc = scenes.c1(n=16)
    w = abi.precond_init_weights(1)
    ext = float(np.ptp(sc.vertices, axis=0).max())
    sj, xj = run_frames(abi, sc, "block_jacobi", None, 3, dict(pcg_tol=1e-4))
    sl, xl = run_frames(abi, sc, "learned", w, 3, dict(pcg_tol=1e-4))
    assert sum(s["pcg_iters"] for s in sl) < sum(s["pcg_iters"] for s in sj)
    assert sum(s["precond_fallbacks"] for s in sl) == 0
    assert np.abs(xl - xj).max() <= 1e-5 * ext


def test_learned_falls_back_to_block_jacobi(abi):
    sc = scenes.c1(n=16)
    w = abi.precond_init_weights(1)
    params = dict(pcg_max_iters=3, pcg_tol=1e-8)        # neither solve converges: the learned one hands over
    sj, xj = run_frames(abi, sc, "block_jacobi", None, 2, params)
    sl, xl = run_frames(abi, sc, "learned", w, 2, params)
    assert all(s["precond_fallbacks"] == s["newton_iters"] for s in sl)
    np.testing.assert_array_equal(xl, xj)                # the fallback is the block-Jacobi solve itself


def test_learned_needs_weights_and_corrected_semantics(abi):
    sc = scenes.c1(n=8)
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    p = abi.make_params(sc.params, semantics="corrected", precond="learned")
    with pytest.raises(abi.AbiError, match="no weights"):
        S.step(p, sc.pins, sc.walls)
    S.set_precond_weights(abi.precond_init_weights(0))
    with pytest.raises(abi.AbiError, match="CORRECTED"):
        S.step(abi.make_params(sc.params, semantics="reference", precond="learned"), sc.pins, sc.walls)
    S.close()


def test_learned_and_block_jacobi_steps_agree_on_the_curtains(abi):
    """The curtain workload (64 x 64, the shipped weights, pcg_tol 1e-4 as configured): from the same
    state, a step with the learned preconditioner and one with block Jacobi land within 1e-4 of the
    extent of each other on every one of 20 paired frames. Both solves stop on the same block-scaled
    residual test and both Newton loops on the same gradient test."""
    from andosim_b200 import learned as learned_mod

    sc = scenes.c4(n=64)
    ext = float(np.ptp(sc.vertices, axis=0).max())
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    S.set_precond_weights(learned_mod.load_weights(None))
    pl = abi.make_params(sc.params, semantics="corrected", precond="learned")
    pj = abi.make_params(sc.params, semantics="corrected", precond="block_jacobi")
    for f in range(5):
        S.apply_gravity(sc.gravity, pl.dt)
        S.step(pl, sc.pins_at(f), sc.walls)
    diffs = []
    for f in range(5, 25):
        x0, v0 = S.download()
        S.apply_gravity(sc.gravity, pj.dt)
        sj = S.step(pj, sc.pins_at(f), sc.walls)
        xj = S.download()[0]
        S.upload(x0, v0)
        S.apply_gravity(sc.gravity, pl.dt)
        sl = S.step(pl, sc.pins_at(f), sc.walls)
        xl = S.download()[0]
        assert sj["line_search_fail"] == 0 and sl["line_search_fail"] == 0
        assert sj["beta"] > 0.99 and sl["beta"] > 0.99            # both Newton loops converged
        diffs.append(float(np.abs(xl - xj).max()) / ext)
    S.close()
    assert max(diffs) <= 1e-4, diffs
