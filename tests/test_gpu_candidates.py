"""Broad-phase candidate buffers that start too small: the contact pass grows
its buffer and runs again, and a time-of-impact pass that overflows leaves
the positions untouched (pin advance and line search check a device flag)
until the host has grown the buffer and redone it. The trajectory must be the
one a large enough buffer gives, bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import scenes

pytestmark = pytest.mark.gpu


def run(abi, sc, capacity, frames=4, top_cap=None):
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    if top_cap is not None:
        S.set_refit_top_capacity(top_cap)
    p = abi.make_params(sc.params, semantics="corrected")
    stats = []
    for f in range(frames):
        if capacity:
            S.set_pair_capacity(capacity)  # every frame starts over-full again
        S.apply_gravity(sc.gravity, p.dt)
        stats.append(S.step(p, sc.pins_at(f), sc.walls))
    x, v = S.download()
    S.close()
    return x, v, stats


def test_small_candidate_buffers_give_the_same_trajectory(abi):
    sc = scenes.c4(n=48)
    x0, v0, s0 = run(abi, sc, None)
    x1, v1, s1 = run(abi, sc, 16)
    assert sum(st["newton_iters"] for st in s0) > 0
    assert [st["pcg_iters"] for st in s1] == [st["pcg_iters"] for st in s0]
    assert np.array_equal(x1, x0) and np.array_equal(v1, v0)


def test_pair_capacity_must_be_positive(abi):
    sc = scenes.c4(n=16)
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    with pytest.raises(abi.AbiError):
        S.set_pair_capacity(0)
    S.close()


def test_global_counter_refit_gives_the_same_trajectory(abi):
    """A top capacity of 0 sends every node above the refit's cut through the
    global acquire/release arrival counters instead of the one-CTA shared
    memory climb; the boxes, hence the trajectory, are the same bits."""
    sc = scenes.c4(n=48)  # 8,836 triangles and 13,442 edges: nodes above the 1,024-leaf cut
    x0, v0, s0 = run(abi, sc, None)
    x1, v1, s1 = run(abi, sc, None, top_cap=0)
    x2, v2, s2 = run(abi, sc, None, top_cap=3)
    assert [st["pcg_iters"] for st in s1] == [st["pcg_iters"] for st in s0]
    assert np.array_equal(x1, x0) and np.array_equal(v1, v0)
    assert np.array_equal(x2, x0) and np.array_equal(v2, v0)


def test_refit_top_capacity_is_checked(abi):
    sc = scenes.c4(n=16)
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    for bad in (-2, 4097):
        with pytest.raises(abi.AbiError):
            S.set_refit_top_capacity(bad)
    S.set_refit_top_capacity(-1)
    S.close()
