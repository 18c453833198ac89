"""Batched scenes (ando_step_batch): uneven cloths of the batched workload
stepped concurrently must end exactly where stepping each alone ends."""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import scenes

pytestmark = pytest.mark.gpu


def make(abi, sc):
    return abi.Scene(sc.vertices, sc.triangles, sc.material)


@pytest.mark.parametrize("semantics", ["corrected", "reference"])
def test_batch_equals_scene_by_scene(abi, semantics):
    scs = scenes.c3(seed=1, scenes=6)
    params = [abi.make_params(sc.params, semantics=semantics) for sc in scs]
    alone = [make(abi, sc) for sc in scs]
    batch = [make(abi, sc) for sc in scs]
    for f in range(3):
        for S, sc, p in zip(alone, scs, params):
            S.apply_gravity(sc.gravity, p.dt)
            S.step(p, sc.pins_at(f), sc.walls)
        for S, sc, p in zip(batch, scs, params):
            S.apply_gravity(sc.gravity, p.dt)
        stats = abi.step_batch(batch, params, [sc.pins_at(f) for sc in scs], [sc.walls for sc in scs], threads=4)
        assert len(stats) == len(scs) and all(st["newton_iters"] >= 0 for st in stats)
    for a, b in zip(alone, batch):
        xa, va = a.download()
        xb, vb = b.download()
        assert np.array_equal(xa, xb) and np.array_equal(va, vb)
        a.close(); b.close()


def test_batch_rejects_a_repeated_context(abi):
    sc = scenes.c3(seed=2, scenes=1)[0]
    S = make(abi, sc)
    p = abi.make_params(sc.params, semantics="corrected")
    with pytest.raises(abi.AbiError):
        abi.step_batch([S, S], [p, p], [sc.pins_at(0)] * 2, [sc.walls] * 2)
    S.close()
