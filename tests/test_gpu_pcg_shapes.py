"""Launch shapes of the scaled PCG and block sizes of the scaled assembly:
every candidate the autotuner may pick gives the same result bits
(per-slice partials reduced in one fixed order, FMA order written out; one
thread per vertex or slot in the assembly), so tuning can never change a
trajectory."""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import learned, scenes

pytestmark = pytest.mark.gpu


def run(abi, sc, precond, index, frames=3):
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    if precond == "learned":
        S.set_precond_weights(learned.load_weights())
    S.select_pcg_shape(precond == "learned", index)
    S.select_assembly_tpb(1)  # fixed, so that tune_ms counts the PCG's timing only
    p = abi.make_params(sc.params, semantics="corrected", precond=precond)
    iters = 0
    for f in range(frames):
        S.apply_gravity(sc.gravity, p.dt)
        iters += S.step(p, sc.pins_at(f), sc.walls)["pcg_iters"]
    x, v = S.download()
    shape = S.pcg_shape(precond == "learned")
    S.close()
    return x, v, iters, shape


@pytest.mark.parametrize("precond", ["block_jacobi", "learned"])
def test_every_shape_gives_the_same_bits(abi, precond):
    sc = scenes.c4(n=48)
    x0, v0, it0, tuned = run(abi, sc, precond, -1)
    assert tuned["candidates"] >= 2 and tuned["tpb"] > 0 and tuned["tune_ms"] > 0
    assert it0 > 0
    for k in range(tuned["candidates"]):
        x, v, it, shape = run(abi, sc, precond, k)
        assert shape["tpb"] > 0 and shape["tune_ms"] == 0
        assert it == it0
        assert np.array_equal(x, x0) and np.array_equal(v, v0), f"shape {k} {shape}"


def run_asm(abi, sc, index, frames=3):
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    S.select_assembly_tpb(index)
    p = abi.make_params(sc.params, semantics="corrected")
    for f in range(frames):
        S.apply_gravity(sc.gravity, p.dt)
        S.step(p, sc.pins_at(f), sc.walls)
    x, v = S.download()
    t = S.assembly_tpb()
    S.close()
    return x, v, t


def test_every_assembly_block_size_gives_the_same_bits(abi):
    sc = scenes.c4(n=48)
    x0, v0, tuned = run_asm(abi, sc, -1)
    assert tuned["candidates"] == 3 and tuned["tpb"] in (128, 256, 512)
    for k in range(tuned["candidates"]):
        x, v, t = run_asm(abi, sc, k)
        assert t["tpb"] == (128, 256, 512)[k]
        assert np.array_equal(x, x0) and np.array_equal(v, v0)
