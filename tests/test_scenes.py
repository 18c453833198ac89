"""The seeded synthetic workloads (CPU): shapes, seeds and the C4 drive.

The bench's C4 workload is defined by `scenes.c4`; its pin schedule is
checked here against the drive written out pin by pin (top rows pinned,
±0.3 m along x at 0.5 Hz in opposite phase, smoothstep ramp over 0.5 s)."""
from __future__ import annotations

import math

import numpy as np

from andosim_b200 import scenes


def test_c4_shapes_and_seed():
    n = 16
    a, b, c = scenes.c4(0, n), scenes.c4(0, n), scenes.c4(1, n)
    assert a.num_vertices == 2 * n * n
    assert a.num_triangles == 2 * 2 * (n - 1) * (n - 1)
    assert np.array_equal(a.vertices, b.vertices)
    assert not np.array_equal(a.vertices, c.vertices)
    assert len(a.pins) == 2 * n


def test_c4_pin_schedule_matches_the_drive():
    n = 16
    sc = scenes.c4(3, n)
    base = {i: sc.vertices[i].copy() for i, _ in sc.pins}
    half = n * n
    dt = 1.0 / 60.0
    for frame in (0, 5, 29, 30, 77):
        t = (frame + 1) * dt
        r = min(1.0, t / 0.5)
        ramp = r * r * (3.0 - 2.0 * r)
        got = sc.pins_at(frame)
        assert [i for i, _ in got] == [i for i, _ in sc.pins]
        for i, tgt in got:
            want = base[i].copy()
            sgn = 1.0 if i < half else -1.0
            want[0] += sgn * 0.3 * ramp * math.sin(2 * math.pi * 0.5 * t)
            assert np.array_equal(tgt, want), (frame, i)
