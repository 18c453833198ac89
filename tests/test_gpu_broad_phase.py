"""Device LBVH broad phase against the reference's overlap predicate.

The reference's own BVH keeps no primitive in leaves of 2..4 (collision.cpp:81-86),
so its literal query is empty for every mesh with >= 2 triangles; the query it
intends is the brute-force test of its predicate (collision.h:37-41, point box
+-1e-4, incident-face and shared-vertex exclusions). The LBVH must return
exactly that set, bit for bit after sorting, on FP32 boxes (Real=float) --
optionally inflated by a pad.
"""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import scenes

pytestmark = pytest.mark.gpu


def oracle_pairs(oracle, sc, x, pad):
    O = oracle.f32
    m = O.Mesh()
    m.initialize(sc.vertices, sc.triangles, O.Material(**sc.material))
    vt, ee = O.broad_phase(m, x, "intended", pad)
    return np.array(sorted(vt), dtype=np.int64).reshape(-1, 2), np.array(sorted(ee), dtype=np.int64).reshape(-1, 2)


def gpu_pairs(abi, sc, x, pad):
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    S.upload(x, np.zeros_like(x), sc.vertices, None)
    vt = S.broad_phase(0, pad).astype(np.int64)
    ee = S.broad_phase(1, pad).astype(np.int64)
    S.close()
    return vt, ee


def stacked(n=40, layers=3, gap=0.004, seed=1):
    sc = scenes.c2(seed=seed, n=n, sheets=layers)
    sc.vertices[:, 2] = 0.5 + (sc.vertices[:, 2] - 0.5) * 0.3
    for k in range(layers):
        sc.vertices[k * n * n:(k + 1) * n * n, 2] += gap * k - 0.005 * k
    return sc


@pytest.mark.parametrize("pad", [0.0, 1e-3, 5e-3])
def test_lbvh_matches_bruteforce_stack(oracle, abi, pad):
    sc = stacked()
    x = sc.vertices.astype(np.float32).astype(np.float64)
    vo, eo = oracle_pairs(oracle, sc, x, pad)
    vg, eg = gpu_pairs(abi, sc, x, pad)
    assert len(vo) > 0 and len(eo) > 0
    np.testing.assert_array_equal(vg, vo)
    np.testing.assert_array_equal(eg, eo)


def test_lbvh_interpenetrating_sheets(oracle, abi):
    """Two crossing sheets: vertices within 0.1 mm of the other sheet's triangles."""
    n = 30
    a = scenes.grid_plane(n, 1.0)
    b = scenes.grid_plane(n, 1.0)
    b[:, 2] = (b[:, 0] - 0.5) * 0.2          # tilted sheet crossing the flat one along x = 0.5
    v = np.concatenate([a, b])
    t = np.concatenate([scenes.grid_triangles(n, n), scenes.grid_triangles(n, n, offset=n * n)])
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3)
    sc = scenes.Scene("crossing", v, t, mat, scenes.cloth_params(), [], [])
    x = v.astype(np.float32).astype(np.float64)
    vo, eo = oracle_pairs(oracle, sc, x, 0.0)
    vg, eg = gpu_pairs(abi, sc, x, 0.0)
    assert len(vo) > 0
    np.testing.assert_array_equal(vg, vo)
    np.testing.assert_array_equal(eg, eo)


def test_lbvh_flat_grid_and_single_triangle(oracle, abi):
    """Degenerate extents (all z equal: identical Morton z bits) and the one-triangle mesh."""
    sc = scenes.c1(n=24)
    x = sc.vertices.astype(np.float32).astype(np.float64)
    for pad in (0.0, 0.05):
        vo, eo = oracle_pairs(oracle, sc, x, pad)
        vg, eg = gpu_pairs(abi, sc, x, pad)
        np.testing.assert_array_equal(vg, vo)
        np.testing.assert_array_equal(eg, eo)
    v = np.array([[0.0, 0.0, 0.0], [0.2, 0.0, 0.0], [0.0, 0.2, 0.0], [0.05, 0.05, 0.00005], [0.5, 0.5, 0.5]])
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3)
    one = scenes.Scene("tri1", v, np.array([[0, 1, 2]], dtype=np.int32), mat, scenes.cloth_params(), [], [])
    vo, eo = oracle_pairs(oracle, one, v, 0.0)
    vg, eg = gpu_pairs(abi, one, v, 0.0)
    np.testing.assert_array_equal(vg, vo)
    assert vg.tolist() == [[3, 0]]
    assert len(eg) == 0
