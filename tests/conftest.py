"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle extension (built on first use)."""
    from oracle.build import load

    return load()


@pytest.fixture(scope="session")
def core():
    """The product module (`ando_barrier_core`), built in-tree on first use."""
    from andosim_b200.build import build

    build()
    from andosim_b200 import ando_barrier_core

    return ando_barrier_core


@pytest.fixture(scope="session")
def abi():
    from andosim_b200.build import build

    build()
    from andosim_b200 import abi as abi_mod

    return abi_mod


def oracle_scene(mod, sc):
    """Mesh/State/SimParams of a synthetic scene in one oracle precision."""
    m = mod.Mesh()
    m.initialize(sc.vertices, sc.triangles, mod.Material(**sc.material))
    s = mod.State()
    s.initialize(m)
    p = mod.SimParams()
    for k, v in sc.params.items():
        setattr(p, k, v)
    return m, s, p


def oracle_constraints(mod, sc, frame=0):
    c = mod.Constraints()
    for i, t in sc.pins_at(frame):
        c.add_pin(int(i), t)
    for n, o, g in sc.walls:
        c.add_wall(n, o, g)
    return c
