"""The reference's own Python API tests, run against this module.

The reference tests its pybind11 surface from Python (tests/test_adaptive_timestep.py:
CFL time step, minimum edge length, velocity scan and smoothing;
tests/test_state_constraints.py: State and Constraints accessors, pins, walls;
tests/test_e2e.py: gravity fall, pins, the adaptive time step workflow, ground
approach, multi-frame stability and energy trends, all through
State.apply_gravity, which runs on the host while a state has no device
context).
Where a checkout of the reference sits beside this container's repository,
each of those test functions is imported from the reference's file with
`ando_barrier_core` resolved to this repository's module and called as is: the
drop-in must pass the reference's checks unchanged. Nothing is copied; without
the checkout (the GPU box has none) the test is skipped. test_heatmap_colors.py
tests the add-on's overlay colours and is not run.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

REFERENCE_TESTS = Path("/root/reference/tests")
SUITES = ["test_adaptive_timestep.py", "test_state_constraints.py", "test_e2e.py"]


def reference_tests(name):
    path = REFERENCE_TESTS / name
    if not path.exists():
        return []
    spec = importlib.util.spec_from_file_location(f"reference_{path.stem}", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return [(name, fn_name, getattr(mod, fn_name)) for fn_name in sorted(dir(mod)) if fn_name.startswith("test_")]


@pytest.fixture(scope="module")
def as_reference_module(core):
    """Make `import ando_barrier_core` inside the reference's files give this module."""
    saved = sys.modules.get("ando_barrier_core")
    sys.modules["ando_barrier_core"] = core
    yield core
    if saved is None:
        sys.modules.pop("ando_barrier_core", None)
    else:
        sys.modules["ando_barrier_core"] = saved


@pytest.mark.skipif(not REFERENCE_TESTS.exists(), reason="no reference checkout beside the repository")
@pytest.mark.parametrize("suite", SUITES)
def test_reference_python_suite_passes(as_reference_module, suite):
    cases = reference_tests(suite)
    assert cases, f"{suite}: no test functions found"
    for name, fn_name, fn in cases:
        fn()            # the reference's assertions, unchanged
