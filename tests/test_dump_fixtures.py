"""The solver-dump format (andosim_b200.dump) and its regression fixtures, on the CPU.

tests/golden/sheets_bending.npz was written by tests/golden/make_systems.py
from the FP64 oracle (one CORRECTED Newton system of two sheets in contact
with bending). Here the fixture loads through the format's checks, matches a
fresh oracle evaluation of the same state (the oracle has not drifted), and
describes a symmetric matrix; a file with a broken row pointer is refused.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from andosim_b200 import dump

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))

import make_systems  # noqa: E402


def test_fixture_matches_the_oracle(oracle):
    fx = dump.load_system(GOLDEN / "sheets_bending.npz")
    assert fx["meta"]["workload"] == "sheets_bending"
    st = np.load(GOLDEN / "sheets_bending_state.npz")
    sc, _, _ = make_systems.sheets_bending()
    fresh = make_systems.oracle_system(oracle.f64, sc, st["x"], st["v"])
    for k in ("rowptr", "cols", "extra_rows", "extra_cols"):
        np.testing.assert_array_equal(fx[k], fresh[k], err_msg=k)
    for k in ("vals", "extra_vals", "rhs"):
        np.testing.assert_allclose(fx[k], fresh[k], rtol=1e-6, atol=1e-6 * np.abs(fresh[k]).max(), err_msg=k)
    np.testing.assert_allclose(fx["gradient"], fresh["gradient"], rtol=1e-12, atol=1e-12 * np.abs(fresh["gradient"]).max())
    assert len(fx["extra_rows"]) > 0                      # contact blocks outside the pattern
    A = dump.dense(fx)
    assert np.abs(A - A.T).max() <= 1e-6 * np.abs(A).max()
    assert np.linalg.eigvalsh(0.5 * (A + A.T)).min() > 0  # the Newton system is SPD


def test_broken_file_is_refused(tmp_path):
    fx = dump.load_system(GOLDEN / "sheets_bending.npz")
    arrays = {k: fx[k] for k in dump.KEYS}
    arrays["rowptr"] = arrays["rowptr"].copy()
    arrays["rowptr"][-1] += 1
    bad = dump.save_arrays(tmp_path / "bad.npz", arrays)
    with pytest.raises(ValueError, match="row pointer"):
        dump.load_system(bad)
    good = dump.save_arrays(tmp_path / "good.npz", {k: fx[k] for k in dump.KEYS}, frame=3)
    again = dump.load_system(good)
    assert again["meta"] == {"frame": 3}
    for k in dump.KEYS:
        np.testing.assert_array_equal(again[k], fx[k])
