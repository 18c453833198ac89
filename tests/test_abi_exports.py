"""The C-ABI library loads without a GPU and exports every entry point that
include/ando_gpu.h declares (no compute call is made)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "ando_gpu.h").read_text()
    return sorted(set(re.findall(r"ANDO_API\s+[\w\s\*]+?\b(ando_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 30
    for must in ("ando_step", "ando_ctx_create", "ando_pcg_solve_noalloc", "ando_trainer_step", "ando_precond_eval"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from andosim_b200.build import build, gpu_lib

    build()
    lib = ctypes.CDLL(str(gpu_lib()))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_entry_points_without_gpu():
    from andosim_b200 import abi

    assert abi.lib().ando_abi_version() == 1
    n = abi.precond_num_params()
    w = abi.precond_init_weights(7)
    assert w.shape == (n,) and abs(w[-2] - 0.5) < 1e-7 and abs(w[-1] + 0.5) < 1e-7
    assert (abi.precond_init_weights(7) == w).all()
