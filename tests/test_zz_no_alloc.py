"""ando_pcg_solve_noalloc against the solve inside ando_step.

The allocation-free entry point runs the same PCG over a caller-owned BSR
system with its reduction partials in a static device array. Here it re-solves
the last Newton system of a CORRECTED step (taken with ando_last_system) and
must return that step's PCG solution, on two calls in a row (the second call
reuses the scratch the first one left behind). This file is collected last so
that it also runs after every other GPU test in the same process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from andosim_b200 import scenes
from test_gpu_parity import bsr_to_dense

pytestmark = pytest.mark.gpu


def last_newton_system(abi, tol):
    sc = scenes.c1(n=16)
    p = abi.make_params(dict(sc.params, pcg_tol=tol), semantics="corrected")
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    S.keep_system()                    # the step also keeps the unscaled system it solves
    S.upload(sc.vertices, np.zeros_like(sc.vertices), sc.vertices, None)
    S.apply_gravity(sc.gravity, p.dt)
    st = S.step(p, sc.pins, sc.walls)
    rowptr, cols, vals, rhs, sol = S.last_system()
    extra = S.last_contact_blocks()
    S.close()
    assert st["newton_iters"] >= 1 and st["pcg_iters"] > 5
    assert len(extra[0]) == 0          # the whole system is in the BSR pattern
    return p, rowptr, cols, vals, rhs, sol


def solve_noalloc(abi, dev, p, V, work_floats=None, bufs=None):
    import torch

    rowptr, cols, vals, rhs = dev
    if bufs is None:
        bufs = (torch.empty(3 * V, dtype=torch.float32, device="cuda:0"), torch.empty(24 * V, dtype=torch.float32, device="cuda:0"))
    x, work = bufs
    x.zero_()
    work.fill_(float("nan"))                        # contents must not matter
    it, status, rel = C.c_int32(-1), C.c_int32(-1), C.c_double(-1.0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = abi.lib().ando_pcg_solve_noalloc(
        0, stream, V, C.c_void_p(rowptr.data_ptr()), C.c_void_p(cols.data_ptr()), C.c_void_p(vals.data_ptr()),
        C.c_void_p(rhs.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(work.data_ptr()),
        24 * V if work_floats is None else work_floats, float(p.pcg_tol), int(p.pcg_max_iters),
        C.byref(it), C.byref(status), C.byref(rel))
    return rc, x.cpu().numpy().astype(np.float64), it.value, status.value, rel.value


def test_noalloc_pcg_matches_step_solve(abi):
    import torch

    p, rowptr, cols, vals, rhs, sol = last_newton_system(abi, 1e-5)
    V = len(rowptr) - 1
    dev = (torch.from_numpy(np.ascontiguousarray(rowptr, dtype=np.int32)).cuda(),
           torch.from_numpy(np.ascontiguousarray(cols, dtype=np.int32)).cuda(),
           torch.from_numpy(np.ascontiguousarray(vals, dtype=np.float32).ravel()).cuda(),
           torch.from_numpy(np.ascontiguousarray(rhs, dtype=np.float32).ravel()).cuda())
    sol = np.asarray(sol, dtype=np.float64).ravel()
    scale = np.abs(sol).max()
    assert scale > 0
    A = bsr_to_dense(rowptr, cols, np.asarray(vals, dtype=np.float64).reshape(-1, 3, 3), V)
    b = np.asarray(rhs, dtype=np.float64).ravel()
    exact = np.linalg.solve(A, b)
    # caller-owned output and work buffers, allocated once up front
    bufs = (torch.empty(3 * V, dtype=torch.float32, device="cuda:0"), torch.empty(24 * V, dtype=torch.float32, device="cuda:0"))
    rc, *_ = solve_noalloc(abi, dev, p, V, bufs=bufs)   # warm-up: the first call on a device may load the module
    assert rc == abi.ANDO_OK, abi.lib().ando_last_error().decode()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    results = []
    for _ in range(2):
        rc, x, iters, status, rel = solve_noalloc(abi, dev, p, V, bufs=bufs)
        assert rc == abi.ANDO_OK, abi.lib().ando_last_error().decode()
        assert status == 0 and 0 < iters <= p.pcg_max_iters and rel < p.pcg_tol
        # The step's solve iterates the same block-Jacobi PCG but stops on the
        # block-scaled residual, this entry point on the reference's unscaled one
        # (pcg_solver.cpp:8-75), so at one tolerance the two stop at slightly
        # different iterates: both answers lie within 1e-3 of their size of each
        # other and of the exact solution.
        assert np.abs(x - sol).max() <= 1e-3 * scale, np.abs(x - sol).max() / scale
        assert np.abs(x - exact).max() <= 1e-3 * scale, np.abs(x - exact).max() / scale
        # and it does solve the system: true residual at the FP32 level of the tolerance
        assert np.abs(b - A @ x).max() <= 10 * p.pcg_tol * np.abs(b).max()
        results.append(x)
    np.testing.assert_array_equal(results[0], results[1])
    # the calls took no device memory: a cudaMalloc (or a cudaFree) would move the free byte count
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free_before


def test_noalloc_pcg_rejects_small_work_buffer(abi):
    import torch

    V = 8
    dev = (torch.zeros(V + 1, dtype=torch.int32, device="cuda:0"), torch.zeros(1, dtype=torch.int32, device="cuda:0"),
           torch.zeros(9, dtype=torch.float32, device="cuda:0"), torch.zeros(3 * V, dtype=torch.float32, device="cuda:0"))
    p = abi.make_params(scenes.cloth_params())
    rc, *_ = solve_noalloc(abi, dev, p, V, work_floats=24 * V - 1)
    assert rc == abi.ANDO_ERR_CAPACITY
    assert "work buffer" in abi.lib().ando_last_error().decode()
