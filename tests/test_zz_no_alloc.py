"""The allocation-free residual norm entry point (dare_residual_norm_noalloc).

It serves host codes that cannot allocate device memory in the middle of a
run (their allocator owns the device, or a cudaMalloc would stall their other
streams).  This file is collected last so that, if it fails, a run that stops
at the first failure has already run every other test.  It must pass alone in
a fresh process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

import dare_b200 as D
from dare_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12   # the same kernel arithmetic; only the summation grouping may differ


def _solved_system(ctx, n, seed):
    case = W.tvd_convection_diffusion(n=n, seed=seed)
    g = D.Grid(ctx, case["n"], case["size"], 2, case["periodic"])
    f = D.Field(g, 2)
    phi = np.ascontiguousarray(case["phi0"].reshape(-1))
    f.upload(phi, 0)
    f.upload(phi, 1)
    s = D.MatrixSystem(g)
    vel = [D.DeviceArray(a) for a in case["face_vel"]]
    s.build(f, D.Assembly(dt=case["dt"], D=case["D"], face_vel=tuple(vel), limiter="VANLEER"))
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 500, "tol_relative": 1}).solve(s)
    assert rep["converged"]
    return g, f, s, vel, rep


def _noalloc_norm(g, s, out, stream):
    n = (C.c_int64 * 3)(*g.n)
    per = (C.c_int * 3)(*[int(g.info.periodic[d]) for d in range(3)])
    err = C.create_string_buffer(256)
    rc = D.lib().dare_residual_norm_noalloc(g.dim, n, per, s.device_ptr(0), s.device_ptr(8), s.device_ptr(7),
                                            out.data_ptr(), stream, err, 256)
    return rc, err.value.decode()


def test_noalloc_residual_matches_solver_report():
    import torch
    ctx = D.Context(0)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    # two systems, two calls in a row: the shared scratch must not carry state over
    sys_a = _solved_system(ctx, 20, seed=3)
    sys_b = _solved_system(ctx, 16, seed=4)
    for k, (g, f, s, vel, rep) in enumerate((sys_a, sys_b)):
        rc, msg = _noalloc_norm(g, s, out[k:], stream)
        assert rc == 0, msg
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for k, (g, f, s, vel, rep) in enumerate((sys_a, sys_b)):
        ref = rep["true_res_abs"]
        assert ref > 0.0
        assert abs(got[k] - ref) <= REL_TOL * ref, (k, got[k], ref)
    # a second pass over the same inputs gives the same numbers
    for k, (g, f, s, vel, rep) in enumerate((sys_a, sys_b)):
        rc, msg = _noalloc_norm(g, s, out[k:], stream)
        assert rc == 0, msg
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), got)


def test_noalloc_rejects_oversized_plane():
    n = (C.c_int64 * 3)(4, 4096, 4096)
    per = (C.c_int * 3)(1, 1, 1)
    err = C.create_string_buffer(256)
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    rc = D.lib().dare_residual_norm_noalloc(3, n, per, dummy, dummy, dummy, dummy, None, err, 256)
    assert rc == -5 and b"4096 tiles" in err.value
