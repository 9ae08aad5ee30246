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


def _np_residual(n, periodic, diag, x, b):
    """||b - A x||_2 in NumPy: slot order CENTER, W, E, S, N, B, T; a
    neighbour past a non-periodic face contributes nothing."""
    X = x.reshape(n)
    ax = diag[0].reshape(n) * X
    for d in range(3):
        for side, slot in ((0, 2 * d + 1), (1, 2 * d + 2)):
            nb = np.roll(X, 1 if side == 0 else -1, axis=d)
            if not periodic[d]:
                edge = [slice(None)] * 3
                edge[d] = 0 if side == 0 else n[d] - 1
                nb[tuple(edge)] = 0.0
            ax += diag[slot].reshape(n) * nb
    return float(np.linalg.norm(b - ax.reshape(-1)))


def _call_raw(dim, n, periodic, diag, x, b, out, stream):
    nn = (C.c_int64 * 3)(*n)
    per = (C.c_int * 3)(*periodic)
    err = C.create_string_buffer(256)
    rc = D.lib().dare_residual_norm_noalloc(dim, nn, per, diag.data_ptr(), x.data_ptr(), b.data_ptr(),
                                            out.data_ptr(), stream, err, 256)
    return rc, err.value.decode()


def test_noalloc_matches_numpy_on_the_exported_matrix():
    """Independent of the solver's residual kernel: NumPy's ||b - A x|| of the
    exported CSR matrix and rhs, at a random iterate (a residual of the size
    of b, compared at 1e-12 relative) and at the converged solution (a
    residual at the rounding level, compared against the scale
    || |A| |x| + |b| ||)."""
    import scipy.sparse as sp
    import torch
    ctx = D.Context(0)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    g, f, s, vel, rep = _solved_system(ctx, 24, seed=5)
    rp, cols, vals = s.export_csr()
    A = sp.csr_matrix((vals, cols, rp), shape=(rp.size - 1, rp.size - 1))
    _, rhs = s.coefficients()
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    x_sol = s.solution()
    x_rand = np.random.default_rng(6).random(x_sol.size)
    for x, converged in ((x_sol, True), (x_rand, False)):
        s.set_initial_guess(x)
        rc, msg = _noalloc_norm(g, s, out, stream)
        assert rc == 0, msg
        torch.cuda.synchronize()
        ref = float(np.linalg.norm(rhs - A @ x))
        if converged:
            scale = float(np.linalg.norm(abs(A) @ abs(x) + abs(rhs)))
            assert abs(out.item() - ref) <= 1e-14 * scale, (out.item(), ref, scale)
        else:
            assert abs(out.item() - ref) <= 1e-12 * ref, (out.item(), ref)


@pytest.mark.parametrize("dim,n,periodic", [
    (1, (200000, 1, 1), (0, 0, 0)),     # 6250 items at 32 planes: the run length doubles to 64 (3125 items)
    (1, (200000, 1, 1), (1, 0, 0)),
    (3, (2, 256, 4096), (1, 0, 1)),     # 128 x 32 tiles of 32 x 8 cells: exactly 4096 items, the limit
])
def test_noalloc_large_item_counts(dim, n, periodic):
    import torch
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    N = int(np.prod(n))
    gen = torch.Generator(device="cuda").manual_seed(sum(n))
    diag = torch.rand(7, N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    diag[0] += 4.0
    x = torch.rand(N, dtype=torch.float64, device="cuda", generator=gen)
    b = torch.rand(N, dtype=torch.float64, device="cuda", generator=gen)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    nn = tuple(n[:dim]) + (1,) * (3 - dim)
    for k in range(2):     # two calls in a row on the shared scratch
        rc, msg = _call_raw(dim, nn, periodic, diag, x, b, out[k:], stream)
        assert rc == 0, msg
    torch.cuda.synchronize()
    ref = _np_residual(nn, periodic, diag.cpu().numpy(), x.cpu().numpy(), b.cpu().numpy())
    got = out.cpu().numpy()
    assert abs(got[0] - ref) <= 1e-12 * ref, (got[0], ref)
    assert got[1] == got[0]


def test_noalloc_rejects_oversized_plane():
    n = (C.c_int64 * 3)(4, 4096, 4096)
    per = (C.c_int * 3)(1, 1, 1)
    err = C.create_string_buffer(256)
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    rc = D.lib().dare_residual_norm_noalloc(3, n, per, dummy, dummy, dummy, dummy, None, err, 256)
    assert rc == -5 and b"4096 tiles" in err.value
