"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Bars: cell numbering, ghost fill and the exported CSR pattern bit-exact;
assembled FP64 coefficients within 1e-13 relative on 3-D grids (the staged
3-D kernel contracts to FMA and evaluates the limiters in division-light
forms) and bit-exact on 1-D / 2-D grids (that kernel keeps the reference's
operation order without FMA contraction); solutions within 1e-9 relative L2
at the same tolerance.
"""
import numpy as np
import pytest

import dare_b200 as D
from dare_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import (assert_coef_close, coupled_components_diag, diag_to_csr, interior, oracle_assembly,
                           oracle_grid, oracle_timeloop, profile_functor_diag, rel_l2, interleave_csr)

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-9   # relative L2, solutions at the same residual tolerance


@pytest.fixture(scope="module")
def ctx():
    c = D.Context(0)
    yield c
    c.synchronize()


def _gpu_case(ctx, case):
    dim = len(case["n"])
    g = D.Grid(ctx, case["n"], case.get("size"), 2, case.get("periodic"))
    f = D.Field(g, 2)
    phi = np.ascontiguousarray(np.asarray(case["phi0"], dtype=np.float64).reshape(-1))
    f.upload(phi, 0)
    f.upload(np.ascontiguousarray(np.asarray(case.get("phi_old", phi), dtype=np.float64).reshape(-1)), 1)
    s = D.MatrixSystem(g)
    for face, (kind, val) in case.get("bc", {}).items():
        s.set_bc(int(face), kind, val)
    keep = []
    face_vel = None
    if case.get("face_vel") is not None:
        keep = [D.DeviceArray(np.asarray(a)) for a in case["face_vel"]]
        face_vel = tuple(keep)
    face_D = None
    if case.get("face_D") is not None:
        fd = [D.DeviceArray(np.asarray(a)) for a in case["face_D"]]
        keep += fd
        face_D = tuple(fd)
    asm = D.Assembly(dt=case.get("dt", 0.0), D=case.get("D"), face_D=face_D, vel=case.get("vel"),
                     face_vel=face_vel, limiter=case.get("limiter", "VANLEER"),
                     scheme=case.get("scheme", "EULER_BACKWARD"))
    return g, f, s, asm, keep, dim


def _random_case(kind, seed=0):
    rng = np.random.default_rng(seed)
    if kind == "diffusion3d":
        n = (12, 10, 9)
        phi = rng.random(tuple(x + 4 for x in n))
        return {"n": n, "size": (1.0, 2.0, 0.5), "periodic": (0, 0, 0), "dt": 0.01, "D": 1e-3, "phi0": phi,
                "phi_old": rng.random(phi.shape),
                "bc": {1: (1, 1.0), 2: (1, 0.0), 3: (2, 0.0), 4: (1, 0.25), 5: (2, 0.0), 6: (2, 0.0)}}
    if kind.startswith("tvd3d"):
        lim = kind.split("-")[1]
        c = W.tvd_convection_diffusion(n=16, seed=seed)
        c["limiter"] = lim
        return c
    if kind == "facediff3d":
        c = W.heterogeneous(n=16, seed=seed)
        Dc = c["cell_D"]
        faces = []
        for d in range(3):
            lo = np.roll(Dc, 1, axis=d)
            f = (lo + Dc) * 0.5
            first = [slice(None)] * 3
            first[d] = slice(0, 1)
            faces.append(np.concatenate([f, f[tuple(first)]], axis=d))
        c["face_D"] = faces
        return c
    if kind.startswith("tiles3d"):
        # several 31 x 8 (k, j) assembly tiles and plane runs; quantised phi
        # (equal neighbours: r = +-inf and 0/0 in the limiters), face
        # velocities with exact zeros, heterogeneous face D, mixed boundaries
        n = (23, 19, 70) if kind == "tiles3d" else (9, 17, 65)
        periodic = (1, 0, 0) if kind == "tiles3d" else (1, 1, 1)
        phi = rng.integers(0, 4, size=tuple(x + 4 for x in n)) / 4.0
        fv, fd = [], []
        for d in range(3):
            shape = tuple(x + (1 if e == d else 0) for e, x in enumerate(n))
            v = rng.normal(size=shape)
            v[rng.random(shape) < 0.05] = 0.0
            fv.append(v)
            fd.append(10.0 ** rng.uniform(-4, -2, size=shape))
        c = {"n": n, "size": (1.0, 0.7, 2.0), "periodic": periodic, "dt": 0.03, "D": None, "phi0": phi,
             "phi_old": rng.random(phi.shape), "face_vel": fv, "face_D": fd,
             "limiter": "VANLEER" if kind == "tiles3d" else "VANALBADA"}
        if kind == "tiles3d":
            c["bc"] = {3: (1, 0.5), 4: (2, 0.0), 5: (2, 0.0), 6: (1, -1.0)}
        return c
    if kind == "range3d":
        # phi spanning twelve decades with random signs: the limiter's
        # divisions see operands of every magnitude
        c = _random_case("tiles3d-periodic", seed)
        shape = c["phi0"].shape
        c["phi0"] = rng.choice([-1.0, 1.0], size=shape) * 10.0 ** rng.uniform(-6, 6, size=shape)
        c["limiter"] = "VANLEER"
        return c
    if kind.startswith("scheme3d"):
        # the Divergence time schemes on the 3-D kernel (several tiles)
        c = _random_case("tiles3d", seed)
        c["scheme"] = kind.split("-")[1]
        return c
    if kind.startswith("scheme2d"):
        c = _random_case("tvd2d", seed)
        c["scheme"] = kind.split("-")[1]
        return c
    if kind == "mixed3d":
        n = (5, 7, 9)
        phi = rng.random(tuple(x + 4 for x in n)) - 0.5
        return {"n": n, "size": (1.0, 1.0, 1.0), "periodic": (1, 0, 0), "dt": 0.05, "D": 2e-3,
                "vel": (0.3, -0.2, 0.1), "limiter": "MINMOD", "phi0": phi,
                "bc": {3: (1, 1.0), 4: (2, 0.0), 5: (1, -1.0), 6: (1, 0.5)}}
    if kind == "tvd2d":
        n = (11, 13)
        phi = rng.random((15, 17, 1))
        return {"n": n, "size": (1.0, 2.0), "periodic": (1, 1), "dt": 0.02, "D": 1e-3, "vel": (-0.4, 0.7),
                "limiter": "VANALBADA", "phi0": phi}
    if kind == "tvd1d":
        phi = rng.random((14, 1, 1))
        return {"n": (10,), "size": (1.0,), "periodic": (0,), "dt": 0.1, "D": 0.5, "vel": (-1.0,),
                "limiter": "VANLEER", "phi0": phi, "bc": {1: (2, 0.0), 2: (1, 2.0)}}
    raise KeyError(kind)


ASM_CASES = ["diffusion3d", "tvd3d-VANLEER", "tvd3d-CDS", "tvd3d-UPWIND", "tvd3d-MINMOD", "tvd3d-VANALBADA",
             "facediff3d", "mixed3d", "tiles3d", "tiles3d-periodic", "range3d", "tvd2d", "tvd1d",
             "scheme3d-EULER_FORWARD", "scheme3d-CRANK_NICHOLSON", "scheme3d-ADAMS_BASHFORTH",
             "scheme3d-ADAMS_MOULTON", "scheme2d-CRANK_NICHOLSON", "scheme2d-ADAMS_MOULTON"]


@pytest.mark.parametrize("kind", ASM_CASES)
def test_assembly_matches_oracle(ctx, kind):
    case = _random_case(kind)
    if kind == "facediff3d":
        case["D"] = None
    g, f, s, asm, keep, dim = _gpu_case(ctx, case)
    s.build(f, asm)
    diag, rhs = s.coefficients()
    x0 = s.solution()
    og = oracle_grid(case)
    desc = oracle_assembly(og, case, face_D=case.get("face_D"))
    phi = np.ascontiguousarray(np.asarray(case["phi0"], dtype=np.float64).reshape(-1))
    old = np.ascontiguousarray(np.asarray(case.get("phi_old", case["phi0"]), dtype=np.float64).reshape(-1))
    odiag, orhs, omask = O.assemble(desc, phi, old)
    same = assert_coef_close if dim == 3 else np.testing.assert_array_equal
    same(diag, odiag)
    same(rhs, orhs)
    np.testing.assert_array_equal(x0, O.field_to_vector(og, phi))
    # CSR export: identical pattern, values as the coefficients
    rp, cols, vals = s.export_csr()
    orp, ocols, ovals = O.export_csr(og, odiag, omask)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(cols, ocols)
    same(vals, ovals)


@pytest.mark.parametrize("dims,periodic", [((9, 8, 7), (1, 1, 1)), ((9, 8, 7), (0, 1, 0)), ((6, 5), (1, 0)),
                                           ((10,), (1,)), ((10,), (0,))])
def test_halo_exchange_bit_exact(ctx, dims, periodic):
    g = D.Grid(ctx, dims, None, 2, periodic)
    og = O.make_grid(len(dims), dims, None, 2, periodic)
    phi = np.random.default_rng(1).random(g.num_cells_ghosted)
    f = D.Field(g, 2)
    f.upload(phi)
    f.exchange_halo()
    got = f.download()
    ref = phi.copy()
    O.exchange_halo(og, ref)
    np.testing.assert_array_equal(got, ref)
    # CopyDataVectorsToOldTimeStep
    f.copy_to_old()
    np.testing.assert_array_equal(f.download(1), ref)


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("precond", ["NONE", "JACOBI"])
def test_bicgstab2_linear_profile(ctx, dim, precond):
    """test_integration_Cartesian_Trilinos.cpp SolveScalar(X): BiCGStab2,
    tolerance 1e-14, solution = linear profile within 1e-8."""
    n = [20 + d for d in range(dim)]
    diag, rhs, x0 = profile_functor_diag(dim, n)
    g = D.Grid(ctx, n, [1.0 + d for d in range(dim)], 2, None)
    s = D.MatrixSystem(g)
    s.set_coefficients(diag, rhs, x0)
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-14, "Maximum Iterations": 5000}, precond=precond)
    rep = solver.solve(s)
    assert rep["converged"], rep
    x = s.solution()
    nn = n + [1] * (3 - dim)
    i = np.repeat(np.arange(nn[0]), nn[1] * nn[2])
    assert np.max(np.abs(x - (i + 0.5) / nn[0])) < 1e-8
    rp, cols, vals = diag_to_csr(dim, n, diag)
    ox, info = O.bicgstab2(rp, cols, vals, rhs, x0, 1e-14, 5000,
                           O.PREC_JACOBI if precond == "JACOBI" else O.PREC_NONE)
    assert rel_l2(x, ox) < SOL_TOL
    assert abs(rep["iters"] - info["iters"]) <= max(2, info["iters"] // 10)


def test_bicgstab2_coupled_components(ctx):
    """MatrixSystem/test/test_TrilinosSolver.cpp:98-205 (BumbleBee BICGSTAB2,
    tolerance 1e-12), as a 23 x 4 structured grid."""
    diag, rhs, x0 = coupled_components_diag()
    g = D.Grid(ctx, (23, 4), None, 2, None)
    s = D.MatrixSystem(g)
    s.set_coefficients(diag, rhs, x0)
    for precond in ("NONE", "JACOBI"):
        s.set_initial_guess(x0)
        rep = D.BiCGStab2({"Convergence Tolerance": 1e-12, "Maximum Iterations": 5000}, precond=precond).solve(s)
        assert rep["converged"], rep
        x = s.solution()
        node = np.repeat(np.arange(23), 4)
        assert np.max(np.abs(x - (node + 0.5) / 23)) < 1e-8


def _gpu_timeloop(ctx, case, steps, precond="JACOBI"):
    g, f, s, asm, keep, dim = _gpu_case(ctx, case)
    solver = D.BiCGStab2({"Convergence Tolerance": case.get("rel_tol", 1e-10), "Maximum Iterations": 5000,
                          "tol_relative": 1}, precond=precond)
    hist, iters = [], []
    for _ in range(steps):
        rep = D.timestep(s, f, asm, solver)
        assert rep["converged"], rep
        hist.append(f.download(0))
        iters.append(rep["iters"])
    return hist, iters, g


@pytest.mark.parametrize("kind", ["gaussian", "tvd", "tvd-CRANK_NICHOLSON", "tvd-ADAMS_MOULTON"])
def test_timeloop_matches_oracle(ctx, kind):
    if kind == "gaussian":
        case = W.gaussian_diffusion(n=20, steps=3)
    else:
        case = W.tvd_convection_diffusion(n=24, steps=3)
        if "-" in kind:
            case["scheme"] = kind.split("-")[1]
    hist, iters, g = _gpu_timeloop(ctx, case, 3)
    ohist, oiters = oracle_timeloop(case, 3)
    for a, b in zip(hist, ohist):
        assert rel_l2(interior(a, g.ghosted_shape), interior(b, g.ghosted_shape)) < SOL_TOL
        # the periodic halo is refilled identically
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * np.abs(b).max())
    for a, b in zip(iters, oiters):
        assert abs(a - b) <= 2


def test_analytical_slab_diffusion(ctx):
    """Companion of the Gaussian diffusion workload against
    AnalyticalSolutions/Diffusion.h (phi = 0 at t = 0, Dirichlet 1 at x = 1,
    zero gradient at x = 0; tau = D t / L^2).  The reference asserts no
    threshold; the bar here is first-order-in-time implicit Euler."""
    n, D_, dt, steps = 32, 1.0, 1e-3, 20
    case = {"n": (n, 3, 3), "size": (1.0, 1.0, 1.0), "periodic": (0, 0, 0), "dt": dt, "D": D_,
            "phi0": np.zeros((n + 4, 7, 7)), "rel_tol": 1e-12,
            "bc": {1: (2, 0.0), 2: (1, 1.0), 3: (2, 0.0), 4: (2, 0.0), 5: (2, 0.0), 6: (2, 0.0)}}
    hist, _, g = _gpu_timeloop(ctx, case, steps)
    phi = interior(hist[-1], g.ghosted_shape)[:, 1, 1]
    zeta = (np.arange(n) + 0.5) / n
    exact = np.array([O.diffusion_n0d1(D_ * dt * steps, z) for z in zeta])
    err = np.abs(phi - exact)
    assert err.mean() < 5e-3 and err.max() < 2e-2, (err.mean(), err.max())


def test_breakdown_and_limits_report_status(ctx):
    n = (6, 5, 4)
    g = D.Grid(ctx, n, None, 2, (1, 1, 1))
    s = D.MatrixSystem(g)
    N = g.num_cells
    diag = np.zeros((7, N))
    diag[0] = 7.0
    diag[1:] = -1.0
    rhs = np.random.default_rng(3).random(N)
    # iteration budget: max_it = 1 stops with k = 2 > 1 (BiCGStab2.inl:322-326)
    s.set_coefficients(diag, rhs, np.zeros(N))
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-300, "Maximum Iterations": 1}).solve(s)
    assert rep["status_name"] == "max_iterations" and not rep["converged"] and rep["iters"] == 2
    # zero residual at the start: converged with k = 0
    s.set_coefficients(diag, np.zeros(N), np.zeros(N))
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-12, "Maximum Iterations": 10}).solve(s)
    assert rep["converged"] and rep["iters"] == 0
    # NaN injected into the rhs: reported, not looped on
    bad = rhs.copy()
    bad[5] = np.nan
    s.set_coefficients(diag, bad, np.zeros(N))
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-12, "Maximum Iterations": 50}).solve(s)
    assert rep["status_name"] == "nan" and not rep["converged"]
    # a zero matrix without preconditioning breaks down at step (7): gamma = 0
    s.set_coefficients(np.zeros((7, N)), rhs, np.zeros(N))
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-12, "Maximum Iterations": 50}, precond="NONE").solve(s)
    assert rep["status_name"] == "breakdown" and rep["breakdown_step"] == 7
    # the context is still usable afterwards
    s.set_coefficients(diag, rhs, np.zeros(N))
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-12, "Maximum Iterations": 100}).solve(s)
    assert rep["converged"]


def test_face_average_matches_interpolation(ctx):
    n = (7, 6, 5)
    g = D.Grid(ctx, n, None, 2, (1, 0, 1))
    cell = np.random.default_rng(4).random(n)
    dc = D.DeviceArray(cell)
    faces = [D.DeviceArray(np.zeros(g.face_shape(d))) for d in range(3)]
    D.face_average(g, dc.ptr, faces)
    ctx.synchronize()
    for d, per in enumerate((1, 0, 1)):
        got = faces[d].t.cpu().numpy()
        lo = np.roll(cell, 1, axis=d)
        exp_inner = (lo + cell) * 0.5
        sl = [slice(None)] * 3
        sl[d] = slice(0, n[d])
        if per:
            np.testing.assert_array_equal(got[tuple(sl)], exp_inner)
        else:
            sl2 = [slice(None)] * 3
            sl2[d] = slice(1, n[d])
            np.testing.assert_array_equal(got[tuple(sl2)], exp_inner[tuple(sl2)])
            sl0 = [slice(None)] * 3
            sl0[d] = 0
            np.testing.assert_array_equal(got[tuple(sl0)], np.take(cell, 0, axis=d))


def _hetero_system(ctx, n, seed=0):
    c = W.heterogeneous(n=n, seed=seed)
    Dc = c["cell_D"]
    faces = []
    for d in range(3):
        f = (np.roll(Dc, 1, axis=d) + Dc) * 0.5
        first = [slice(None)] * 3
        first[d] = slice(0, 1)
        faces.append(np.concatenate([f, f[tuple(first)]], axis=d))
    c["face_D"] = faces
    c["D"] = None
    g, f, s, asm, keep, dim = _gpu_case(ctx, c)
    s.build(f, asm)
    return c, g, f, s, asm, keep


def test_mixed_precision_refinement_matches_fp64(ctx):
    """FP32 inner BiCGStab2 + FP64 refinement reaches the FP64 residual and
    the FP64 oracle solution (heterogeneous-D TVD operator)."""
    c, g, f, s, asm, keep = _hetero_system(ctx, 24)
    diag, rhs = s.coefficients()
    x0 = s.solution()
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-12, "Maximum Iterations": 500, "tol_relative": 1},
                      precision="FP32_REFINE").solve(s)
    assert rep["converged"] and not rep["fallback_used"], rep
    assert rep["refinements"] >= 2
    assert rep["true_res_abs"] <= 1e-12 * rep["b_norm"] * 1.0000001
    x = s.solution()
    og = oracle_grid(c)
    mask = np.full(g.num_cells, 127, dtype=np.uint8)
    rp, cols, vals = O.export_csr(og, np.ascontiguousarray(diag), mask)
    ox, info = O.bicgstab2(rp, cols, vals, rhs, x0, 1e-12 * np.linalg.norm(rhs), 500)
    assert info["converged"]
    assert rel_l2(x, ox) < SOL_TOL


def test_mixed_precision_fallback(ctx):
    """An inner budget too small to contract the residual engages the FP64 fallback."""
    c, g, f, s, asm, keep = _hetero_system(ctx, 16, seed=1)
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 500, "tol_relative": 1,
                       "inner_max_it": 1, "inner_rel_tol": 1e-30, "max_refinements": 2},
                      precision="FP32_REFINE").solve(s)
    assert rep["converged"] and rep["fallback_used"] == 1, rep
    assert rep["true_res_abs"] <= 1e-10 * rep["b_norm"] * 1.0000001


def test_cxx_host_api_example(tmp_path):
    """The C++ API (include/dare_gpu.hpp) drives the same path: a DaRe-style
    time loop in C++ matches the oracle's loop on the same inputs."""
    import json
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "dare_b200", "bin", "example_diffusion")
    n, steps = 20, 3
    out = tmp_path / "phi.bin"
    res = subprocess.run([exe, str(n), str(steps), str(out)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    line = json.loads(res.stdout.strip().splitlines()[-1])
    got = np.fromfile(out, dtype=np.float64)
    c = (np.arange(n) + 0.5) / n - 0.5
    r2 = c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2
    case = {"n": (n, n, n), "size": (1.0, 1.0, 1.0), "periodic": (0, 0, 0), "dt": 1e-2, "D": 1e-3,
            "phi0": W.ghosted(np, None, np.exp(-r2 / (2.0 * 0.01))), "rel_tol": 1e-10,
            "bc": {1: (1, 1.0), 2: (1, 0.0), 3: (2, 0.0), 4: (2, 0.0), 5: (2, 0.0), 6: (2, 0.0)}}
    ohist, oiters = oracle_timeloop(case, steps)
    shape = (n + 4, n + 4, n + 4)
    assert rel_l2(interior(got, shape), interior(ohist[-1], shape)) < SOL_TOL
    assert all(abs(a - b) <= 2 for a, b in zip(line["iters"], oiters))


def test_profiling_mode_same_result(ctx):
    """Per-kernel event timing launches the same kernels directly; results match the graph path."""
    case = W.tvd_convection_diffusion(n=20, steps=2)
    hist_a, it_a, g = _gpu_timeloop(ctx, case, 2)
    ctx.set_profiling(True)
    ctx.reset_kernel_stats()
    try:
        hist_b, it_b, _ = _gpu_timeloop(ctx, case, 2)
        stats = {k: ctx.kernel_stats(k) for k in ("assemble", "step1", "step4")}
    finally:
        ctx.set_profiling(False)
    assert it_a == it_b
    for a, b in zip(hist_a, hist_b):
        np.testing.assert_array_equal(a, b)
    assert stats["assemble"][1] == 2 and stats["assemble"][0] > 0


def test_vtk_writer_device_matches_host(ctx, tmp_path):
    """dare_vtk_write (device fields) writes the same bytes as the host-array
    writer tested in tests/test_vtk_writer.py."""
    n, size = (9, 6, 7), (1.0, 0.6, 1.4)
    g = D.Grid(ctx, n, size, 2, (1, 0, 1))
    rng = np.random.default_rng(11)
    shape = tuple(x + 4 for x in n)
    a, b = rng.normal(size=shape).reshape(-1), rng.normal(size=shape).reshape(-1)
    f1, f2 = D.Field(g, 2), D.Field(g, 2)
    f1.upload(a, 0)
    f1.upload(b, 1)
    f2.upload(b, 0)
    D.write_vtk([f1, f2], ["phi", "other"], str(tmp_path / "dev"), "Cartesian3D", 7, time=1.5, level=0)
    D.write_vtk([f1], ["phi_old"], str(tmp_path / "dev"), "Old", 7, level=1)
    D.write_vtk_host(n, size, 2, [a, b], ["phi", "other"], str(tmp_path / "host"), "Cartesian3D", 7, time=1.5)
    D.write_vtk_host(n, size, 2, [b], ["phi_old"], str(tmp_path / "host"), "Old", 7)
    for rel in ("Cartesian3D_7.pvts", "Cartesian3D_7/Cartesian3D_7_0.vts", "Old_7.pvts", "Old_7/Old_7_0.vts"):
        assert (tmp_path / "dev" / rel).read_bytes() == (tmp_path / "host" / rel).read_bytes(), rel


# ---- several field components (Field<Grid,SC,N>, MatrixBlock<...,N>) ----------
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_multicomponent_linear_profiles(ctx, dim):
    """test_integration_Cartesian_Trilinos.cpp (N = 3 components, SolveScalar
    variants): every component its own Dirichlet values; rows cell * 3 + c."""
    n = [20 + d for d in range(dim)]
    bvals = [(0.0, 1.0), (1.0, 0.0), (-1.0, 2.0)]
    parts = [profile_functor_diag(dim, n, w, e) for w, e in bvals]
    N = len(parts)
    ncell = int(np.prod(n))
    diag = np.stack([p[0] for p in parts], axis=-1).reshape(7, ncell * N)
    rhs = np.stack([p[1] for p in parts], axis=-1).reshape(-1)
    x0 = np.stack([p[2] for p in parts], axis=-1).reshape(-1)
    g = D.Grid(ctx, n, [1.0 + d for d in range(dim)], 2, None)
    s = D.MatrixSystem(g, components=N)
    s.set_coefficients(diag, rhs, x0)
    d2, r2 = s.coefficients()
    np.testing.assert_array_equal(d2, diag)
    np.testing.assert_array_equal(r2, rhs)
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-14, "Maximum Iterations": 5000}, precond="JACOBI").solve(s)
    assert rep["converged"], rep
    x = s.solution().reshape(ncell, N)
    nn = n + [1] * (3 - dim)
    i = np.repeat(np.arange(nn[0]), nn[1] * nn[2])
    for c, (w, e) in enumerate(bvals):
        assert np.max(np.abs(x[:, c] - (w + (e - w) * (i + 0.5) / nn[0]))) < 1e-8
    # the exported pattern interleaves the components, and the oracle's
    # BiCGStab2 on that matrix gives the same solution
    rp, cols, vals = interleave_csr([diag_to_csr(dim, n, p[0]) for p in parts])
    grp, gcols, gvals = s.export_csr()
    np.testing.assert_array_equal(grp, rp)
    np.testing.assert_array_equal(gcols, cols)
    np.testing.assert_array_equal(gvals, vals)
    ox, info = O.bicgstab2(rp, cols, vals, rhs, x0, 1e-14, 5000, O.PREC_JACOBI)
    assert rel_l2(x.reshape(-1), ox) < SOL_TOL
    assert abs(rep["iters"] - info["iters"]) <= max(2, info["iters"] // 10)


@pytest.mark.parametrize("periodic", [(1, 1, 1), (0, 1, 0)])
def test_multicomponent_assembly_and_timeloop(ctx, periodic):
    """Two components of one convected scalar pair: the descriptor applies to
    each component's values (1e-13), one BiCGStab2 runs on both (runs of
    planes and the periodic x wrap stay inside a component)."""
    case = _random_case("tiles3d", 5)
    n = case["n"]
    case["periodic"] = periodic
    case["bc"] = {} if periodic[0] else {1: (1, 0.3), 2: (2, 0.0), 5: (2, 0.0), 6: (1, -0.5)}
    rng = np.random.default_rng(9)
    shape = tuple(x + 4 for x in n)
    comps = [rng.random(shape), 0.5 + 0.25 * rng.random(shape)]
    old = [rng.random(shape), rng.random(shape)]
    N = len(comps)
    inter = lambda arrs: np.stack([a.reshape(-1) for a in arrs], axis=-1).reshape(-1)
    g = D.Grid(ctx, n, case["size"], 2, periodic)
    f = D.Field(g, 2, components=N)
    f.upload(inter(comps), 0)
    f.upload(inter(old), 1)
    np.testing.assert_array_equal(f.download(0), inter(comps))
    s = D.MatrixSystem(g, components=N)
    for face, (kind, val) in case["bc"].items():
        s.set_bc(int(face), kind, val)
    keep = [D.DeviceArray(np.asarray(a)) for a in case["face_vel"]] + [D.DeviceArray(np.asarray(a)) for a in
                                                                      case["face_D"]]
    asm = D.Assembly(dt=case["dt"], face_D=tuple(keep[3:]), face_vel=tuple(keep[:3]), limiter="VANLEER")
    s.build(f, asm)
    diag, rhs = s.coefficients()
    og = oracle_grid(case)
    desc = oracle_assembly(og, case, face_D=case["face_D"])
    per = [O.assemble(desc, np.ascontiguousarray(c.reshape(-1)), np.ascontiguousarray(o.reshape(-1)))
           for c, o in zip(comps, old)]
    ncell = int(np.prod(n))
    assert_coef_close(diag, np.stack([p[0] for p in per], axis=-1).reshape(7, ncell * N))
    assert_coef_close(rhs, np.stack([p[1] for p in per], axis=-1).reshape(-1))
    # two implicit steps against the oracle's solve of the interleaved system
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1})
    ocomps = [c.reshape(-1).copy() for c in comps]
    oold = [o.reshape(-1).copy() for o in old]
    for _ in range(2):
        rep = D.timestep(s, f, asm, solver)
        assert rep["converged"], rep
        per = [O.assemble(desc, c, o) for c, o in zip(ocomps, oold)]
        rp, cols, vals = interleave_csr([O.export_csr(og, p[0], p[2]) for p in per])
        b = np.stack([p[1] for p in per], axis=-1).reshape(-1)
        x0 = np.stack([O.field_to_vector(og, c) for c in ocomps], axis=-1).reshape(-1)
        x, info = O.bicgstab2(rp, cols, vals, b, x0, 1e-10 * np.linalg.norm(b), 5000)
        xs = x.reshape(ncell, N)
        for c in range(N):
            O.copy_to_field(og, np.ascontiguousarray(xs[:, c]), ocomps[c])
            O.exchange_halo(og, ocomps[c])
            oold[c] = ocomps[c].copy()
        got = f.download(0).reshape(-1, N)
        for c in range(N):
            assert rel_l2(interior(got[:, c], g.ghosted_shape), interior(ocomps[c], g.ghosted_shape)) < SOL_TOL
        assert abs(rep["iters"] - info["iters"]) <= 2


@pytest.mark.parametrize("kind", ["tvd-periodic", "gaussian-bounded"])
def test_host_resident_steps_match_single_calls(ctx, kind):
    """dare_timesteps_host (each step's field from pinned host memory, the
    result back to it, transfers of consecutive steps pipelined in slices,
    each slice's planes assembled as it lands) gives the loop of single
    upload / copy-to-old / timestep / download calls bit for bit, the old
    level included; an unpinned buffer is refused."""
    import torch
    if kind == "tvd-periodic":
        case = W.tvd_convection_diffusion(n=24, steps=3)
    else:
        case = W.gaussian_diffusion(n=20, steps=3)
    g, f, s, asm, keep, dim = _gpu_case(ctx, case)
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1})
    phi0 = f.download(0)
    host = torch.empty(g.num_cells_ghosted, dtype=torch.float64, pin_memory=True).numpy()
    host[:] = phi0
    reps = D.timesteps_host(s, f, asm, solver, 3, host)
    assert len(reps) == 3 and all(r["converged"] for r in reps)
    np.testing.assert_array_equal(f.download(0), host)
    np.testing.assert_array_equal(f.download(1), host)   # CopyDataVectorsToOldTimeStep of the last step
    ref = phi0.copy()
    iters = []
    for _ in range(3):
        f.upload(ref, 0)
        f.copy_to_old()
        iters.append(D.timestep(s, f, asm, solver)["iters"])
        ref = f.download(0)
    assert [r["iters"] for r in reps] == iters
    assert np.array_equal(host, ref)
    with pytest.raises(D.DareError):
        D.timesteps_host(s, f, asm, solver, 1, np.zeros(g.num_cells_ghosted))


def _periodic_2d_case():
    rng = np.random.default_rng(31)
    n = (20, 18)
    return {"n": n, "size": (1.0, 1.25), "periodic": (1, 1), "dt": 0.01, "D": 1e-3, "vel": (0.3, -0.2),
            "limiter": "VANLEER", "phi0": rng.random((24, 22, 1)), "phi_old": rng.random((24, 22, 1)), "bc": {}}


@pytest.mark.parametrize("kind,precond", [("tvd-periodic", "JACOBI"), ("tvd-periodic", "NONE"),
                                          ("gaussian-bounded", "JACOBI"), ("periodic-2d", "JACOBI")])
def test_timestep_field_write_matches_separate_calls(ctx, kind, precond):
    """dare_timestep writes the solution into the field, with its periodic
    face ghosts, in the pass that ends the solve (x = M^-1 y); the separate
    calls Build, Solve, CopyTo, ExchangeHaloCells and
    CopyDataVectorsToOldTimeStep give the same field (both levels, every
    ghost) and the same solution vector, bit for bit."""
    if kind == "tvd-periodic":
        case = W.tvd_convection_diffusion(n=24, steps=1)
    elif kind == "gaussian-bounded":
        case = W.gaussian_diffusion(n=20, steps=1)
    else:
        case = _periodic_2d_case()
    g, f, s, asm, keep, dim = _gpu_case(ctx, case)
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1,
                          "compute_true_residual": 0}, precond=precond)
    phi0, old0 = f.download(0), f.download(1)
    rep = D.timestep(s, f, asm, solver)
    got0, got1, gx = f.download(0), f.download(1), s.solution()
    f.upload(phi0, 0)
    f.upload(old0, 1)
    s.build(f, asm)
    rep2 = solver.solve(s)
    s.copy_to(f)
    f.exchange_halo()
    f.copy_to_old()
    assert rep["converged"] and rep["iters"] == rep2["iters"]
    np.testing.assert_array_equal(gx, s.solution())
    np.testing.assert_array_equal(got0, f.download(0))
    np.testing.assert_array_equal(got1, f.download(1))


@pytest.mark.parametrize("precond", ["NONE", "JACOBI"])
def test_breakdown_after_step10_keeps_its_update(ctx, precond):
    """A = 2 I: alpha = 1/2 makes r' = r - alpha v exactly 0, so s = 0 and
    gamma = 0 at step (14).  The reference leaves its loop there with step
    (10)'s x = x0 + alpha u, the exact solution b / 2 (BiCGStab2.inl:373-392);
    the device solve, which applies step (10) in its last kernel, must apply
    it on this exit too.  The oracle's solve stops at the same step."""
    n = (6, 5, 4)
    g = D.Grid(ctx, n, None, 2, (1, 1, 1))
    s = D.MatrixSystem(g)
    N = g.num_cells
    diag = np.zeros((7, N))
    diag[0] = 2.0
    rng = np.random.default_rng(11)
    rhs, x0 = rng.random(N), rng.random(N)
    s.set_coefficients(diag, rhs, x0)
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-300, "Maximum Iterations": 50}, precond=precond).solve(s)
    assert rep["status_name"] == "breakdown" and rep["breakdown_step"] == 14, rep
    x = s.solution()
    # x0 + (b - 2 x0) / 2 (or D^-1 (x0 + (b - x0))): b / 2 up to the rounding
    # of that sum; without step (10) it would be x0
    np.testing.assert_allclose(x, rhs / 2, rtol=0, atol=2e-16)
    if precond == "NONE":
        # the oracle stops at the same step with the same x.  (With Jacobi its
        # OpenMP dot products may sum in another order, alpha misses 1 by an
        # ulp, and it goes on with steps of tiny quantities divided by tiny
        # quantities, which end anywhere: no comparator for this exit.)
        rp, cols, vals = s.export_csr()
        ox, info = O.bicgstab2(rp, cols, vals, rhs, x0, 1e-300, 50, O.PREC_NONE)
        np.testing.assert_allclose(x, ox, rtol=0, atol=1e-15)
    # the FP32 inner solves break down the same way; their step (10) makes
    # the correction exact, so the refinement converges without the fallback
    s.set_coefficients(diag, rhs, x0)
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-12, "Maximum Iterations": 50, "tol_relative": 1},
                      precond="JACOBI", precision="FP32_REFINE").solve(s)
    assert rep["converged"] and rep["fallback_used"] == 0, rep
    np.testing.assert_allclose(s.solution(), rhs / 2, rtol=1e-6)


def test_handles_outlive_their_context():
    """Handles may be destroyed after the context they came from (a garbage
    collector picks the order): each destroy uses the device it recorded,
    and no stale CUDA error reaches the next launch."""
    c1 = D.Context(0)
    g = D.Grid(c1, (8, 6, 4), None, 2, (1, 1, 1))
    f = D.Field(g, 2)
    s = D.MatrixSystem(g)
    sl = D.Slabs(s, 2)
    c1.close()
    del sl, s, f, g
    c2 = D.Context(0)
    g2 = D.Grid(c2, (8, 6, 4), None, 2, (1, 1, 1))
    s2 = D.MatrixSystem(g2)
    diag = np.zeros((7, g2.num_cells))
    diag[0] = 7.0
    diag[1:] = -1.0
    s2.set_coefficients(diag, np.random.default_rng(5).random(g2.num_cells), np.zeros(g2.num_cells))
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-12, "Maximum Iterations": 100}).solve(s2)
    assert rep["converged"]
