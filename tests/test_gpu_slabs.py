"""Slabs of i-planes on one device (dare_slabs_*): the reference's
distribution over ranks (CartesianDistribution.h:94-380, HaloBuffer.inl:30-208,
a sum over ranks in every dot product of BiCGStab2.inl) with the semantics
oracle/slabs.py pins on CPU ranks.  Each slab assembles its own rows from its
own field planes plus num_ghost planes exchanged from its x neighbours, and
the solve exchanges one operand plane per neighbour before every SpMV.

Bars: the slabs' rows equal the single-grid assembly bit for bit; the slab
solve (S = 2, 3, uneven splits, periodic and bounded x, plain and Jacobi)
matches the single-grid GPU solve and the oracle's solve to 1e-10 relative,
with the same iteration count under Jacobi;
one slab reproduces the single-grid solve bit for bit; two time steps of the
driver loop on slabs match the single-grid loop to 1e-10 with the same
iteration counts."""
import numpy as np
import pytest

import dare_b200 as D
from oracle import oracle as O
from tests.helpers import oracle_assembly, oracle_grid, rel_l2

pytestmark = pytest.mark.gpu

SHAPES = [(20, 24, 32), (17, 12, 10)]   # two cells per thread (even n2 >= 32) / one


@pytest.fixture(scope="module")
def ctx():
    c = D.Context(0)
    yield c
    c.synchronize()


def _case(n, periodic_x, seed=5):
    """A van Leer TVD convection-diffusion implicit step with face
    velocities; bounded axes get a Dirichlet face below, Neumann above."""
    rng = np.random.default_rng(seed)
    periodic = (periodic_x, 0, 1)
    case = {"n": n, "size": (1.0, 0.8, 1.3), "periodic": periodic, "dt": 0.02, "D": 3e-3,
            "phi0": rng.random(tuple(x + 4 for x in n)), "limiter": "VANLEER",
            "face_vel": [rng.normal(size=tuple(x + (1 if e == d else 0) for e, x in enumerate(n)))
                         for d in range(3)]}
    case["bc"] = {2 * d + 1: (D.BC_DIRICHLET, 1.0 + d) for d in range(3) if not periodic[d]}
    case["bc"].update({2 * d + 2: (D.BC_NEUMANN, 0.0) for d in range(3) if not periodic[d]})
    return case


class Setup:
    """The single grid (field, system, assembly) and its slabs."""

    def __init__(self, ctx, case, num_slabs):
        self.case = case
        self.g = D.Grid(ctx, case["n"], case["size"], 2, case["periodic"])
        self.f = D.Field(self.g, 2)
        phi = np.ascontiguousarray(case["phi0"].reshape(-1))
        self.f.upload(phi, 0)
        self.f.upload(phi, 1)
        self.s = D.MatrixSystem(self.g)
        for face, (kind, val) in case["bc"].items():
            self.s.set_bc(face, kind, val)
        self.keep = [D.DeviceArray(a) for a in case["face_vel"]]
        self.asm = D.Assembly(dt=case["dt"], D=case["D"], face_vel=tuple(self.keep), limiter=case["limiter"])
        self.sl = D.Slabs(self.s, num_slabs, 2)
        self.sl.scatter(self.f)
        self.slab_asm = []
        for fx, fy, fz in self.sl.face_slices(case["face_vel"]):
            arrs = [D.DeviceArray(fx), D.DeviceArray(fy), D.DeviceArray(fz)]
            self.keep += arrs
            self.slab_asm.append(D.Assembly(dt=case["dt"], D=case["D"], face_vel=tuple(arrs),
                                            limiter=case["limiter"]))


def _solver(precond, tol, max_it=2000):
    return D.BiCGStab2({"Convergence Tolerance": tol, "Maximum Iterations": max_it}, precond=precond)


@pytest.mark.parametrize("n", SHAPES)
@pytest.mark.parametrize("periodic_x", [1, 0])
@pytest.mark.parametrize("num_slabs", [2, 3])
def test_slab_rows_equal_single_grid_rows(ctx, n, periodic_x, num_slabs):
    st = Setup(ctx, _case(n, periodic_x), num_slabs)
    st.s.build(st.f, st.asm)
    st.sl.assemble(st.slab_asm)
    diag, rhs = st.s.coefficients()
    x0 = st.s.solution()
    P = n[1] * n[2]
    for s, (i0, i1) in enumerate(st.sl.ranges):
        sd, sr = st.sl.system(s).coefficients()
        assert np.array_equal(sd, diag[:, i0 * P:i1 * P]), (s, i0, i1)
        assert np.array_equal(sr, rhs[i0 * P:i1 * P])
        assert np.array_equal(st.sl.system(s).solution(), x0[i0 * P:i1 * P])


@pytest.mark.parametrize("n", SHAPES)
@pytest.mark.parametrize("periodic_x", [1, 0])
@pytest.mark.parametrize("num_slabs", [2, 3])
@pytest.mark.parametrize("precond", ["JACOBI", "NONE"])
def test_slab_solve_matches_single_grid_and_oracle(ctx, n, periodic_x, num_slabs, precond):
    case = _case(n, periodic_x)
    st = Setup(ctx, case, num_slabs)
    st.s.build(st.f, st.asm)
    st.sl.assemble(st.slab_asm)
    rhs = st.s.coefficients()[1]
    tol = 1e-13 * float(np.linalg.norm(rhs))
    rep_g = _solver(precond, tol).solve(st.s)
    rep_s = st.sl.solve(_solver(precond, tol))
    assert rep_g["converged"] and rep_s["converged"], (rep_g, rep_s)
    if precond == "JACOBI":
        assert rep_g["iters"] == rep_s["iters"]
    # (the unpreconditioned solve of the bounded 20 x 24 x 32 case is itself
    # rounding-sensitive: the oracle's iteration count differs from the
    # single-grid GPU solve's by up to 8 at the same tolerance, so only the
    # solutions are compared there)
    x_g = st.s.solution()
    x_s = st.sl.solution()
    assert rel_l2(x_s, x_g) < 1e-10
    # the oracle's solve of the oracle's assembly of the same step
    og = oracle_grid(case)
    phi = np.ascontiguousarray(case["phi0"].reshape(-1))
    odiag, orhs, mask = O.assemble(oracle_assembly(og, case), phi, phi)
    rp, cols, vals = O.export_csr(og, odiag, mask)
    ox, info = O.bicgstab2(rp, cols, vals, orhs, O.field_to_vector(og, phi), tol, 2000,
                           O.PREC_JACOBI if precond == "JACOBI" else O.PREC_NONE)
    assert info["converged"]
    assert rel_l2(x_s, ox) < 1e-10


@pytest.mark.parametrize("periodic_x", [1, 0])
def test_one_slab_is_the_single_grid_solve(ctx, periodic_x):
    """One slab: the x halo comes from the slab itself (periodic) or not at
    all, the items and reduction slots are the single grid's, so the solve
    is the same to the last bit."""
    st = Setup(ctx, _case(SHAPES[0], periodic_x), 1)
    st.s.build(st.f, st.asm)
    st.sl.assemble(st.slab_asm)
    tol = 1e-12 * float(np.linalg.norm(st.s.coefficients()[1]))
    rep_g = _solver("JACOBI", tol).solve(st.s)
    rep_s = st.sl.solve(_solver("JACOBI", tol))
    assert rep_g["iters"] == rep_s["iters"]
    assert np.array_equal(st.sl.solution(), st.s.solution())


@pytest.mark.parametrize("periodic_x", [1, 0])
@pytest.mark.parametrize("num_slabs", [2, 3])
def test_slab_driver_loop_matches_single_grid(ctx, periodic_x, num_slabs):
    """Two steps of Build, Solve, CopyTo, ExchangeHaloCells, copy to old on
    the slabs against the same on the single grid."""
    n = SHAPES[1]
    st = Setup(ctx, _case(n, periodic_x), num_slabs)
    solver_g, solver_s = _solver("JACOBI", 1e-12), _solver("JACOBI", 1e-12)
    its_g, its_s = [], []
    for _ in range(2):
        its_g.append(D.timestep(st.s, st.f, st.asm, solver_g)["iters"])
        its_s.append(st.sl.timestep(st.slab_asm, solver_s)["iters"])
    assert its_g == its_s
    out = D.Field(st.g, 2)
    st.sl.gather(out)
    for level in (0, 1):
        a = out.download(level).reshape(st.g.ghosted_shape)[2:-2, 2:-2, 2:-2]
        b = st.f.download(level).reshape(st.g.ghosted_shape)[2:-2, 2:-2, 2:-2]
        assert rel_l2(a.reshape(-1), b.reshape(-1)) < 1e-10


def test_exchange_fills_ghost_planes(ctx):
    """After the exchange each slab's x ghost planes hold its neighbours'
    boundary planes (wrapping on a periodic x), gathered back into a field
    identical to the single grid's halo fill."""
    n = SHAPES[1]
    st = Setup(ctx, _case(n, 1), 3)
    st.sl.exchange_halo()
    out = D.Field(st.g, 2)
    st.sl.gather(out)
    st.f.exchange_halo()
    a = out.download(0).reshape(st.g.ghosted_shape)
    b = st.f.download(0).reshape(st.g.ghosted_shape)
    assert np.array_equal(a[:, 2:-2, 2:-2], b[:, 2:-2, 2:-2])


def test_slab_arguments_rejected(ctx):
    g = D.Grid(ctx, (5, 8, 8), None, 2, None)
    s = D.MatrixSystem(g)
    with pytest.raises(D.DareError):
        D.Slabs(s, 3)            # fewer than two planes per slab
    sl = D.Slabs(s, 2)
    with pytest.raises(D.DareError):
        sl.solve(D.BiCGStab2({}, precision="FP32_REFINE"))
    with pytest.raises(D.DareError):
        sl.set_bc(D.WEST, D.BC_PERIODIC)


def test_cxx_slabs_match_whole_grid(tmp_path):
    """The C++ API's Slabs (include/dare_gpu.hpp) run the example's loop
    (Dirichlet 1 / 0 on the x ends, Neumann elsewhere) on 3 slabs: the
    gathered field matches the whole-grid run to 1e-10, same iterations."""
    import json
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "dare_b200", "bin", "example_diffusion")
    n, steps = 20, 3
    lines, fields = [], []
    for slabs in (0, 3):
        out = tmp_path / f"phi{slabs}.bin"
        res = subprocess.run([exe, str(n), str(steps), str(out), str(slabs)], capture_output=True, text=True,
                             timeout=120)
        assert res.returncode == 0, res.stderr
        lines.append(json.loads(res.stdout.strip().splitlines()[-1]))
        fields.append(np.fromfile(out, dtype=np.float64).reshape(n + 4, n + 4, n + 4)[2:-2, 2:-2, 2:-2])
    assert lines[1]["slabs"] == 3
    assert lines[0]["iters"] == lines[1]["iters"]
    assert rel_l2(fields[1].reshape(-1), fields[0].reshape(-1)) < 1e-10


def test_slab_breakdown_after_step10_keeps_its_update(ctx):
    """A = 2 I on two slabs: the solve stops at step (14) (gamma = 0) after
    step (10), whose update every slab applies on that exit: x = b / 2."""
    g = D.Grid(ctx, (6, 5, 4), None, 2, (1, 1, 1))
    s = D.MatrixSystem(g)
    sl = D.Slabs(s, 2)
    rng = np.random.default_rng(12)
    rhs, x0 = rng.random(g.num_cells), rng.random(g.num_cells)
    P = 5 * 4
    for k, (i0, i1) in enumerate(sl.ranges):
        rows = (i1 - i0) * P
        diag = np.zeros((7, rows))
        diag[0] = 2.0
        sl.system(k).set_coefficients(diag, rhs[i0 * P:i1 * P], x0[i0 * P:i1 * P])
    rep = sl.solve(D.BiCGStab2({"Convergence Tolerance": 1e-300, "Maximum Iterations": 50}, precond="NONE"))
    assert rep["status_name"] == "breakdown" and rep["breakdown_step"] == 14, rep
    np.testing.assert_allclose(sl.solution(), rhs / 2, rtol=0, atol=2e-16)


@pytest.mark.parametrize("periodic", [(1, 0), (0, 1)])
@pytest.mark.parametrize("num_slabs", [2, 3])
def test_slabs_2d(ctx, periodic, num_slabs):
    """A 2-D grid (the 1-D / 2-D assembly kernel, which keeps the CPU path's
    operation order): the slabs' rows equal the single grid's bit for bit and
    the slab solve matches the single-grid solve to 1e-10."""
    n = (19, 40)
    rng = np.random.default_rng(9)
    g = D.Grid(ctx, n, (1.0, 2.0), 2, periodic)
    f = D.Field(g, 2)
    phi = rng.random(g.num_cells_ghosted)
    f.upload(phi, 0)
    f.upload(phi, 1)
    s = D.MatrixSystem(g)
    for d in range(2):
        if not periodic[d]:
            s.set_bc(2 * d + 1, D.BC_DIRICHLET, 0.5)
            s.set_bc(2 * d + 2, D.BC_NEUMANN, 0.0)
    faces = [rng.normal(size=(n[0] + 1, n[1])), rng.normal(size=(n[0], n[1] + 1))]
    keep = [D.DeviceArray(a) for a in faces]
    s.build(f, D.Assembly(dt=0.02, D=2e-3, face_vel=tuple(keep), limiter="VANLEER"))
    sl = D.Slabs(s, num_slabs, 2)
    sl.scatter(f)
    asms = []
    for fx, fy in sl.face_slices(faces):
        arrs = [D.DeviceArray(fx), D.DeviceArray(fy)]
        keep += arrs
        asms.append(D.Assembly(dt=0.02, D=2e-3, face_vel=tuple(arrs), limiter="VANLEER"))
    sl.assemble(asms)
    diag, rhs = s.coefficients()
    for k, (i0, i1) in enumerate(sl.ranges):
        sd, sr = sl.system(k).coefficients()
        assert np.array_equal(sd, diag[:, i0 * n[1]:i1 * n[1]]), k
        assert np.array_equal(sr, rhs[i0 * n[1]:i1 * n[1]])
    tol = 1e-13 * float(np.linalg.norm(rhs))
    rg = _solver("JACOBI", tol).solve(s)
    rs = sl.solve(_solver("JACOBI", tol))
    assert rg["converged"] and rs["converged"] and rg["iters"] == rs["iters"]
    assert rel_l2(sl.solution(), s.solution()) < 1e-10


@pytest.mark.parametrize("ncomp", [2, 3])
@pytest.mark.parametrize("periodic_x", [1, 0])
def test_slabs_with_components(ctx, ncomp, periodic_x):
    """N field components (rows cell * N + c, MatrixBlock_Cartesian.inl:127-240),
    each with its own face values, on 3 slabs: each component's boundary
    planes cross separately; rows bit-exact, the solve and two steps of the
    driver loop match the single grid (1e-10, the same iterations)."""
    n = (17, 12, 32)
    rng = np.random.default_rng(21 + ncomp)
    periodic = (periodic_x, 0, 1)
    g = D.Grid(ctx, n, (1.0, 0.8, 1.3), 2, periodic)
    f = D.Field(g, 2, components=ncomp)
    phi = rng.random(g.num_cells_ghosted * ncomp)
    f.upload(phi, 0)
    f.upload(phi, 1)
    s = D.MatrixSystem(g, components=ncomp)
    for c in range(ncomp):
        for d in range(3):
            if not periodic[d]:
                s.set_bc(2 * d + 1, D.BC_DIRICHLET, 0.3 + 0.2 * c + d, component=c)
                s.set_bc(2 * d + 2, D.BC_NEUMANN, 0.0, component=c)
    faces = [rng.normal(size=tuple(x + (1 if e == d else 0) for e, x in enumerate(n))) for d in range(3)]
    keep = [D.DeviceArray(a) for a in faces]
    asm = D.Assembly(dt=0.02, D=3e-3, face_vel=tuple(keep), limiter="VANLEER")
    sl = D.Slabs(s, 3, 2)
    sl.scatter(f)
    asms = []
    for fs in sl.face_slices(faces):
        arrs = [D.DeviceArray(a) for a in fs]
        keep += arrs
        asms.append(D.Assembly(dt=0.02, D=3e-3, face_vel=tuple(arrs), limiter="VANLEER"))
    s.build(f, asm)
    sl.assemble(asms)
    diag, rhs = s.coefficients()
    P = n[1] * n[2] * ncomp
    for k, (i0, i1) in enumerate(sl.ranges):
        sd, sr = sl.system(k).coefficients()
        assert np.array_equal(sd, diag[:, i0 * P:i1 * P]), k
        assert np.array_equal(sr, rhs[i0 * P:i1 * P])
    tol = 1e-13 * float(np.linalg.norm(rhs))
    rg = _solver("JACOBI", tol).solve(s)
    rs = sl.solve(_solver("JACOBI", tol))
    assert rg["converged"] and rs["converged"] and rg["iters"] == rs["iters"]
    assert rel_l2(sl.solution(), s.solution()) < 1e-10
    # the driver loop, from the same field
    f.upload(phi, 0)
    f.upload(phi, 1)
    sl.scatter(f)
    solver_g, solver_s = _solver("JACOBI", 1e-12), _solver("JACOBI", 1e-12)
    its_g = [D.timestep(s, f, asm, solver_g)["iters"] for _ in range(2)]
    its_s = [sl.timestep(asms, solver_s)["iters"] for _ in range(2)]
    assert its_g == its_s
    out = D.Field(g, 2, components=ncomp)
    sl.gather(out)
    shape = tuple(x + 4 for x in n) + (ncomp,)
    a = out.download(0).reshape(shape)[2:-2, 2:-2, 2:-2]
    b = f.download(0).reshape(shape)[2:-2, 2:-2, 2:-2]
    assert rel_l2(a.reshape(-1), b.reshape(-1)) < 1e-10
