"""Composed assembly functors (dare_assemble_terms) against the oracle: the
reference's own verification functors -- counter_diffusion1D.cpp:107-148
(mb = ddt(field); mb -= div(grad(mb)); Dirichlet for one component and
Neumann for the other on each end) and advection_periodic2D.cpp:108-126
(mb = ddt(field); mb.Add(c, div(TVD(u_c) * field).GetSlice(c)) with a
velocity per component) -- assembled on the GPU bit for bit (the 1-D / 2-D
kernel keeps the reference's operation order) and stepped in time against
the oracle's loop; a 3-D composition within 1e-13 of the fused descriptor
and of the oracle."""
import numpy as np
import pytest

import dare_b200 as D
from dare_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import (assert_coef_close, interior, interleave_csr, oracle_grid, oracle_terms, rel_l2)

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-9


@pytest.fixture(scope="module")
def ctx():
    return D.Context(0)


def _inter(arrs):
    return np.stack([np.asarray(a).reshape(-1) for a in arrs], axis=-1).reshape(-1)


def _setup(ctx, case, comps, olds, bcs):
    N = len(comps)
    g = D.Grid(ctx, case["n"], case["size"], 2, case["periodic"])
    f = D.Field(g, 2, components=N)
    f.upload(_inter(comps), 0)
    f.upload(_inter(olds), 1)
    s = D.MatrixSystem(g, components=N)
    for c, bc in enumerate(bcs):
        for face, (kind, value) in bc.items():
            if face <= 2 * len(case["n"]) and not case["periodic"][(face - 1) // 2]:
                s.set_bc(face, kind, value, component=c)
    return g, f, s


def _gpu_terms(terms):
    return [D.Term(t["kind"], t["op"], component=t["component"], dt=t.get("dt", 0.0), D=t.get("D", 1.0),
                   vel=t.get("vel"), limiter=t.get("limiter", "VANLEER")) for t in terms]


def _oracle_step(og, case, terms, ph, ol, bcs):
    """One step of the driver loop on the oracle, fields updated in place;
    returns the iterations."""
    N = len(ph)
    diag, rhs, (pd, pr), mask = oracle_terms(og, case, terms, ph, ol, bcs)
    rp, cols, vals = interleave_csr([O.export_csr(og, d, mask) for d in pd])
    x0 = _inter([O.field_to_vector(og, p) for p in ph])
    x, info = O.bicgstab2(rp, cols, vals, rhs, x0, 1e-10 * np.linalg.norm(rhs), 5000)
    assert info["converged"]
    xs = x.reshape(-1, N)
    for c in range(N):
        O.copy_to_field(og, np.ascontiguousarray(xs[:, c]), ph[c])
        O.exchange_halo(og, ph[c])
        ol[c][:] = ph[c]
    return info["iters"]


def _loop(ctx, case, terms, comps, olds, bcs, steps):
    """The reference's driver loop with a composed functor, on the GPU and on
    the oracle: Build, Solve, CopyTo, ExchangeHaloCells, CopyDataVectorsToOldTimeStep."""
    N = len(comps)
    g, f, s = _setup(ctx, case, comps, olds, bcs)
    gt = _gpu_terms(terms)
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1})
    og = oracle_grid(case)
    ph = [np.ascontiguousarray(c.reshape(-1)).copy() for c in comps]
    ol = [np.ascontiguousarray(o.reshape(-1)).copy() for o in olds]
    dim = len(case["n"])
    for _ in range(steps):
        s.build(f, gt)
        rep = solver.solve(s)
        assert rep["converged"], rep
        s.copy_to(f)
        f.exchange_halo()
        f.copy_to_old()
        its = _oracle_step(og, case, terms, ph, ol, bcs)
        got = f.download(0).reshape(-1, N)
        for c in range(N):
            a = interior(got[:, c], g.ghosted_shape, dim=dim)
            assert rel_l2(a, interior(ph[c], g.ghosted_shape, dim=dim)) < SOL_TOL, c
        assert abs(rep["iters"] - its) <= 2


def _counter_diffusion(nx, seed=None):
    """counter_diffusion1D.cpp: nx cells on [0, 1], dt = 1e-3, two components;
    component 0 Dirichlet 1 at the west face and zero-gradient at the east,
    component 1 the reverse.  The reference starts from zero; a seed gives a
    random start."""
    case = {"n": (nx,), "size": (1.0,), "periodic": (0,)}
    shape = (nx + 4, 1, 1)
    if seed is None:
        comps = [np.zeros(shape), np.zeros(shape)]
    else:
        rng = np.random.default_rng(seed)
        comps = [rng.random(shape), rng.random(shape)]
    terms = [{"kind": "DDT", "op": "SET", "component": -1, "dt": 1e-3},
             {"kind": "DIFFUSION", "op": "SUB", "component": -1, "D": 1.0}]
    bcs = [{1: (O.BC_DIRICHLET, 1.0), 2: (O.BC_NEUMANN, 0.0)}, {1: (O.BC_NEUMANN, 0.0), 2: (O.BC_DIRICHLET, 1.0)}]
    return case, comps, terms, bcs


def _advection(n, limiter="MINMOD"):
    """advection_periodic2D.cpp: periodic unit square, dt = 1e-3, a disk of
    radius 0.25 at the centre set to 1 in both components; component 0
    carried by u = (1, 0), component 1 by u = (0, 1), TVD MINMOD."""
    case = {"n": (n, n), "size": (1.0, 1.0), "periodic": (1, 1)}
    c = (np.arange(n) + 0.5) / n - 0.5
    disk = (np.sqrt(c[:, None] ** 2 + c[None, :] ** 2) < 0.25).astype(np.float64)
    phi = np.zeros((n + 4, n + 4, 1))
    phi[2:n + 2, 2:n + 2, 0] = disk
    comps = [phi.copy(), phi.copy()]
    terms = [{"kind": "DDT", "op": "SET", "component": -1, "dt": 1e-3},
             {"kind": "CONVECTION", "op": "ADD", "component": 0, "vel": (1.0, 0.0), "limiter": limiter},
             {"kind": "CONVECTION", "op": "ADD", "component": 1, "vel": (0.0, 1.0), "limiter": limiter}]
    return case, comps, terms, [{}, {}]


@pytest.mark.parametrize("nx,seed", [(10, None), (64, 3)])
def test_counter_diffusion_functor_bit_exact(ctx, nx, seed):
    case, comps, terms, bcs = _counter_diffusion(nx, seed)
    rng = np.random.default_rng(7)
    olds = [c + 0.1 * rng.random(c.shape) for c in comps]
    g, f, s = _setup(ctx, case, comps, olds, bcs)
    s.build(f, _gpu_terms(terms))
    diag, rhs = s.coefficients()
    odiag, orhs, _, _ = oracle_terms(oracle_grid(case), case, terms, [c.reshape(-1) for c in comps],
                                     [o.reshape(-1) for o in olds], bcs)
    np.testing.assert_array_equal(diag, odiag)
    np.testing.assert_array_equal(rhs, orhs)
    # the components are folded differently: Dirichlet on the west face of
    # component 0 moves 2 bc X into its rhs, Neumann on component 1 does not
    assert rhs[0] != rhs[1]


def test_counter_diffusion_functor_time_loop(ctx):
    case, comps, terms, bcs = _counter_diffusion(40)
    _loop(ctx, case, terms, comps, [c.copy() for c in comps], bcs, steps=5)


@pytest.mark.parametrize("limiter", ["MINMOD", "VANLEER"])
def test_advection_functor_bit_exact(ctx, limiter):
    case, comps, terms, bcs = _advection(50, limiter)
    g, f, s = _setup(ctx, case, comps, comps, bcs)
    s.build(f, _gpu_terms(terms))
    diag, rhs = s.coefficients()
    odiag, orhs, _, _ = oracle_terms(oracle_grid(case), case, terms, [c.reshape(-1) for c in comps],
                                     [c.reshape(-1) for c in comps], bcs)
    np.testing.assert_array_equal(diag, odiag)
    np.testing.assert_array_equal(rhs, orhs)


def test_advection_functor_time_loop(ctx):
    case, comps, terms, bcs = _advection(32)
    _loop(ctx, case, terms, comps, [c.copy() for c in comps], bcs, steps=3)


def test_terms_3d_match_fused_and_oracle(ctx):
    """mb = ddt(field); mb += div(TVD(u) * field); mb -= div(D grad(mb)) as
    three terms gives the fused descriptor's coefficients (1e-13) and the
    oracle's composition; a second component convected by its own constant
    velocity shows the per-component term."""
    case = W.tvd_convection_diffusion(n=24, seed=5)
    fv = [np.asarray(a) for a in case["face_vel"]]
    g = D.Grid(ctx, case["n"], case["size"], 2, case["periodic"])
    f1 = D.Field(g, 2)
    phi = np.ascontiguousarray(case["phi0"].reshape(-1))
    f1.upload(phi, 0)
    f1.upload(phi, 1)
    vel = [D.DeviceArray(a) for a in fv]
    s_fused = D.MatrixSystem(g)
    s_fused.build(f1, D.Assembly(dt=case["dt"], D=case["D"], face_vel=tuple(vel), limiter="VANLEER"))
    s_terms = D.MatrixSystem(g)
    s_terms.build(f1, [D.Term("DDT", "SET", dt=case["dt"]), D.Term("CONVECTION", "ADD", face_vel=tuple(vel)),
                       D.Term("DIFFUSION", "SUB", D=case["D"])])
    d1, r1 = s_fused.coefficients()
    d2, r2 = s_terms.coefficients()
    assert_coef_close(d2, d1)
    assert_coef_close(r2, r1)
    # two components: component 1 with a constant velocity term of its own
    rng = np.random.default_rng(2)
    comps = [case["phi0"], rng.random(case["phi0"].shape)]
    terms = [{"kind": "DDT", "op": "SET", "component": -1, "dt": case["dt"]},
             {"kind": "DIFFUSION", "op": "SUB", "component": -1, "D": case["D"]},
             {"kind": "CONVECTION", "op": "ADD", "component": 1, "vel": (0.05, -0.02, 0.01), "limiter": "MINMOD"}]
    gg, f2, s2 = _setup(ctx, case, comps, comps, [{}, {}])
    s2.build(f2, _gpu_terms(terms))
    d, r = s2.coefficients()
    od, orr, _, _ = oracle_terms(oracle_grid(case), case, terms, [c.reshape(-1) for c in comps],
                                 [c.reshape(-1) for c in comps], [{}, {}])
    assert_coef_close(d, od)
    assert_coef_close(r, orr)


def test_cxx_counter_diffusion_example(tmp_path):
    """counter_diffusion1D.cpp written against the C++ API's MatrixBlock
    (dare_b200/cxx/example_counter_diffusion.cpp): 20 steps against the
    oracle's loop of the same functor."""
    import json
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "dare_b200", "bin", "example_counter_diffusion")
    nx, steps = 10, 20
    out = tmp_path / "phi.bin"
    res = subprocess.run([exe, str(nx), str(steps), str(out)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    line = json.loads(res.stdout.strip().splitlines()[-1])
    got = np.fromfile(out, dtype=np.float64).reshape(-1, 2)
    case, comps, terms, bcs = _counter_diffusion(nx)
    og = oracle_grid(case)
    ph = [np.ascontiguousarray(c.reshape(-1)).copy() for c in comps]
    ol = [p.copy() for p in ph]
    its = [_oracle_step(og, case, terms, ph, ol, bcs) for _ in range(steps)]
    shape = (nx + 4, 1, 1)
    for c in range(2):
        assert rel_l2(interior(got[:, c], shape, dim=1), interior(ph[c], shape, dim=1)) < SOL_TOL
    assert all(abs(a - b) <= 2 for a, b in zip(line["iters"], its))
    # the two components mirror each other: c0(x) = c1(1 - x)
    i0 = interior(got[:, 0], shape, dim=1).ravel()
    i1 = interior(got[:, 1], shape, dim=1).ravel()
    np.testing.assert_allclose(i0, i1[::-1], rtol=0, atol=1e-8)


@pytest.mark.parametrize("n,periodic", [((18, 14), (0, 1)), ((12, 10, 9), (0, 1, 1))])
def test_caller_coefficients_term(ctx, n, periodic):
    """COEFFS terms (per-cell slot and rhs values the caller computed on the
    device) composed with DDT and diffusion, for every component and for
    one, then folded with each component's conditions: 2-D bit for bit,
    3-D within 1e-13 of the oracle's composition of the same parts."""
    import torch
    rng = np.random.default_rng(41)
    dim, N = len(n), 2
    case = {"n": n, "size": tuple(1.0 + 0.1 * d for d in range(dim)), "periodic": periodic}
    gh = tuple(x + 4 for x in n)
    comps = [rng.random(gh) for _ in range(N)]
    olds = [rng.random(gh) for _ in range(N)]
    bcs = [{1: (O.BC_DIRICHLET, 1.0 + c), 2: (O.BC_NEUMANN, 0.0)} for c in range(N)]
    g, f, s = _setup(ctx, case, comps, olds, bcs)
    ncell = int(np.prod(n))
    coef = [rng.random(ncell) + 1.0] + [-0.1 * rng.random(ncell) if q <= 2 * dim else None for q in range(1, 7)]
    rhs = rng.normal(size=ncell)
    extra = [rng.random(ncell)] + [None] * 6
    dev = lambda a: None if a is None else D.DeviceArray(a)
    coef_d, rhs_d, extra_d = [dev(a) for a in coef], dev(rhs), [dev(a) for a in extra]
    terms = [dict(kind="DDT", op="SET", component=-1, dt=0.05),
             dict(kind="COEFFS", op="ADD", component=-1, coef=coef, rhs=rhs),
             dict(kind="DIFFUSION", op="SUB", component=-1, D=0.01),
             dict(kind="COEFFS", op="SUB", component=1, coef=extra, rhs=None)]
    gpu = [D.Term("DDT", "SET", dt=0.05),
           D.Term("COEFFS", "ADD", coef=tuple(coef_d), rhs=rhs_d),
           D.Term("DIFFUSION", "SUB", D=0.01),
           D.Term("COEFFS", "SUB", component=1, coef=tuple(extra_d))]
    s.build(f, gpu)
    gd, gr = s.coefficients()
    od, orhs, _, _ = oracle_terms(oracle_grid(case), case, terms, [c.reshape(-1) for c in comps],
                                  [o.reshape(-1) for o in olds], bcs)
    if dim < 3:
        assert np.array_equal(gd, od) and np.array_equal(gr, orhs)
    else:
        assert_coef_close(gd, od)
        assert_coef_close(gr, orhs)
