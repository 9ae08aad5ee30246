"""GPU parity at the benchmark configurations' own sizes, through the C ABI,
against the CPU oracle on the same seeded inputs.

* 64^3 transient diffusion (Gaussian bump, Dirichlet 1 / 0 on x, Neumann
  elsewhere), 10 implicit steps: every step's field within 1e-9 relative L2
  of the oracle's driver loop, iterations within 2.
* 128^3 TVD convection-diffusion (van Leer, Pe 5, CFL 0.5), two steps:
  the same bar (the 256^3 case is compared in the benchmark's `parity` key).
* 128^3 heterogeneous log-normal D: the FP32-inner / FP64-refinement solve
  against the oracle's FP64 solve of the same assembled system, 1e-9.
* 35 boxes of the batched workload with sides 16, 24, 32, 48 and 64 (every
  size class, so every cells-per-thread class of the batched kernel runs):
  each instance against the oracle's assembly + BiCGStab2, 1e-9.
"""
import numpy as np
import pytest

import dare_b200 as D
from dare_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import interior, oracle_grid, oracle_timeloop, rel_l2
from tests.test_gpu_batched import _oracle_solve
from tests.test_gpu_parity import _gpu_case, _gpu_timeloop, _hetero_system

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-9


@pytest.fixture(scope="module")
def ctx():
    c = D.Context(0)
    yield c
    c.synchronize()


def test_gaussian_64_ten_steps(ctx):
    case = W.gaussian_diffusion(n=64, seed=0, steps=10)
    hist, iters, g = _gpu_timeloop(ctx, case, 10)
    ohist, oiters = oracle_timeloop(case, 10)
    for step, (a, b) in enumerate(zip(hist, ohist)):
        err = rel_l2(interior(a, g.ghosted_shape), interior(b, g.ghosted_shape))
        assert err < SOL_TOL, (step, err)
    assert all(abs(a - b) <= 2 for a, b in zip(iters, oiters)), (iters, oiters)


def test_tvd_128_two_steps(ctx):
    case = W.tvd_convection_diffusion(n=128, seed=3, steps=2)
    hist, iters, g = _gpu_timeloop(ctx, case, 2)
    ohist, oiters = oracle_timeloop(case, 2)
    for a, b in zip(hist, ohist):
        assert rel_l2(a, b) < SOL_TOL       # internal and (periodic) ghost cells
    assert all(abs(a - b) <= 2 for a, b in zip(iters, oiters)), (iters, oiters)


def test_mixed_precision_128_lognormal(ctx):
    c, g, f, s, asm, keep = _hetero_system(ctx, 128, seed=2)
    diag, rhs = s.coefficients()
    x0 = s.solution()
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1},
                      precision="FP32_REFINE").solve(s)
    assert rep["converged"] and not rep["fallback_used"], rep
    assert rep["true_res_abs"] <= 1e-10 * rep["b_norm"] * 1.0000001
    og = oracle_grid(c)
    mask = np.full(g.num_cells, 127, dtype=np.uint8)
    rp, cols, vals = O.export_csr(og, np.ascontiguousarray(diag), mask)
    ox, info = O.bicgstab2(rp, cols, vals, rhs, x0, 1e-10 * np.linalg.norm(rhs), 5000)
    assert info["converged"]
    assert rel_l2(s.solution(), ox) < SOL_TOL


def test_batched_every_size_class():
    ctx = D.Context(0)
    pool = W.batched_diffusion(count=400, seed=11)
    by_side = {}
    for ins in pool:
        by_side.setdefault(ins["n"][0], []).append(ins)
    assert sorted(by_side) == [16, 24, 32, 48, 64]
    inst = [ins for side in sorted(by_side) for ins in by_side[side][:7]]
    rng = np.random.default_rng(12)
    order = rng.permutation(len(inst))
    inst = [inst[q] for q in order]
    bt = D.Batch(ctx, inst)
    bt.zero_fields()
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 10000, "tol_relative": 1})
    reps = bt.solve(solver)
    for q, ins in enumerate(inst):
        assert reps[q]["converged"], (q, ins["n"], reps[q])
        ox, info = _oracle_solve(ins, np.zeros(bt.num_cells(q)), 1e-10)
        assert info["converged"]
        assert rel_l2(bt.get_field(q), ox) < SOL_TOL, (q, ins["n"])
        assert abs(reps[q]["iters"] - info["iters"]) <= 2, (q, reps[q]["iters"], info["iters"])
