"""Batched persistent solver: every instance against the oracle's own
assemble + BiCGStab2 on the same inputs; per-instance status isolation;
the autotuner's choice does not change results beyond rounding."""
import numpy as np
import pytest

import dare_b200 as D
from dare_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _instances(seed, count=10):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        n = tuple(int(v) for v in rng.integers(5, 13, size=3))
        bc = {f: (2, 0.0) for f in range(1, 7)}
        for f in rng.choice(np.arange(1, 7), size=int(rng.integers(1, 3)), replace=False):
            bc[int(f)] = (1, float(rng.uniform(0.0, 1.0)))
        out.append({"n": n, "size": tuple(float(v) for v in rng.uniform(0.5, 2.0, size=3)),
                    "D": float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-1)))), "dt": 1e-2, "bc": bc})
    return out


def _oracle_solve(ins, phi, rel_tol):
    g = O.make_grid(3, ins["n"], ins["size"], 2, (0, 0, 0))
    ghost = np.zeros(O.ghosted_shape(g))
    n = ins["n"]
    ghost[2:2 + n[0], 2:2 + n[1], 2:2 + n[2]] = phi.reshape(n)
    ghost = np.ascontiguousarray(ghost.reshape(-1))
    desc = O.AssemblyDesc(g, dt=ins["dt"], D=ins["D"], bc=ins["bc"])
    diag, rhs, mask = O.assemble(desc, ghost, ghost)
    rp, cols, vals = O.export_csr(g, diag, mask)
    x, info = O.bicgstab2(rp, cols, vals, rhs, phi.copy(), rel_tol * np.linalg.norm(rhs), 5000)
    return x, info


def test_batched_matches_oracle_per_instance():
    ctx = D.Context(0)
    inst = _instances(1)
    rng = np.random.default_rng(2)
    fields = [rng.random(int(np.prod(i["n"]))) for i in inst]
    bt = D.Batch(ctx, inst)
    for q, f in enumerate(fields):
        bt.set_field(q, f)
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1})
    reps = bt.solve(solver)
    for q, ins in enumerate(inst):
        assert reps[q]["converged"], (q, reps[q])
        ox, info = _oracle_solve(ins, fields[q], 1e-10)
        assert info["converged"]
        assert rel_l2(bt.get_field(q), ox) < 1e-9, q
        assert abs(reps[q]["iters"] - info["iters"]) <= 2, (q, reps[q]["iters"], info["iters"])


def test_batched_status_is_per_instance():
    ctx = D.Context(0)
    inst = _instances(3, count=6)
    bt = D.Batch(ctx, inst)
    rng = np.random.default_rng(4)
    for q in range(len(inst)):
        f = rng.random(bt.num_cells(q))
        if q == 2:
            f[7] = np.nan
        bt.set_field(q, f)
    reps = bt.solve(D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1}))
    for q, r in enumerate(reps):
        if q == 2:
            assert r["status"] == "nan" and not r["converged"]
        else:
            assert r["converged"], (q, r)


def test_batched_autotune_keeps_results():
    ctx = D.Context(0)
    inst = W.batched_diffusion(count=40, seed=5, sides=(8, 12, 16, 24))
    bt = D.Batch(ctx, inst)
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1})
    tuning = bt.autotune(solver)
    assert tuning["block"] in (256, 512, 1024)
    assert all(v in (1, 2, 4) for v in tuning["cells_per_thread_by_size"])
    reps = bt.solve(solver)
    assert all(r["converged"] for r in reps)
    for q in (0, 13, 39):
        ox, info = _oracle_solve(inst[q], np.zeros(bt.num_cells(q)), 1e-10)
        assert rel_l2(bt.get_field(q), ox) < 1e-9
