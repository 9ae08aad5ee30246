"""Seeded random configurations against the oracle: grids of 1 to 3
dimensions and sizes 5-39 (some with 32-64 cells along k, the two-cells-per-
thread kernels), random periodicity, limiters, Dirichlet / Neumann faces,
plain / Jacobi FP64 and FP32-refine solves to 1e-12 relative, and, where the
x extent allows, the same solve on 2 or 3 slabs.  Bar: 1e-8 relative L2
against the oracle's solve of the oracle's assembly."""
import numpy as np
import pytest

import dare_b200 as D
from oracle import oracle as O
from tests.helpers import oracle_assembly, oracle_grid, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return D.Context(0)


def _case(seed):
    rng = np.random.default_rng(seed)
    dim = int(rng.choice([1, 2, 3], p=[0.15, 0.25, 0.6]))
    n = tuple(int(rng.integers(5, 40)) for _ in range(dim))
    if dim == 3 and rng.random() < 0.3:
        n = n[:2] + (int(rng.choice([32, 34, 48, 64])),)
    periodic = tuple(int(rng.random() < 0.5) for _ in range(dim))
    precision = str(rng.choice(["FP64", "FP64", "FP32_REFINE"]))
    precond = "JACOBI" if precision == "FP32_REFINE" else str(rng.choice(["NONE", "JACOBI"]))
    case = {"n": n, "size": tuple(float(rng.uniform(0.5, 2)) for _ in range(dim)), "periodic": periodic,
            "dt": float(rng.choice([0.005, 0.02, 0.1])), "D": float(10 ** rng.uniform(-4, -2)),
            "phi0": rng.random(tuple(x + 4 for x in n)),
            "limiter": str(rng.choice(["CDS", "UPWIND", "VANALBADA", "MINMOD", "VANLEER"])),
            "face_vel": [rng.normal(size=tuple(x + (1 if e == d else 0) for e, x in enumerate(n)))
                         for d in range(dim)], "bc": {}}
    for d in range(dim):
        if not periodic[d]:
            case["bc"][2 * d + 1] = (int(rng.choice([1, 2])), float(rng.random()))
            case["bc"][2 * d + 2] = (int(rng.choice([1, 2])), float(rng.random()))
    return case, precond, precision


@pytest.mark.parametrize("seed", range(16))
def test_random_configuration(ctx, seed):
    case, precond, precision = _case(1000 + seed)
    n, dim, lim = case["n"], len(case["n"]), case["limiter"]
    g = D.Grid(ctx, n, case["size"], 2, case["periodic"])
    f = D.Field(g, 2)
    phi = np.ascontiguousarray(case["phi0"].reshape(-1))
    f.upload(phi, 0)
    f.upload(phi, 1)
    s = D.MatrixSystem(g)
    for face, (kind, val) in case["bc"].items():
        s.set_bc(face, kind, val)
    keep = [D.DeviceArray(a) for a in case["face_vel"]]
    s.build(f, D.Assembly(dt=case["dt"], D=case["D"], face_vel=tuple(keep), limiter=lim))
    tol = 1e-12 * float(np.linalg.norm(s.coefficients()[1]))
    params = {"Convergence Tolerance": tol, "Maximum Iterations": 3000}
    rep = D.BiCGStab2(params, precond=precond, precision=precision).solve(s)
    og = oracle_grid(case)
    desc = oracle_assembly(og, dict(case, face_vel=None))
    desc.face_vel = [np.ascontiguousarray(a) for a in case["face_vel"]] + [None] * (3 - dim)
    od, orhs, mask = O.assemble(desc, phi, phi)
    rp, cols, vals = O.export_csr(og, od, mask)
    ox, info = O.bicgstab2(rp, cols, vals, orhs, O.field_to_vector(og, phi), tol, 3000,
                           O.PREC_JACOBI if precond == "JACOBI" else O.PREC_NONE)
    assert rep["converged"] and info["converged"], (rep, info)
    assert rel_l2(s.solution(), ox) < 1e-8
    if dim >= 2 and n[0] >= 6 and precision == "FP64":
        sl = D.Slabs(s, 2 if n[0] < 9 else 3, 2)
        sl.scatter(f)
        asms = []
        for fs in sl.face_slices(case["face_vel"]):
            arrs = [D.DeviceArray(a) for a in fs]
            keep += arrs
            asms.append(D.Assembly(dt=case["dt"], D=case["D"], face_vel=tuple(arrs), limiter=lim))
        sl.assemble(asms)
        srep = sl.solve(D.BiCGStab2(params, precond=precond))
        assert srep["converged"]
        assert rel_l2(sl.solution(), ox) < 1e-8
