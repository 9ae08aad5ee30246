"""Pins the CPU oracle against the reference's own known-answer tests.

Fixtures: tests/golden/operators.json (generated by make_golden.py from the
formulas in Grid/test/test_Cartesian_Operators.cpp and
Equations/test/test_DDT.cpp).  Solver cases restate the functors of
test/test_integration_Cartesian_Trilinos.cpp and
MatrixSystem/test/test_TrilinosSolver.cpp.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "operators.json")))
SLOT = {"C": O.C_, "W": O.W, "E": O.E, "S": O.S, "N": O.N, "B": O.B, "T": O.T}


@pytest.mark.parametrize("case", GOLD["laplacian"], ids=lambda c: f"{c['dim']}D")
def test_laplacian_known_answer(case):
    # periodic grid so that the boundary folding does not touch ordinal 0;
    # the operator itself does not depend on periodicity
    dim = case["dim"]
    g = O.make_grid(dim, case["n"], case["size"], periodic=[1] * dim)
    desc = O.AssemblyDesc(g, dt=0.0, D=1.0)
    phi = np.zeros(O.ghosted_shape(g)).ravel()
    diag, rhs, mask = O.assemble(desc, phi)
    c = case["ordinal"]
    for key, val in case["expected"].items():
        assert diag[SLOT[key], c] == val, key     # EXPECT_EQ in the reference
    assert rhs[c] == 0.0


def _tvd_row(face, A0=1.0):
    # ApplyDivergence of the expected face stencil, in the reference's order
    # (Divergence_Cartesian.inl:143-197); A0 = V/dx = 1 on the 1D test grid
    C = A0 * face["E"]["c"]
    C -= A0 * face["W"]["c"]
    return {"E": A0 * face["E"]["nb"], "W": -A0 * face["W"]["nb"], "C": C,
            "rhs": A0 * (face["E"]["rhs"] - face["W"]["rhs"])}


@pytest.mark.parametrize("case", GOLD["tvd"],
                         ids=lambda c: f"{c['limiter']}-v{c['vel']:+.0f}-n{c['component']}")
def test_tvd_known_answer(case):
    lim = {"CDS": O.LIM_CDS, "UPWIND": O.LIM_UPWIND, "MINMOD": O.LIM_MINMOD,
           "VANALBADA": O.LIM_VANALBADA}[case["limiter"]]
    g = O.make_grid(1, case["n"], case["size"], periodic=[1])
    nloc = O.ghosted_shape(g)[0]
    comp = case["component"]
    i = np.arange(nloc, dtype=np.float64)
    phi = (i * comp) if case["field"] == "linear" else (i * i * comp)
    desc = O.AssemblyDesc(g, dt=0.0, vel=[case["vel"]], limiter=lim)
    diag, rhs, mask = O.assemble(desc, np.ascontiguousarray(phi))
    exp = _tvd_row(case["expected_face"])
    c = case["ordinal"]
    assert diag[O.E, c] == exp["E"]
    assert diag[O.W, c] == exp["W"]
    assert diag[O.C_, c] == exp["C"]
    if case["rhs_exact"]:
        assert rhs[c] == exp["rhs"]
    else:
        tol = case["rhs_eps_tol"] * np.finfo(np.float64).eps * max(abs(exp["rhs"]), 1.0)
        assert abs(rhs[c] - exp["rhs"]) <= tol


@pytest.mark.parametrize("case", GOLD["ddt"])
def test_ddt_known_answer(case):
    g = O.make_grid(3, case["n"], case["size"], periodic=[1, 1, 1])
    shape = O.ghosted_shape(g)
    phi_new = np.full(shape, case["phi_new"]).ravel()
    phi_old = np.full(shape, case["phi_old"]).ravel()
    desc = O.AssemblyDesc(g, dt=case["dt"])
    diag, rhs, _ = O.assemble(desc, phi_new, phi_old)
    assert abs(diag[O.C_, 0] - case["expected"]["C"]) <= case["abs_tol"]
    assert abs(rhs[0] - case["expected"]["rhs"]) <= case["abs_tol"]


def test_limiters_edge_cases():
    nan, inf = math.nan, math.inf
    # NaN -> 0 for MINMOD / VANALBADA (FluxLimiter.h:129,170)
    assert O.limiter(O.LIM_MINMOD, nan) == 0.0
    assert O.limiter(O.LIM_VANALBADA, nan) == 0.0
    assert O.limiter(O.LIM_MINMOD, inf) == 1.0
    assert O.limiter(O.LIM_MINMOD, -inf) == 0.0
    assert math.isnan(O.limiter(O.LIM_VANALBADA, inf))
    # van Leer (added): NaN -> 0, +inf -> 2, -inf -> 0, psi(1) = 1
    assert O.limiter(O.LIM_VANLEER, nan) == 0.0
    assert O.limiter(O.LIM_VANLEER, inf) == 2.0
    assert O.limiter(O.LIM_VANLEER, -inf) == 0.0
    assert O.limiter(O.LIM_VANLEER, 1.0) == 1.0
    assert O.limiter(O.LIM_VANLEER, -3.0) == 0.0
    assert O.limiter(O.LIM_CDS, 7.0) == 1.0
    assert O.limiter(O.LIM_UPWIND, 7.0) == 0.0


def test_numbering_last_dimension_fastest():
    g = O.make_grid(3, [5, 6, 7], num_ghost=2)
    lib = O.lib()
    import ctypes as C
    assert lib.dor_ordinal_internal(C.byref(g), 1, 2, 3) == (1 * 6 + 2) * 7 + 3
    # internal -> local adds num_ghost per dimension on the ghosted grid
    assert lib.dor_internal_to_local(C.byref(g), 0) == (2 * 10 + 2) * 11 + 2
    gp = O.make_grid(3, [5, 6, 7], periodic=[1, 0, 0])
    # periodic wrap (any periodic dimension wraps all, CartesianRepresentation.inl:432-443)
    assert lib.dor_global_internal_periodic(C.byref(gp), -1, 0, 0) == (4 * 6 + 0) * 7
    assert lib.dor_global_internal_periodic(C.byref(gp), 5, 0, 0) == 0


def test_halo_exchange_semantics():
    # 1D non-periodic (test_integration_Cartesian_Field.cpp:281-316, np=1):
    # physical ghosts are not touched
    g = O.make_grid(1, [10])
    phi = np.full(14, -7.0)
    phi[2:12] = 3.0
    O.exchange_halo(g, phi)
    assert np.all(phi[:2] == -7.0) and np.all(phi[12:] == -7.0)
    # periodic: face ghosts take the periodic image; edge/corner ghosts are
    # not part of the halo (CartesianRepresentation.inl:165-175)
    g2 = O.make_grid(2, [5, 4], periodic=[1, 1])
    sh = O.ghosted_shape(g2)
    phi2 = np.full(sh, -1.0)
    vals = np.arange(20, dtype=np.float64).reshape(5, 4)
    phi2[2:7, 2:6, 0] = vals
    flat = np.ascontiguousarray(phi2.ravel())
    O.exchange_halo(g2, flat)
    p = flat.reshape(sh)[:, :, 0]
    assert np.all(p[0:2, 2:6] == vals[3:5, :])
    assert np.all(p[7:9, 2:6] == vals[0:2, :])
    assert np.all(p[2:7, 0:2] == vals[:, 2:4])
    assert np.all(p[2:7, 6:8] == vals[:, 0:2])
    assert np.all(p[0:2, 0:2] == -1.0) and np.all(p[7:9, 6:8] == -1.0)


def _structured_csr(dim, n, rows_fn):
    """CSR from a per-cell functor returning {slot: value} and rhs (global
    ordinals, last dimension fastest, sorted columns)."""
    nn = list(n) + [1] * (3 - dim)
    ncell = nn[0] * nn[1] * nn[2]
    offs = {O.W: (-1, 0, 0), O.E: (1, 0, 0), O.S: (0, -1, 0), O.N: (0, 1, 0),
            O.B: (0, 0, -1), O.T: (0, 0, 1), O.C_: (0, 0, 0)}
    rowptr = [0]
    cols, vals = [], []
    b = np.zeros(ncell)
    x0 = np.zeros(ncell)
    for i in range(nn[0]):
        for j in range(nn[1]):
            for k in range(nn[2]):
                entries, rhs, guess = rows_fn((i, j, k), nn)
                row = []
                for slot, v in entries.items():
                    o = offs[slot]
                    row.append((((i + o[0]) * nn[1] + (j + o[1])) * nn[2] + (k + o[2]), v))
                row.sort()
                for cidx, v in row:
                    cols.append(cidx)
                    vals.append(v)
                rowptr.append(len(cols))
                c = (i * nn[1] + j) * nn[2] + k
                b[c] = rhs
                x0[c] = guess
    return (np.array(rowptr, dtype=np.int64), np.array(cols, dtype=np.int64),
            np.array(vals, dtype=np.float64), b, x0)


def scalar_x_functor(dim, west=0.0, east=1.0):
    """test_integration_Cartesian_Trilinos.cpp SolveScalar(X) (1D :99-130,
    2D :245-294, 3D :602-672): center 2*dim, neighbours -1, Dirichlet mirror
    on W/E (C += 1, rhs = 2*value), Neumann on the rest (C -= 1)."""
    def fn(ind, nn):
        e = {O.C_: 2.0 * dim}
        rhs, guess = 0.0, 0.0
        for d in range(dim):
            lo, hi = (O.W, O.E) if d == 0 else ((O.S, O.N) if d == 1 else (O.B, O.T))
            for slot, edge, val in ((lo, ind[d] == 0, west), (hi, ind[d] == nn[d] - 1, east)):
                if not edge:
                    e[slot] = -1.0
                elif d == 0:
                    e[O.C_] += 1.0
                    rhs = 2.0 * val
                    guess = val
                else:
                    e[O.C_] -= 1.0
        return e, rhs, guess
    return fn


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("precond", [O.PREC_NONE, O.PREC_JACOBI])
def test_bicgstab2_linear_profile(dim, precond):
    n = [20 + d for d in range(dim)]
    rowptr, cols, vals, b, x0 = _structured_csr(dim, n, scalar_x_functor(dim))
    x, info = O.bicgstab2(rowptr, cols, vals, b, x0, tol=1e-14, max_it=5000, precond=precond)
    assert info["converged"]
    nn = n + [1] * (3 - dim)
    i = np.repeat(np.arange(nn[0]), nn[1] * nn[2])
    expect = 0.0 + (i + 0.5) * (1.0 / nn[0])
    assert np.max(np.abs(x - expect)) < 1e-8


def test_bicgstab2_coupled_components():
    """MatrixSystem/test/test_TrilinosSolver.cpp:98-205: pseudo-2D Laplace
    with N=4 interleaved components on 21+2 cells, tolerance 1e-12."""
    ncomp, ncell = 4, 23
    rowptr, cols, vals = [0], [], []
    b = np.zeros(ncell * ncomp)
    x0 = np.full(ncell * ncomp, 0.5)
    for node in range(ncell):
        for n in range(ncomp):
            row = node * ncomp + n
            ent = {}
            if node == 0:
                ent[row] = 3.0
                ent[row + ncomp] = -1.0
                b[row] = 0.0
                x0[row] = 0.0
            elif node == ncell - 1:
                ent[row - ncomp] = -1.0
                ent[row] = 3.0
                b[row] = 2.0
                x0[row] = 1.0
            else:
                ent[row - ncomp] = -1.0
                ent[row] = 2.0
                ent[row + ncomp] = -1.0
            if n != 0:
                ent[row - 1] = -1.0
                ent[row] += 1
            if n != ncomp - 1:
                ent[row + 1] = -1.0
                ent[row] += 1
            for cidx in sorted(ent):
                cols.append(cidx)
                vals.append(ent[cidx])
            rowptr.append(len(cols))
    for precond in (O.PREC_NONE, O.PREC_JACOBI):
        x, info = O.bicgstab2(np.array(rowptr, dtype=np.int64), np.array(cols, dtype=np.int64),
                              np.array(vals), b, x0, tol=1e-12, max_it=5000, precond=precond)
        assert info["converged"]
        node = np.repeat(np.arange(ncell), ncomp)
        assert np.max(np.abs(x - (node + 0.5) / ncell)) < 1e-8


def test_csr_export_pattern_and_order():
    g = O.make_grid(3, [4, 5, 6], periodic=[1, 0, 0])
    bc = {O.S: (O.BC_DIRICHLET, 1.0), O.N: (O.BC_NEUMANN, 0.0),
          O.B: (O.BC_NEUMANN, 0.0), O.T: (O.BC_DIRICHLET, 0.0)}
    desc = O.AssemblyDesc(g, dt=0.01, D=1e-3, bc=bc)
    phi = np.random.default_rng(0).random(O.ghosted_shape(g)).ravel()
    diag, rhs, mask = O.assemble(desc, phi)
    rowptr, cols, vals = O.export_csr(g, diag, mask)
    assert rowptr[-1] == int(sum(bin(m).count("1") for m in mask))
    for r in range(len(rowptr) - 1):
        cc = cols[rowptr[r]:rowptr[r + 1]]
        assert np.all(np.diff(cc) > 0)                 # sorted, unique
        assert r in cc                                 # diagonal present
    # periodic x wrap: cell (0,2,2) couples to (3,2,2)
    c = (0 * 5 + 2) * 6 + 2
    assert (3 * 5 + 2) * 6 + 2 in cols[rowptr[c]:rowptr[c + 1]]
    # removed S neighbour at j == 0
    c0 = (1 * 5 + 0) * 6 + 3
    assert len(cols[rowptr[c0]:rowptr[c0 + 1]]) == 6


def test_diffusion_analytical_series():
    # Diffusion.h:46-58: at tau -> large, phi -> 1; at zeta = 1 the series vanishes
    assert abs(O.diffusion_n0d1(30.0, 0.3) - 1.0) < 1e-12
    assert abs(O.diffusion_n0d1(0.05, 1.0) - 1.0) < 1e-12
    assert 0.0 < O.diffusion_n0d1(0.05, 0.0) < 0.1
