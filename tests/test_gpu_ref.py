"""GPU parity against the reference's own code, without the oracle between.

oracle/_ref/libdare_ref.so is the reference's assembly (DDT, Gradient,
Divergence, TVD, MatrixBlock, Finalize through Trilinos<SC>::BuildNew's
per-cell loop) and its BiCGStab2, compiled from its own sources against
single-rank stand-ins for MPI / Kokkos / Tpetra / Belos / Teuchos.  Here the
CUDA path, through the C ABI, meets it directly: CSR pattern and right-hand
side bit for bit, coefficients bit for bit on 1-D / 2-D grids and within
1e-13 relative on 3-D grids (the 3-D kernel contracts to FMA), solutions of
whole time loops within 1e-9 relative L2.  Cases are those the reference's
code runs as stated: scalar or face diffusivity, a constant velocity.
"""
import numpy as np
import pytest

import dare_b200 as D
from dare_b200 import workloads as W
from oracle import ref as R
from tests.helpers import assert_coef_close, ref_timeloop, rel_l2
from tests.test_gpu_parity import _gpu_case, _gpu_timeloop

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (the reference's sources are absent)")]

SOL_TOL = 1e-9


@pytest.fixture(scope="module")
def ctx():
    c = D.Context(0)
    yield c
    c.synchronize()


def _case(seed):
    rng = np.random.default_rng(2000 + seed)
    dim = 1 + seed % 3
    periodic = tuple(int(rng.integers(0, 2)) for _ in range(dim))
    n = tuple(int(rng.integers(4, 12 if dim == 3 else 24)) for _ in range(dim))
    if dim == 3:
        n = (n[0], n[1], 8 * int(rng.integers(1, 9)) + int(rng.integers(0, 3)))   # several assembly tiles
    shape = tuple(x + 4 for x in n) + (1,) * (3 - dim)
    phi = rng.normal(size=shape)
    if seed % 3 == 2:
        phi = np.round(phi)                     # equal neighbours: r = 0/0 and x/0 in the limiters
    bc = {}
    for q in range(dim):
        if not periodic[q]:
            for side in range(2):
                bc[2 * q + 1 + side] = (int(rng.integers(1, 3)), float(rng.uniform(-1, 1)))
    return {"n": n, "size": tuple(1.0 + 0.25 * q for q in range(dim)), "periodic": periodic,
            "dt": float(10.0 ** rng.uniform(-3, -1)), "D": float(10.0 ** rng.uniform(-4, -2)),
            "vel": tuple(float(rng.uniform(-1, 1)) for _ in range(dim)),
            "limiter": ["CDS", "UPWIND", "VANALBADA", "MINMOD", "VANLEER"][seed % 5],
            "phi0": phi, "phi_old": rng.normal(size=shape), "bc": bc}


@pytest.mark.parametrize("seed", range(15))
def test_assembly_matches_reference_code(ctx, seed):
    case = _case(seed)
    g, f, s, asm, keep, dim = _gpu_case(ctx, case)
    s.build(f, asm)
    rp, cols, vals = s.export_csr()
    _, rhs = s.coefficients()
    x0 = s.solution()
    phi = np.ascontiguousarray(case["phi0"].reshape(-1))
    old = np.ascontiguousarray(case["phi_old"].reshape(-1))
    rrp, rcols, rvals, rrhs, rx0 = R.assemble(dim, case["n"], case["size"], case["periodic"], phi, old,
                                              dt=case["dt"], D=case["D"], vel=case["vel"], limiter=case["limiter"],
                                              bc=case["bc"])
    np.testing.assert_array_equal(rp, rrp)
    np.testing.assert_array_equal(cols, rcols)
    np.testing.assert_array_equal(x0, rx0)
    if dim == 3:
        assert_coef_close(vals, rvals)
        assert_coef_close(rhs, rrhs)
    else:
        np.testing.assert_array_equal(vals, rvals)
        np.testing.assert_array_equal(rhs, rrhs)


def test_gaussian_diffusion_loop_matches_reference_code(ctx):
    """The 64^3 Gaussian-diffusion workload's loop (Dirichlet 1 / 0 on x,
    Neumann elsewhere) at 24^3, 10 steps: the reference's assembly and
    BiCGStab2 against the GPU time step."""
    case = W.gaussian_diffusion(n=24, seed=5, steps=10)
    hist, iters, _ = _gpu_timeloop(ctx, case, case["steps"])
    rhist, riters, _ = ref_timeloop(case, case["steps"])
    for k in range(case["steps"]):
        assert rel_l2(hist[k], rhist[k]) < SOL_TOL, k
        assert abs(iters[k] - riters[k]) <= 2


def test_constant_velocity_tvd_loop_matches_reference_code(ctx):
    """Periodic 3-D convection-diffusion with a constant velocity and van
    Leer, 5 steps, against the reference's code."""
    rng = np.random.default_rng(8)
    n = (20, 18, 24)
    phi = rng.random(tuple(x + 4 for x in n))
    case = {"n": n, "size": (1.0, 1.0, 1.0), "periodic": (1, 1, 1), "dt": 0.02, "D": 1e-3,
            "vel": (0.4, -0.3, 0.2), "limiter": "VANLEER", "phi0": phi}
    from oracle import oracle as O
    O.exchange_halo(O.make_grid(3, n, (1.0, 1.0, 1.0), 2, (1, 1, 1)), case["phi0"].reshape(-1))
    hist, iters, _ = _gpu_timeloop(ctx, case, 5)
    rhist, riters, _ = ref_timeloop(case, 5)
    for k in range(5):
        assert rel_l2(hist[k], rhist[k]) < SOL_TOL, k
        assert abs(iters[k] - riters[k]) <= 2


@pytest.mark.parametrize("dim", [2, 3])
def test_two_component_system_matches_reference_code(ctx, dim):
    """Two field components with their own conditions (Dirichlet on one where
    the other is Neumann, as the counter-diffusion driver folds them): the
    GPU's interleaved system (rows cell * 2 + c) against the reference's
    MatrixBlock<Grid, GO, SC, 2>."""
    rng = np.random.default_rng(60 + dim)
    n = (7, 9) if dim == 2 else (6, 7, 40)
    periodic = (1, 0) if dim == 2 else (0, 1, 0)
    shape = tuple(x + 4 for x in n) + (1,) * (3 - dim)
    comps = [rng.normal(size=shape) for _ in range(2)]
    olds = [rng.normal(size=shape) for _ in range(2)]
    bc0, bc1 = {}, {}
    for q in range(dim):
        if not periodic[q]:
            bc0[2 * q + 1], bc0[2 * q + 2] = (1, 1.0), (2, 0.0)
            bc1[2 * q + 1], bc1[2 * q + 2] = (2, 0.0), (1, 1.0)
    vel = tuple(float(v) for v in rng.uniform(-0.5, 0.5, size=dim))
    size = tuple(1.0 for _ in range(dim))
    inter = lambda arrs: np.stack([a.reshape(-1) for a in arrs], axis=-1).reshape(-1)
    g = D.Grid(ctx, n, size, 2, periodic)
    f = D.Field(g, 2, components=2)
    f.upload(inter(comps), 0)
    f.upload(inter(olds), 1)
    s = D.MatrixSystem(g, components=2)
    for c, bc in enumerate((bc0, bc1)):
        for face, (kind, val) in bc.items():
            s.set_bc(face, kind, val, component=c)
    asm = D.Assembly(dt=1e-2, D=2e-3, vel=vel, limiter="MINMOD")
    s.build(f, asm)
    rp, cols, vals = s.export_csr()
    _, rhs = s.coefficients()
    x0 = s.solution()
    rrp, rcols, rvals, rrhs, rx0 = R.assemble(dim, n, size, periodic,
                                              np.concatenate([np.ascontiguousarray(a.reshape(-1)) for a in comps]),
                                              np.concatenate([np.ascontiguousarray(a.reshape(-1)) for a in olds]),
                                              dt=1e-2, D=2e-3, vel=vel, limiter="MINMOD", bc=bc0, ncomp=2, bc1=bc1)
    np.testing.assert_array_equal(rp, rrp)
    np.testing.assert_array_equal(cols, rcols)
    np.testing.assert_array_equal(x0, rx0)
    if dim == 3:
        assert_coef_close(vals, rvals)
        assert_coef_close(rhs, rrhs)
    else:
        np.testing.assert_array_equal(vals, rvals)
        np.testing.assert_array_equal(rhs, rrhs)
